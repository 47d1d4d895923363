"""The feasibility pump loop with the B200 projector and root-LP solver.

Host-side mirror of src/pump.jl:1-447: ``feasibility_pump`` and ``PumpResult``
keep the reference's keyword arguments, defaults, tolerance schedule, log lines
and counters.  The projector (``PDFPState``), the root LP
(``solve_lp_relaxation``) and the preconditioner (``scale_problem``) run on the
GPU through ``libpdfp_b200.so``; rounding, propagation, flips, perturbations
and cycle detection stay on the CPU.

``solvers`` selects the object that provides those three entry points; the
default is the GPU library.  Tests pass the CPU oracle here to run the same
pump loop against the reference's algorithm.
"""
from __future__ import annotations

import math
import sys
import time
from dataclasses import dataclass

import numpy as np

from .milp import MILP, is_integral, max_violation, num_constraints, num_continuous, num_variables
from .params import SolverParameters
from .rounding import Rounder, BatchPolicy, round_guarded, _round


@dataclass
class PumpResult:
    """Outcome of ``feasibility_pump`` (src/pump.jl:22-35)."""

    found: bool
    x: np.ndarray
    objective: float
    max_violation: float
    iterations: int
    perturbations: int
    pdhg_iterations: int
    root_lp_status: str
    root_lp_time: float
    projection_time: float
    rounding_time: float
    time: float


@dataclass
class PumpCounters:
    """src/pump.jl:40-48"""

    iterations: int = 0
    perturbations: int = 0
    pdhg_iterations: int = 0
    root_lp_status: str = "UNSPECIFIED"
    root_lp_time: float = 0.0
    projection_time: float = 0.0
    rounding_time: float = 0.0


def _differs(a, b, idx) -> bool:
    return bool(np.any(a[idx] != b[idx]))


def _round_to_nearest(x: np.ndarray, milp: MILP) -> np.ndarray:
    """Nearest integer on I, kept inside the bounds (src/pump.jl:53-62)."""
    xt = np.array(x, dtype=np.float64, copy=True)
    for j in milp.int_idx.tolist():
        v = _round(x[j])
        if math.isfinite(milp.l[j]) and v < milp.l[j]:
            v = float(math.ceil(milp.l[j]))
        if math.isfinite(milp.u[j]) and v > milp.u[j]:
            v = float(math.floor(milp.u[j]))
        xt[j] = v
    return xt


def _hash_integers(x: np.ndarray, int_idx: np.ndarray) -> int:
    """Hash of the integer coordinates for cycle detection (src/pump.jl:66-74); -0.0 == 0.0."""
    v = x[int_idx] + 0.0
    return hash(v.tobytes())


def _batch_schedule(milp: MILP, x, dual_slack, push_threshold: float) -> str:
    """src/pump.jl:81-93"""
    n_pushed = 0
    n_integral = 0
    for j in milp.int_idx.tolist():
        if abs(x[j] - _round(x[j])) != 0.0:
            continue
        n_integral += 1
        at_lower = math.isfinite(milp.l[j]) and abs(x[j] - milp.l[j]) < 1e-9
        at_upper = math.isfinite(milp.u[j]) and abs(x[j] - milp.u[j]) < 1e-9
        if (at_lower and dual_slack[j] > 0) or (at_upper and dual_slack[j] < 0):
            n_pushed += 1
    fraction = n_pushed / n_integral if n_integral > 0 else 1.0
    return "regroup" if fraction < push_threshold else "all"


def _total_integer_row_violation(milp: MILP, x: np.ndarray) -> float:
    """src/pump.jl:98-118"""
    activity = milp.A @ x
    is_int = milp.is_int
    A = milp.A.tocsc()
    skip = np.zeros(num_constraints(milp), dtype=bool)
    for j in np.nonzero(~is_int)[0].tolist():
        skip[A.indices[A.indptr[j]:A.indptr[j + 1]]] = True
    total = 0.0
    eq = milp.is_eq
    for i in range(num_constraints(milp)):
        if skip[i]:
            continue
        d = activity[i] - milp.b[i]
        total += abs(d) if eq[i] else max(0.0, d)
    return total


def _flip_farthest(xt, x, milp: MILP, TT: int) -> None:
    """FP's stalling move (src/pump.jl:121-135)."""
    l, u = milp.l, milp.u
    idx = milp.int_idx.tolist()
    distances = [(abs(x[j] - xt[j]), j) for j in idx]
    distances.sort(key=lambda t: t[0], reverse=True)  # stable, like sort!(; rev = true)
    for k in range(min(TT, len(distances))):
        d, j = distances[k]
        if d == 0.0:
            continue
        cur = xt[j]
        direction = 1.0 if x[j] >= cur else -1.0
        v = cur + direction
        if v < l[j] or v > u[j]:
            v = cur - direction
        if v < l[j] or v > u[j]:
            continue
        xt[j] = v


class RestartLadder:
    """src/pump.jl:139-144"""

    def __init__(self, flips, last_restart, average_flips, max_flips):
        self.flips = float(flips)
        self.last_restart = last_restart
        self.average_flips = average_flips
        self.max_flips = max_flips


def _perturb(xt, x, milp: MILP, rng, general, is_general, ladder: RestartLadder,
             iteration: int) -> None:
    """FP's restart (src/pump.jl:149-187)."""
    l, u = milp.l, milp.u
    if general:
        while ladder.last_restart < iteration:
            ladder.last_restart += 1
            ladder.flips *= 0.85
        ladder.flips = min(ladder.flips + 2 * ladder.average_flips + 1, ladder.max_flips)
        for _ in range(max(1, int(math.floor(ladder.flips)))):
            j = general[int(rng.integers(0, len(general)))]
            lo, hi = l[j], u[j]
            r = float(rng.random())
            if math.isfinite(hi - lo) and hi - lo < 1e15:
                v = math.floor(lo + (1.0 + hi - lo) * r)
            elif math.isfinite(lo) and xt[j] - lo < 1e9:
                v = lo + (2e9 - 1.0) * r
            elif math.isfinite(hi) and hi - xt[j] < 1e9:
                v = hi - (2e9 - 1.0) * r
            else:
                v = xt[j] + (2e9 - 1.0) * r - 1e9
            v = _round(min(max(v, lo), hi))
            if abs(v - xt[j]) > 1e-6:
                xt[j] = v
    for j in milp.int_idx.tolist():
        if is_general[j]:
            continue
        rho = -0.3 + float(rng.random())
        if abs(x[j] - xt[j]) + max(rho, 0.0) > 0.5:
            cur = xt[j]
            direction = 1.0 if x[j] >= cur else -1.0
            v = cur + direction
            if v < l[j] or v > u[j]:
                v = cur - direction
            if v < l[j] or v > u[j]:
                continue
            xt[j] = v


DEVICE_CHECK_MIN_NNZ = 1 << 16  # smaller matrices are checked on the host


class _ColumnScaling:
    """The projector's column scaling (src/pump.jl:305-306, 331, 338, 354).

    The pump hands the projector x ./ D_c and x_tilde ./ D_c and reads back
    D_c .* s.pdhg_x.  Projectors that hold D_c themselves (set_col_scale; the
    library's PDFPState and PDFPBatch) do both on the device, bit-identical to
    the host arithmetic, which then never touches the n-vector; for any other
    projector this object does it on the host.  `member` selects a batch member.
    """

    def __init__(self, projector, D_c, member=None):
        self.proj, self.D_c, self.member = projector, D_c, member
        self.device = hasattr(projector, "set_col_scale")
        if self.device:
            self._call("set_col_scale", D_c)

    def _call(self, name, *args):
        f = getattr(self.proj, name)
        return f(*args) if self.member is None else f(self.member, *args)

    def set_x(self, x):
        if self.device:
            self._call("set_x_unscaled", x)
        else:
            self._call("set_x", x / self.D_c)

    def set_target(self, xt):
        if self.device:
            self._call("set_target_unscaled", xt)
        else:
            self._call("set_target", xt / self.D_c)

    def x(self):
        if self.device:
            return self._call("get_unscaled", "pdhg_x")
        if self.member is None:
            return self.D_c * self.proj.pdhg_x
        return self.D_c * self.proj.get(self.member, "pdhg_x")


def _violation_fn(milp: MILP, solvers):
    """max_violation(milp, .) for the pump loop: on the device (bit-identical) when the
    solvers offer it and the matrix is large enough for the copy of x to pay."""
    if milp.A.nnz >= DEVICE_CHECK_MIN_NNZ and hasattr(solvers, "ConstraintChecker"):
        checker = solvers.ConstraintChecker(milp)
        return checker.max_violation
    return lambda x: max_violation(milp, x)


def _log(s: str) -> None:
    sys.stdout.write(s)


def _print_header(milp: MILP, device_name: str) -> None:
    """src/pump.jl:437-443"""
    _log("PDFP feasibility pump: %s\n" % milp.name)
    _log("model       %d rows, %d columns (%d integer, %d continuous), %d nonzeros\n" % (
        num_constraints(milp), num_variables(milp), len(milp.int_idx), num_continuous(milp),
        milp.A.nnz))
    _log("device      %s\n" % device_name)


def _fmt_g(v: float, width: int, prec: int) -> str:
    return ("%" + str(width) + "." + str(prec) + "g") % v


def _print_iteration(iteration, distance, violation, inner, gap, action, t) -> None:
    """``%6d %12.6g %10.3g %10d %9.2e %8s %8.2fs`` (src/pump.jl:445-447)."""
    _log("%6d %12.6g %10.3g %10d %9.2e %8s %8.2fs\n" % (
        iteration, distance, violation, inner, gap, action, t))


def _finish(milp, found, xt, stats: PumpCounters, t, verbose) -> PumpResult:
    """src/pump.jl:412-430"""
    violation = max_violation(milp, xt)
    objective = float(np.dot(milp.c, xt) + milp.c0)
    if verbose:
        if found:
            _log("FEASIBLE    objective %.10g after %d iterations, %.2f s\n" % (
                objective, stats.iterations, t))
        else:
            _log("NOT FOUND   after %d iterations, %.2f s (max violation %.3g)\n" % (
                stats.iterations, t, violation))
        _log("            root LP %.2f s, projections %.2f s, rounding %.2f s\n" % (
            stats.root_lp_time, stats.projection_time, stats.rounding_time))
    return PumpResult(found, xt, objective, violation, stats.iterations, stats.perturbations,
                      stats.pdhg_iterations, stats.root_lp_status, stats.root_lp_time,
                      stats.projection_time, stats.rounding_time, t)


def feasibility_pump(milp: MILP, *, time_limit: float = 1800.0, seed: int = 1,
                     use_gpu: bool = True, verbose: bool = False, flip_parameter: int = 20,
                     restart_period: int = 100, swap_iteration: int = 10,
                     gap_start: float = 1e-2, gap_decay: float = 0.98, gap_floor: float = 1e-4,
                     residual_ratio: float = 0.1, root_lp_tolerance: float = 1e-2,
                     projection_iteration_limit: int = 500_000, batch_policy: str = "cost",
                     push_threshold: float = 0.01, violation_threshold: float = 5000.0,
                     propagation_budget: int = 100_000, feasibility_tolerance: float = 1e-6,
                     precision: str = "fp64", solvers=None) -> PumpResult:
    """Search for a feasible solution of ``milp`` with the feasibility pump (src/pump.jl:231-410).

    Keyword arguments and defaults are the reference's.  ``use_gpu=False`` is
    refused: the CPU path is the reference's own and is not shipped here.
    ``precision`` picks the projector's arithmetic (``"fp64"`` or ``"mixed"``).
    """
    if batch_policy not in ("cost", "always"):
        raise ValueError("batch_policy must be 'cost' or 'always'")
    if solvers is None:
        if not use_gpu:
            raise ValueError("this library runs the pump's solvers on the GPU only (use_gpu=True)")
        from . import gpu as solvers  # noqa: PLC0415  (loads libpdfp_b200.so, fails loudly)
    t0 = time.time()

    def elapsed():
        return time.time() - t0

    def remaining():
        return max(time_limit - elapsed(), 1.0)

    n, m = num_variables(milp), num_constraints(milp)
    int_idx = milp.int_idx
    tol = feasibility_tolerance
    mixed = num_continuous(milp) > 0
    rng = np.random.Generator(np.random.PCG64(seed))
    rounder = Rounder(milp, max_pops=(2**62 if mixed else propagation_budget),
                      swap_iteration=swap_iteration,
                      policy=BatchPolicy() if batch_policy == "cost" else None)
    stats = PumpCounters()
    viol = _violation_fn(milp, solvers)
    if verbose:
        _print_header(milp, solvers.device_name())

    # Root LP relaxation (src/pump.jl:268-278).
    x, dual_slack, stats.root_lp_status, root_iterations = solvers.solve_lp_relaxation(
        milp, tolerance=root_lp_tolerance, time_limit=remaining(), cupdlpx_termination=mixed)
    stats.root_lp_time = elapsed()
    if verbose:
        _log("root LP     %s after %d iterations, %.2f s\n" % (
            stats.root_lp_status, root_iterations, stats.root_lp_time))
    if is_integral(x, int_idx, tol):
        xt = _round_to_nearest(x, milp)
        if max_violation(milp, xt) <= tol:
            return _finish(milp, True, xt, stats, elapsed(), verbose)

    # First rounding, then the decision on the violation-guided rule (:280-291).
    rounder.schedule = _batch_schedule(milp, x, dual_slack, push_threshold)
    t = time.time()
    xt = round_guarded(rounder, x, rng, 0)
    stats.rounding_time += time.time() - t
    total_violation = _total_integer_row_violation(milp, xt)
    if total_violation >= violation_threshold:
        direction = [False] * n
        for j in int_idx.tolist():
            direction[j] = True
        rounder.direction = direction
    if verbose:
        _log("rounder     %s schedule, violation-guided rounding %s (first rounding violates by %.4g)\n" % (
            rounder.schedule, "off" if rounder.direction is None else "on", total_violation))

    # The projector (:293-307), built once -- at the first projection, so that a run
    # whose first rounding is already feasible does not pay for it.
    def build_projector():
        is_eq = milp.is_eq
        is_int = milp.is_int
        con_lb = np.where(is_eq, milp.b, -np.inf)
        sp_ = solvers.scale_problem(milp.A, np.zeros(n), milp.l.copy(), milp.u.copy(), con_lb,
                                    milp.b.copy(), bound_objective_rescaling=False)
        D_c = sp_.D_c
        weights = np.ones(n)
        weights[int_idx] = D_c[int_idx]
        proj = solvers.PDFPState(sp_.A, sp_.con_ub, is_eq, is_int, sp_.var_lb, sp_.var_ub,
                                 weights, precision=precision)
        if mixed:
            proj.original_primal_residual(sp_.D_r)
        sc = _ColumnScaling(proj, D_c)
        sc.set_x(x)
        return proj, sc

    projector = scaling = None
    primal_weight = math.sqrt(1.0 + (len(int_idx) / m if m > 0 else 0.0))
    gap = gap_start
    tightening_budget = gap_start

    general = [j for j in int_idx.tolist() if not (milp.l[j] == 0.0 and milp.u[j] == 1.0)]
    is_general = np.zeros(n, dtype=bool)
    is_general[general] = True
    ladder = RestartLadder(0.0, 0, flip_parameter, max(len(general) // 10, 10))
    seen: set = set()
    h_current = _hash_integers(xt, int_idx)
    since_restart = 0

    if verbose:
        _log("%6s %12s %10s %10s %9s %8s %9s\n" % (
            "iter", "distance", "violation", "pdhg", "gap tol", "action", "time"))
    while elapsed() < time_limit:
        violation = viol(xt)
        if violation <= tol and is_integral(xt, int_idx, tol):
            return _finish(milp, True, xt.copy(), stats, elapsed(), verbose)
        stats.iterations += 1
        iteration = stats.iterations
        since_restart += 1

        # Project x~ onto the LP relaxation (:329-363).
        if projector is None:
            projector, scaling = build_projector()
        t = time.time()
        scaling.set_target(xt)
        gap_used = gap
        params = SolverParameters(iteration_limit=projection_iteration_limit,
                                  eps_optimal_relative=gap,
                                  eps_feasible_relative=gap * residual_ratio,
                                  time_limit=remaining())
        projector.solve(params, primal_weight)
        x = scaling.x()
        inner = projector.total_count
        while (mixed and tightening_budget > 1e-6 and elapsed() < time_limit
               and is_integral(x, int_idx, tol)
               and viol(_round_to_nearest(x, milp)) > tol):
            tightening_budget *= 0.1
            gap = max(gap * 0.1, 1e-8)
            params = SolverParameters(iteration_limit=projection_iteration_limit,
                                      eps_optimal_relative=gap,
                                      eps_feasible_relative=gap * residual_ratio,
                                      time_limit=remaining())
            projector.warm_start()
            projector.solve(params, primal_weight)
            x = scaling.x()
            inner += projector.total_count
        stats.pdhg_iterations += inner
        if gap > gap_floor:
            gap = max(gap * gap_decay, gap_floor)
        stats.projection_time += time.time() - t
        distance = float(np.sum(np.abs(x[int_idx] - xt[int_idx]))) if len(int_idx) else 0.0

        if is_integral(x, int_idx, tol):
            candidate = _round_to_nearest(x, milp)
            if viol(candidate) <= tol:
                if verbose:
                    _print_iteration(iteration, distance, violation, inner, gap_used, "integral",
                                     elapsed())
                return _finish(milp, True, candidate, stats, elapsed(), verbose)

        # Round x; if the rounding did not change, flip (:373-385).
        t = time.time()
        x_round = round_guarded(rounder, x, rng, iteration)
        stats.rounding_time += time.time() - t
        candidate = xt.copy()
        action = "round"
        if _differs(x_round, xt, int_idx):
            candidate[:] = x_round
        else:
            flips = int(rng.integers(flip_parameter // 2, 3 * flip_parameter // 2 + 1))
            _flip_farthest(candidate, x, milp, flips)
            action = "flip"

        # Restart on a cycle and periodically (:387-404).
        h_candidate = _hash_integers(candidate, int_idx)
        cycled = h_candidate in seen
        periodic = since_restart >= restart_period
        if cycled or periodic:
            _perturb(candidate, x, milp, rng, general, is_general, ladder, iteration)
            stats.perturbations += 1
            since_restart = 0
            for _ in range(10):
                h = _hash_integers(candidate, int_idx)
                if not (h in seen or h == h_current):
                    break
                _perturb(candidate, x, milp, rng, general, is_general, ladder, iteration)
            action = "cycle" if cycled else "restart"
        seen.add(h_current)
        h_current = _hash_integers(candidate, int_idx) if (cycled or periodic) else h_candidate
        xt = candidate
        if verbose and (iteration <= 10 or iteration % 10 == 0):
            _print_iteration(iteration, distance, violation, inner, gap_used, action, elapsed())
    found = max_violation(milp, xt) <= tol and is_integral(xt, int_idx, tol)
    return _finish(milp, found, xt, stats, elapsed(), verbose)


@dataclass
class TrajectoryResult:
    """One trajectory of a batched pump run."""

    seed: int
    found: bool
    iterations: int
    perturbations: int
    pdhg_iterations: int
    time_to_feasible: float


class _Trajectory:
    """The CPU-side state of one pump trajectory (src/pump.jl:262-316)."""

    def __init__(self, milp, seed, x, dual_slack, push_threshold, violation_threshold,
                 propagation_budget, swap_iteration, batch_policy, flip_parameter, mixed):
        n = num_variables(milp)
        self.seed = seed
        self.rng = np.random.Generator(np.random.PCG64(seed))
        self.rounder = Rounder(milp, max_pops=(2**62 if mixed else propagation_budget),
                               swap_iteration=swap_iteration,
                               policy=BatchPolicy() if batch_policy == "cost" else None)
        self.rounder.schedule = _batch_schedule(milp, x, dual_slack, push_threshold)
        self.xt = round_guarded(self.rounder, x, self.rng, 0)
        if _total_integer_row_violation(milp, self.xt) >= violation_threshold:
            direction = [False] * n
            for j in milp.int_idx.tolist():
                direction[j] = True
            self.rounder.direction = direction
        self.general = [j for j in milp.int_idx.tolist() if not (milp.l[j] == 0.0 and milp.u[j] == 1.0)]
        self.is_general = np.zeros(n, dtype=bool)
        self.is_general[self.general] = True
        self.ladder = RestartLadder(0.0, 0, flip_parameter, max(len(self.general) // 10, 10))
        self.seen: set = set()
        self.h_current = _hash_integers(self.xt, milp.int_idx)
        self.since_restart = 0
        self.iterations = 0
        self.perturbations = 0
        self.pdhg = 0
        self.found = False
        self.x_found = None
        self.t_found = math.inf


def feasibility_pump_batched(milp: MILP, *, seeds=(101, 201), time_limit: float = 1800.0,
                             flip_parameter: int = 20, restart_period: int = 100,
                             swap_iteration: int = 10, gap_start: float = 1e-2,
                             gap_decay: float = 0.98, gap_floor: float = 1e-4,
                             residual_ratio: float = 0.1, root_lp_tolerance: float = 1e-2,
                             projection_iteration_limit: int = 500_000, batch_policy: str = "cost",
                             push_threshold: float = 0.01, violation_threshold: float = 5000.0,
                             propagation_budget: int = 100_000,
                             feasibility_tolerance: float = 1e-6, precision: str = "fp64",
                             solvers=None, stop=None, asynchronous: bool = False):
    """Concurrent pump trajectories as members of one batched projector.

    Replaces the reference's K concurrent pump processes (scripts/solve.jl:121-148,
    seeds 100k + seed) with K trajectories in one process: one root LP, one
    scaling, and per pump iteration one batched projection (one launch sequence
    for all trajectories, each with its own restart and termination state on the
    device).  Rounding, flips and restarts run per trajectory on the CPU with the
    reference's rules (src/pump.jl:320-406).  Returns (PumpResult of the first
    trajectory to find a feasible point -- or of trajectory 0 if none did --,
    list of TrajectoryResult).

    ``stop(done) -> bool``, when given, is called once at the head of every pump
    iteration with this process's own verdict (a trajectory succeeded or the time
    ran out) and decides whether to stop; the sharded driver uses it to agree on
    stopping across ranks.

    ``asynchronous=False`` runs the trajectories in lockstep: every pump iteration
    projects all of them and waits for the slowest.  ``asynchronous=True`` lets each
    trajectory advance at its own pace, as the reference's separate processes do:
    the batched projection returns as soon as one member's projection ends
    (``solve_any``), that trajectory rounds and asks for its next projection, and
    the others continue where they stopped.  Each trajectory takes exactly the
    steps it takes in lockstep; only which one finishes first, in time, can differ.
    """
    if batch_policy not in ("cost", "always"):
        raise ValueError("batch_policy must be 'cost' or 'always'")
    if len(seeds) < 1:
        raise ValueError("at least one trajectory seed is required")
    if solvers is None:
        from . import gpu as solvers  # noqa: PLC0415
    t0 = time.time()

    def elapsed():
        return time.time() - t0

    def remaining():
        return max(time_limit - elapsed(), 1.0)

    n, m = num_variables(milp), num_constraints(milp)
    int_idx = milp.int_idx
    tol = feasibility_tolerance
    mixed = num_continuous(milp) > 0
    stats = PumpCounters()
    viol = _violation_fn(milp, solvers)
    x, dual_slack, stats.root_lp_status, _ = solvers.solve_lp_relaxation(
        milp, tolerance=root_lp_tolerance, time_limit=remaining(), cupdlpx_termination=mixed)
    stats.root_lp_time = elapsed()
    K = len(seeds)
    if is_integral(x, int_idx, tol):
        xt = _round_to_nearest(x, milp)
        if max_violation(milp, xt) <= tol:
            res = _finish(milp, True, xt, stats, elapsed(), False)
            return res, [TrajectoryResult(s, True, 0, 0, 0, elapsed()) for s in seeds]
    trajs = [_Trajectory(milp, s, x, dual_slack, push_threshold, violation_threshold,
                         propagation_budget, swap_iteration, batch_policy, flip_parameter, mixed)
             for s in seeds]
    # the projector batch, built at the first projection (a run whose first roundings
    # are already feasible does not pay for it)
    def build_batch():
        is_eq, is_int = milp.is_eq, milp.is_int
        con_lb = np.where(is_eq, milp.b, -np.inf)
        sp_ = solvers.scale_problem(milp.A, np.zeros(n), milp.l.copy(), milp.u.copy(), con_lb,
                                    milp.b.copy(), bound_objective_rescaling=False)
        D_c = sp_.D_c
        weights = np.ones(n)
        weights[int_idx] = D_c[int_idx]
        ru = (1.0 / sp_.D_r) if mixed else None
        prob = (sp_.A, sp_.con_ub, is_eq, is_int, sp_.var_lb, sp_.var_ub, weights, ru)
        b = solvers.PDFPBatch([prob] * K, precision=precision)
        scs = [_ColumnScaling(b, D_c, p) for p in range(K)]
        for p in range(K):
            scs[p].set_x(x)
        return b, scs

    batch = scalings = None
    primal_weight = math.sqrt(1.0 + (len(int_idx) / m if m > 0 else 0.0))
    gaps = [gap_start] * K
    budgets = [gap_start] * K

    def params_for(p, active):
        return SolverParameters(iteration_limit=projection_iteration_limit if active else 0,
                                eps_optimal_relative=gaps[p],
                                eps_feasible_relative=gaps[p] * residual_ratio,
                                time_limit=remaining())

    def after_projection(p, xp, inner_p):
        """Trajectory p's steps after its projection xp (src/pump.jl:357-406): the
        tolerance schedule, the success test, rounding, flips and restarts.  True
        when the projection rounds to a feasible point."""
        tr = trajs[p]
        tr.pdhg += inner_p
        if gaps[p] > gap_floor:
            gaps[p] = max(gaps[p] * gap_decay, gap_floor)
        if is_integral(xp, int_idx, tol):
            cand = _round_to_nearest(xp, milp)
            if viol(cand) <= tol:
                tr.found, tr.x_found, tr.t_found = True, cand, elapsed()
                return True
        t = time.time()
        x_round = round_guarded(tr.rounder, xp, tr.rng, tr.iterations)
        stats.rounding_time += time.time() - t
        candidate = tr.xt.copy()
        if _differs(x_round, tr.xt, int_idx):
            candidate[:] = x_round
        else:
            flips = int(tr.rng.integers(flip_parameter // 2, 3 * flip_parameter // 2 + 1))
            _flip_farthest(candidate, xp, milp, flips)
        h_candidate = _hash_integers(candidate, int_idx)
        cycled = h_candidate in tr.seen
        periodic = tr.since_restart >= restart_period
        if cycled or periodic:
            _perturb(candidate, xp, milp, tr.rng, tr.general, tr.is_general, tr.ladder,
                     tr.iterations)
            tr.perturbations += 1
            tr.since_restart = 0
            for _ in range(10):
                h = _hash_integers(candidate, int_idx)
                if not (h in tr.seen or h == tr.h_current):
                    break
                _perturb(candidate, xp, milp, tr.rng, tr.general, tr.is_general, tr.ladder,
                         tr.iterations)
        tr.seen.add(tr.h_current)
        tr.h_current = _hash_integers(candidate, int_idx) if (cycled or periodic) else h_candidate
        tr.xt = candidate
        return False

    winner = None

    def trajectory(p):
        """Trajectory p as a generator: yields once per projection it needs, with its
        target (or warm start) already set on member p, and returns True when it
        found a feasible point (False when the time ran out)."""
        tr = trajs[p]
        while True:
            if viol(tr.xt) <= tol and is_integral(tr.xt, int_idx, tol):
                tr.found, tr.x_found, tr.t_found = True, tr.xt.copy(), elapsed()
                return True
            if elapsed() >= time_limit:
                return False
            tr.iterations += 1
            tr.since_restart += 1
            scalings[p].set_target(tr.xt)
            yield
            xp = scalings[p].x()
            inner_p = batch.results[p]["total_count"]
            # mixed models: tenfold tighter re-solves (src/pump.jl:343-356)
            while mixed and elapsed() < time_limit:
                if not (budgets[p] > 1e-6 and is_integral(xp, int_idx, tol)
                        and viol(_round_to_nearest(xp, milp)) > tol):
                    break
                budgets[p] *= 0.1
                gaps[p] = max(gaps[p] * 0.1, 1e-8)
                batch.warm_start(p)
                yield
                xp = scalings[p].x()
                inner_p += batch.results[p]["total_count"]
            if after_projection(p, xp, inner_p):
                return True

    if asynchronous:
        # the first roundings as the lockstep loop tests them, before any projection
        for p, tr in enumerate(trajs):
            if viol(tr.xt) <= tol and is_integral(tr.xt, int_idx, tol):
                tr.found, tr.x_found, tr.t_found = True, tr.xt.copy(), elapsed()
                winner = p
                break
        gens, want, running = [], [False] * K, set()

        def advance(p):  # run trajectory p to its next projection; True: it succeeded
            try:
                next(gens[p])
                want[p] = True
                return False
            except StopIteration as e:
                want[p] = False
                return bool(e.value)

        if winner is None:
            batch, scalings = build_batch()
            gens = [trajectory(p) for p in range(K)]
            for p in range(K):
                if advance(p):
                    winner = p
                    break
        while winner is None:
            done = elapsed() >= time_limit
            if (stop(done) if stop is not None else done):
                break
            new = [p for p in range(K) if want[p]]
            if not new and not running:
                break  # every trajectory ran out of time
            # members starting a projection get their parameters; running ones
            # resume (their entry is not read); idle ones get no iterations
            t = time.time()
            statuses = batch.solve_any([params_for(p, want[p]) for p in range(K)], primal_weight,
                                       resume=[p in running for p in range(K)])
            stats.projection_time += time.time() - t
            for p in new:
                want[p] = False
                running.add(p)
            for p in sorted(running):
                if statuses[p] == "RUNNING":
                    continue
                running.discard(p)
                if advance(p):
                    winner = p
                    break
    while not asynchronous:
        done = winner is not None or elapsed() >= time_limit
        if (stop(done) if stop is not None else done):
            break
        for p, tr in enumerate(trajs):
            if viol(tr.xt) <= tol and is_integral(tr.xt, int_idx, tol):
                tr.found, tr.x_found, tr.t_found = True, tr.xt.copy(), elapsed()
                winner = p
                break
        if winner is not None:
            continue
        if batch is None:
            batch, scalings = build_batch()
        for p, tr in enumerate(trajs):
            tr.iterations += 1
            tr.since_restart += 1
            scalings[p].set_target(tr.xt)
        t = time.time()
        batch.solve([params_for(p, True) for p in range(K)], primal_weight)
        xs = [scalings[p].x() for p in range(K)]
        inner = [batch.results[p]["total_count"] for p in range(K)]
        # mixed models: tenfold tighter re-solves (src/pump.jl:343-356), batched
        while mixed and elapsed() < time_limit:
            need = [p for p in range(K) if budgets[p] > 1e-6 and is_integral(xs[p], int_idx, tol)
                    and viol(_round_to_nearest(xs[p], milp)) > tol]
            if not need:
                break
            for p in need:
                budgets[p] *= 0.1
                gaps[p] = max(gaps[p] * 0.1, 1e-8)
                batch.warm_start(p)
            batch.solve([params_for(p, p in need) for p in range(K)], primal_weight)
            for p in need:
                xs[p] = scalings[p].x()
                inner[p] += batch.results[p]["total_count"]
        stats.projection_time += time.time() - t
        for p, tr in enumerate(trajs):
            if after_projection(p, xs[p], inner[p]):
                winner = p
                break
    best = trajs[winner] if winner is not None else trajs[0]
    stats.iterations = best.iterations
    stats.perturbations = best.perturbations
    stats.pdhg_iterations = best.pdhg
    xbest = best.x_found if best.found else best.xt
    found = best.found or (max_violation(milp, xbest) <= tol and is_integral(xbest, int_idx, tol))
    res = _finish(milp, found, xbest, stats, elapsed(), False)
    return res, [TrajectoryResult(tr.seed, tr.found, tr.iterations, tr.perturbations, tr.pdhg,
                                  tr.t_found) for tr in trajs]
