"""ctypes wrapper of the CPU FP64 oracle (liboracle_pdfp.so).

TEST INFRASTRUCTURE ONLY: the parity checker for the B200 library.  Only
tests/, ``__graft_entry__.smoke()`` and the CPU-baseline legs of ``bench.py``
import this module; the product package ``pdfp_b200`` never does.

The C library restates the reference's CPU path (src/preconditioner.jl,
src/pdfp.jl, src/pdlp.jl of MIT-Lu-Lab/PDFP); see pdfp_oracle.h.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass

import numpy as np
import scipy.sparse as sp

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle_pdfp.so")

STATUS = {0: "UNSPECIFIED", 1: "OPTIMAL", 2: "ITERATION_LIMIT", 3: "TIME_LIMIT",
          4: "PRIMAL_INFEASIBLE", 5: "DUAL_INFEASIBLE"}


class OrParams(C.Structure):
    _fields_ = [
        ("eps_optimal_relative", C.c_double),
        ("eps_feasible_relative", C.c_double),
        ("iteration_limit", C.c_int64),
        ("time_limit", C.c_double),
        ("termination_evaluation_frequency", C.c_int32),
        ("sv_max_iterations", C.c_int32),
        ("reflection_coefficient", C.c_double),
        ("sv_tolerance", C.c_double),
        ("artificial_restart_threshold", C.c_double),
        ("sufficient_reduction_for_restart", C.c_double),
        ("necessary_reduction_for_restart", C.c_double),
        ("k_p", C.c_double),
        ("k_i", C.c_double),
        ("k_d", C.c_double),
        ("i_smooth", C.c_double),
    ]


class OrResult(C.Structure):
    _fields_ = [
        ("status", C.c_int32),
        ("restarts", C.c_int32),
        ("total_count", C.c_int64),
        ("rel_primal", C.c_double),
        ("rel_dual", C.c_double),
        ("rel_gap", C.c_double),
        ("primal_weight", C.c_double),
        ("step_size", C.c_double),
        ("max_singular_value", C.c_double),
        ("fixed_point_error", C.c_double),
        ("objective_value", C.c_double),
    ]

    def as_dict(self) -> dict:
        d = {k: getattr(self, k) for k, _ in self._fields_}
        d["status"] = STATUS.get(self.status, str(self.status))
        return d


_lib = None


def build() -> str:
    """Compile the oracle with its Makefile (the checker, not the product)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        dp = C.POINTER(C.c_double)
        ip = C.POINTER(C.c_int32)
        up = C.POINTER(C.c_uint8)
        L.or_default_params.argtypes = [C.POINTER(OrParams)]
        L.or_normal_vector.argtypes = [C.c_uint64, C.c_int64, dp]
        L.or_scale_problem.argtypes = [C.c_int32, C.c_int32, ip, ip, dp, dp, dp, dp, dp, dp,
                                       C.c_int32, C.c_double, C.c_int32, dp, dp, dp, dp, dp, dp,
                                       dp, dp, dp, dp]
        L.or_estimate_max_singular_value.argtypes = [C.c_int32, C.c_int32, ip, ip, dp, C.c_int32,
                                                     C.c_double, ip]
        L.or_estimate_max_singular_value.restype = C.c_double
        L.or_pdfp_create.argtypes = [C.c_int32, C.c_int32, ip, ip, dp, dp, up, up, dp, dp, dp]
        L.or_pdfp_create.restype = C.c_void_p
        L.or_pdfp_destroy.argtypes = [C.c_void_p]
        L.or_pdfp_original_primal_residual.argtypes = [C.c_void_p, dp]
        L.or_pdfp_set_x.argtypes = [C.c_void_p, dp]
        L.or_pdfp_set_target.argtypes = [C.c_void_p, dp]
        L.or_pdfp_warm_start.argtypes = [C.c_void_p]
        L.or_pdfp_solve.argtypes = [C.c_void_p, C.POINTER(OrParams), C.c_double,
                                    C.POINTER(OrResult)]
        L.or_pdfp_solve.restype = C.c_int32
        L.or_pdfp_get.argtypes = [C.c_void_p, C.c_int32, dp]
        L.or_pdfp_steps.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_int32, C.c_int32]
        L.or_pdfp_set_max_singular_value.argtypes = [C.c_void_p, C.c_double]
        L.or_solve_lp_relaxation.argtypes = [C.c_int32, C.c_int32, ip, ip, dp, dp, dp, dp, dp, up,
                                             C.c_double, C.c_double, C.c_int32, dp, dp,
                                             C.POINTER(OrResult)]
        L.or_solve_lp_relaxation.restype = C.c_int32
        L.or_pdlp_solve_scaled.argtypes = [C.c_int32, C.c_int32, ip, ip, dp, dp, dp, dp, dp, dp,
                                           C.c_double, C.c_double, dp, dp, C.POINTER(OrParams),
                                           dp, dp, dp, C.POINTER(OrResult)]
        L.or_pdlp_solve_scaled.restype = C.c_int32
        L.or_set_threads.argtypes = [C.c_int32]
        L.or_get_threads.restype = C.c_int32
        _lib = L
    return _lib


def _d(a):
    return a.ctypes.data_as(C.POINTER(C.c_double)) if a is not None else None


def _i(a):
    return a.ctypes.data_as(C.POINTER(C.c_int32))


def _u(a):
    return a.ctypes.data_as(C.POINTER(C.c_uint8))


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _csr(A):
    A = sp.csr_matrix(A, dtype=np.float64)
    A.sort_indices()
    return (np.ascontiguousarray(A.indptr, dtype=np.int32),
            np.ascontiguousarray(A.indices, dtype=np.int32),
            np.ascontiguousarray(A.data, dtype=np.float64), A.shape)


def set_threads(k: int) -> None:
    lib().or_set_threads(int(k))


def get_threads() -> int:
    return int(lib().or_get_threads())


def default_params(**kw) -> OrParams:
    p = OrParams()
    lib().or_default_params(C.byref(p))
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def normal_vector(seed: int, m: int) -> np.ndarray:
    out = np.zeros(max(m, 1))
    lib().or_normal_vector(C.c_uint64(seed), m, _d(out))
    return out[:m]


@dataclass
class ScaledProblem:
    A: sp.csr_matrix
    c: np.ndarray
    var_lb: np.ndarray
    var_ub: np.ndarray
    con_lb: np.ndarray
    con_ub: np.ndarray
    D_r: np.ndarray
    D_c: np.ndarray
    bound_scale: float
    objective_scale: float


def scale_problem(A, c, var_lb, var_ub, con_lb, con_ub, ruiz_iterations=10,
                  pock_chambolle_alpha=1.0, bound_objective_rescaling=True) -> ScaledProblem:
    rp, ci, v, (m, n) = _csr(A)
    vals = np.zeros(max(len(v), 1))
    outs_n = [np.zeros(max(n, 1)) for _ in range(4)]
    outs_m = [np.zeros(max(m, 1)) for _ in range(3)]
    bs, os_ = C.c_double(), C.c_double()
    lib().or_scale_problem(m, n, _i(rp), _i(ci), _d(v), _d(_f64(c)), _d(_f64(var_lb)),
                           _d(_f64(var_ub)), _d(_f64(con_lb)), _d(_f64(con_ub)),
                           ruiz_iterations, pock_chambolle_alpha, int(bool(bound_objective_rescaling)),
                           _d(vals), _d(outs_n[0]), _d(outs_n[1]), _d(outs_n[2]), _d(outs_m[0]),
                           _d(outs_m[1]), _d(outs_m[2]), _d(outs_n[3]), C.byref(bs), C.byref(os_))
    As = sp.csr_matrix((vals[:len(v)].copy(), ci.copy(), rp.copy()), shape=(m, n))
    return ScaledProblem(As, outs_n[0][:n], outs_n[1][:n], outs_n[2][:n], outs_m[0][:m],
                         outs_m[1][:m], outs_m[2][:m], outs_n[3][:n], bs.value, os_.value)


def estimate_max_singular_value(A, max_iterations=5000, tolerance=1e-4):
    rp, ci, v, (m, n) = _csr(A)
    it = C.c_int32()
    s = lib().or_estimate_max_singular_value(m, n, _i(rp), _i(ci), _d(v), max_iterations,
                                             tolerance, C.byref(it))
    return s, it.value


class OraclePDFP:
    """PDFPState on the CPU oracle (src/pdfp.jl:60-76)."""

    def __init__(self, A, b, is_eq, is_int, var_lb, var_ub, w):
        rp, ci, v, (m, n) = _csr(A)
        self.m, self.n = m, n
        self._keep = [rp, ci, v]
        self.h = lib().or_pdfp_create(m, n, _i(rp), _i(ci), _d(v), _d(_f64(b)),
                                      _u(np.ascontiguousarray(is_eq, dtype=np.uint8)),
                                      _u(np.ascontiguousarray(is_int, dtype=np.uint8)),
                                      _d(_f64(var_lb)), _d(_f64(var_ub)), _d(_f64(w)))
        self.total_count = 0
        self.termination_reason = "UNSPECIFIED"
        self.last = None

    def __del__(self):
        if getattr(self, "h", None):
            lib().or_pdfp_destroy(self.h)
            self.h = None

    def original_primal_residual(self, D_r):
        lib().or_pdfp_original_primal_residual(self.h, _d(_f64(D_r)))

    def set_x(self, x):
        lib().or_pdfp_set_x(self.h, _d(_f64(x)))

    def set_target(self, x_tilde):
        lib().or_pdfp_set_target(self.h, _d(_f64(x_tilde)))
        self.total_count = 0

    def warm_start(self):
        lib().or_pdfp_warm_start(self.h)
        self.total_count = 0

    def solve(self, params: OrParams, primal_weight: float) -> str:
        r = OrResult()
        lib().or_pdfp_solve(self.h, C.byref(params), primal_weight, C.byref(r))
        self.last = r.as_dict()
        self.total_count = r.total_count
        self.termination_reason = STATUS[r.status]
        return self.termination_reason

    def get(self, which: str) -> np.ndarray:
        code = {"pdhg_x": 0, "pdhg_y": 1, "pdhg_z": 2, "current_x": 3, "current_y": 4,
                "current_z": 5, "dual_slack": 6, "reflected_x": 7}[which]
        size = self.m if which.endswith("_z") else self.n
        out = np.zeros(max(size, 1))
        lib().or_pdfp_get(self.h, code, _d(out))
        return out[:size]

    @property
    def pdhg_x(self):
        return self.get("pdhg_x")

    def steps(self, step_size, primal_weight, k0, count):
        lib().or_pdfp_steps(self.h, step_size, primal_weight, k0, count)

    def set_max_singular_value(self, sigma):
        """Seed the per-run ||A||_2 cache (src/pdfp.jl:225-229) with a known estimate."""
        lib().or_pdfp_set_max_singular_value(self.h, float(sigma))


def solve_lp_relaxation(milp, tolerance=1e-2, time_limit=3600.0, cupdlpx_termination=False):
    """solve_lp_relaxation on the oracle: (x, dual_slack, status, iterations, result)."""
    rp, ci, v, (m, n) = _csr(milp.A)
    is_le = np.array([s == "le" for s in milp.row_sense], dtype=np.uint8)
    x = np.zeros(max(n, 1))
    ds = np.zeros(max(n, 1))
    r = OrResult()
    lib().or_solve_lp_relaxation(m, n, _i(rp), _i(ci), _d(v), _d(_f64(milp.c)), _d(_f64(milp.l)),
                                 _d(_f64(milp.u)), _d(_f64(milp.b)), _u(is_le), tolerance,
                                 time_limit, int(bool(cupdlpx_termination)), _d(x), _d(ds),
                                 C.byref(r))
    return x[:n], ds[:n], STATUS[r.status], r.total_count, r.as_dict()


def projector_inputs(milp):
    """The projector's scaled data exactly as src/pump.jl:295-303 builds it."""
    n, m = len(milp.c), len(milp.b)
    is_eq = np.array([s == "eq" for s in milp.row_sense], dtype=bool)
    is_int = np.zeros(n, dtype=bool)
    is_int[milp.int_idx] = True
    con_lb = np.where(is_eq, milp.b, -np.inf)
    sc = scale_problem(milp.A, np.zeros(n), milp.l, milp.u, con_lb, milp.b,
                       bound_objective_rescaling=False)
    w = np.ones(n)
    w[milp.int_idx] = sc.D_c[milp.int_idx]
    return sc, is_eq, is_int, w


def project(milp, x_tilde, tol=1e-8, primal_weight=1.0, iteration_limit=1_000_000):
    """The reference test helper ``project`` (test/runtests.jl:12-27) on the oracle."""
    sc, is_eq, is_int, w = projector_inputs(milp)
    s = OraclePDFP(sc.A, sc.con_ub, is_eq, is_int, sc.var_lb, sc.var_ub, w)
    s.set_target(np.asarray(x_tilde, dtype=np.float64) / sc.D_c)
    p = default_params(eps_optimal_relative=tol, eps_feasible_relative=tol,
                       iteration_limit=iteration_limit)
    status = s.solve(p, primal_weight)
    return sc.D_c * s.pdhg_x, status, s


class _OracleProjector(OraclePDFP):
    """OraclePDFP speaking the package's ``SolverParameters`` (pump adapter)."""

    def solve(self, params, primal_weight):  # noqa: D401
        if not isinstance(params, OrParams):
            params = default_params(**params.flat())
        return super().solve(params, primal_weight)


class OracleSolvers:
    """The three solver entry points the pump needs, on the CPU oracle.

    Passed as ``feasibility_pump(..., solvers=OracleSolvers())`` by tests, so
    that the pump loop runs against the reference's CPU algorithm."""

    @staticmethod
    def device_name():
        return "CPU"

    @staticmethod
    def solve_lp_relaxation(milp, tolerance, time_limit, cupdlpx_termination):
        x, ds, st, it, _ = solve_lp_relaxation(milp, tolerance, time_limit, cupdlpx_termination)
        return x, ds, st, it

    @staticmethod
    def scale_problem(A, c, var_lb, var_ub, con_lb, con_ub, ruiz_iterations=10,
                      pock_chambolle_alpha=1.0, bound_objective_rescaling=True):
        return scale_problem(A, c, var_lb, var_ub, con_lb, con_ub, ruiz_iterations,
                             pock_chambolle_alpha, bound_objective_rescaling)

    @staticmethod
    def PDFPState(A, b, is_eq, is_int, var_lb, var_ub, w, precision="fp64"):
        return _OracleProjector(A, b, is_eq, is_int, var_lb, var_ub, w)

    class PDFPBatch:
        """Independent oracle projectors behind the batch interface."""

        def __init__(self, problems, precision="fp64"):
            self.members = []
            for pr in problems:
                s = _OracleProjector(*pr[:7])
                if len(pr) > 7 and pr[7] is not None:
                    s.original_primal_residual(1.0 / np.asarray(pr[7]))
                self.members.append(s)
            self.results = [None] * len(self.members)

        def set_x(self, p, x):
            self.members[p].set_x(x)

        def set_target(self, p, xt):
            self.members[p].set_target(xt)

        def warm_start(self, p):
            self.members[p].warm_start()

        def solve(self, params, primal_weights):
            pws = np.broadcast_to(np.asarray(primal_weights, dtype=float), (len(self.members),))
            out = []
            for p, s in enumerate(self.members):
                out.append(s.solve(params[p], float(pws[p])))
                self.results[p] = dict(s.last)
            return out

        def solve_any(self, params, primal_weights, resume=None):
            # the oracle's members are solved one after the other, each to the end:
            # every member stops in the call, so none is ever left to resume
            if resume is not None and any(resume):
                raise ValueError("no oracle member is left running between calls")
            return self.solve(params, primal_weights)

        def get(self, p, which):
            return self.members[p].get(which)
