"""Pure-Python restatement of the pump's CPR rounding (src/propagation.jl:1-276,
src/rounding.jl:117-256).

TEST INFRASTRUCTURE ONLY: the checker of the library's native rounder
(pdfp_rounder_*, rounding.cpp); tests/ and the CPU-baseline legs of bench.py may
use it, the product package never does.  Plain Python lists and the reference's
arithmetic in the reference's order: same tolerances, wake-up cap, FIFO queue and
row classes.  ``round_phases`` takes the same arguments as pdfp_rounder_round.
"""
from __future__ import annotations

import math
from collections import deque

import numpy as np

BOUND_TOLERANCE = 1e-6          # src/propagation.jl:7
INFEASIBILITY_TOLERANCE = 1e-6  # :8
MAX_TIGHTENINGS = 10            # :9
DOMAIN_INFINITY = 1e12          # :10

ROW_GENERAL = 0      # :14
ROW_CARDINALITY = 1  # :15
ROW_KNAPSACK = 2     # :16


class PropagationData:
    """Everything about the propagation that depends on the model only (src/propagation.jl:19-84)."""

    def __init__(self, milp):
        n, m = len(milp.c), len(milp.b)
        A = milp.A.tocsc()
        A.sort_indices()
        self.col_rows = [A.indices[A.indptr[j]:A.indptr[j + 1]].tolist() for j in range(n)]
        self.col_vals = [A.data[A.indptr[j]:A.indptr[j + 1]].tolist() for j in range(n)]
        At = milp.A.tocsr()
        At.sort_indices()
        self.row_cols = [At.indices[At.indptr[i]:At.indptr[i + 1]].tolist() for i in range(m)]
        self.row_vals = [At.data[At.indptr[i]:At.indptr[i + 1]].tolist() for i in range(m)]
        self.b = [float(v) for v in milp.b]
        self.is_le = [s == "le" for s in milp.row_sense]
        ml, mu = milp.l.tolist(), milp.u.tolist()
        self.l = [v if math.isfinite(v) else -DOMAIN_INFINITY for v in ml]
        self.u = [v if math.isfinite(v) else DOMAIN_INFINITY for v in mu]
        is_int = np.zeros(n, dtype=bool)
        is_int[milp.int_idx] = True
        self.is_int = is_int.tolist()
        self.L_min = [0.0] * m
        self.L_max = [0.0] * m
        self.row_kind = [ROW_GENERAL] * m
        self.row_maxcoef = [0.0] * m
        self.row_maxroom = [0.0] * m
        l, u = self.l, self.u
        for i in range(m):
            lmin = 0.0
            lmax = 0.0
            cols, vals = self.row_cols[i], self.row_vals[i]
            for j, a in zip(cols, vals):
                if a > 0:
                    lmin += a * l[j]
                    lmax += a * u[j]
                else:
                    lmin += a * u[j]
                    lmax += a * l[j]
            self.L_min[i] = lmin
            self.L_max[i] = lmax
            all_one = all_pos = all_bin = True
            maxcoef = 0.0
            for j, a in zip(cols, vals):
                if abs(a) > maxcoef:
                    maxcoef = abs(a)
                if a != 1.0:
                    all_one = False
                if not a > 0.0:
                    all_pos = False
                if not (self.is_int[j] and ml[j] == 0.0 and mu[j] == 1.0):
                    all_bin = False
                if not (all_bin and (all_one or all_pos)):
                    break
            self.row_maxcoef[i] = maxcoef
            if all_bin and all_one:
                self.row_kind[i] = ROW_CARDINALITY
            elif all_bin and all_pos and self.is_le[i]:
                self.row_kind[i] = ROW_KNAPSACK
            room = 0.0
            for j, a in zip(cols, vals):
                width = mu[j] - ml[j]
                r = abs(a) * width if math.isfinite(width) else math.inf
                if r > room:
                    room = r
            self.row_maxroom[i] = room


class PropagationState:
    """Domains of one rounding pass and the propagation queue (src/propagation.jl:87-107)."""

    def __init__(self, d: PropagationData, max_pops: int):
        m = len(d.b)
        n = len(d.l)
        self.data = d
        self.l = list(d.l)
        self.u = list(d.u)
        self.L_min = list(d.L_min)
        self.L_max = list(d.L_max)
        self.in_queue = [False] * m
        self.queue: deque = deque()
        self.tighten_lo = [0] * n
        self.tighten_hi = [0] * n
        self.row_maxroom = list(d.row_maxroom)
        self.max_pops = max_pops
        self.infeasible = False


def _enqueue(s: PropagationState, i: int) -> None:
    if not s.in_queue[i]:
        s.queue.append(i)
        s.in_queue[i] = True


def _tighten_upper(s: PropagationState, j: int, new_u: float) -> bool:
    """src/propagation.jl:117-136"""
    u_old = s.u[j]
    if not new_u < u_old - BOUND_TOLERANCE:
        return False
    nu = float(math.floor(new_u + BOUND_TOLERANCE)) if s.data.is_int[j] else new_u
    if nu < s.l[j] - BOUND_TOLERANCE:
        nu = s.l[j]
    nu = max(nu, s.l[j])
    if nu >= u_old - BOUND_TOLERANCE:
        return False
    s.u[j] = nu
    s.tighten_hi[j] += 1
    wake = s.tighten_hi[j] <= MAX_TIGHTENINGS or abs(nu - s.l[j]) < BOUND_TOLERANCE
    du = nu - u_old
    for i, a in zip(s.data.col_rows[j], s.data.col_vals[j]):
        if a > 0:
            s.L_max[i] += a * du
        else:
            s.L_min[i] += a * du
        if wake:
            _enqueue(s, i)
    return True


def _tighten_lower(s: PropagationState, j: int, new_l: float) -> bool:
    """src/propagation.jl:138-156"""
    l_old = s.l[j]
    if not new_l > l_old + BOUND_TOLERANCE:
        return False
    nl = float(math.ceil(new_l - BOUND_TOLERANCE)) if s.data.is_int[j] else new_l
    if nl > s.u[j] + BOUND_TOLERANCE:
        nl = s.u[j]
    nl = min(nl, s.u[j])
    if nl <= l_old + BOUND_TOLERANCE:
        return False
    s.l[j] = nl
    s.tighten_lo[j] += 1
    wake = s.tighten_lo[j] <= MAX_TIGHTENINGS or abs(s.u[j] - nl) < BOUND_TOLERANCE
    dl = nl - l_old
    for i, a in zip(s.data.col_rows[j], s.data.col_vals[j]):
        if a > 0:
            s.L_min[i] += a * dl
        else:
            s.L_max[i] += a * dl
        if wake:
            _enqueue(s, i)
    return True


def _propagate_cardinality_row(s: PropagationState, i: int) -> None:
    """src/propagation.jl:160-177"""
    d = s.data
    is_eq = not d.is_le[i]
    b = d.b[i]
    slack_up = b - s.L_min[i]
    slack_dn = s.L_max[i] - b
    if slack_up < -INFEASIBILITY_TOLERANCE or (is_eq and slack_dn < -INFEASIBILITY_TOLERANCE):
        s.infeasible = True
        return
    up = slack_up < 1.0 - BOUND_TOLERANCE
    dn = is_eq and slack_dn < 1.0 - BOUND_TOLERANCE
    if not (up or dn):
        return
    for j in d.row_cols[i]:
        if up:
            _tighten_upper(s, j, s.l[j] + slack_up)
        if dn:
            _tighten_lower(s, j, s.u[j] - slack_dn)


def _propagate_knapsack_row(s: PropagationState, i: int) -> None:
    """src/propagation.jl:180-192"""
    d = s.data
    slack_up = d.b[i] - s.L_min[i]
    if slack_up < -INFEASIBILITY_TOLERANCE:
        s.infeasible = True
        return
    if d.row_maxcoef[i] <= slack_up + BOUND_TOLERANCE:
        return
    for j, a in zip(d.row_cols[i], d.row_vals[i]):
        if a > slack_up + BOUND_TOLERANCE:
            _tighten_upper(s, j, s.l[j])


def _propagate_row(s: PropagationState, i: int) -> None:
    """src/propagation.jl:194-232"""
    d = s.data
    kind = d.row_kind[i]
    if kind == ROW_CARDINALITY:
        return _propagate_cardinality_row(s, i)
    if kind == ROW_KNAPSACK:
        return _propagate_knapsack_row(s, i)
    is_le = d.is_le[i]
    b = d.b[i]
    slack_up = b - s.L_min[i]
    slack_dn = s.L_max[i] - b
    if slack_up < -INFEASIBILITY_TOLERANCE or ((not is_le) and slack_dn < -INFEASIBILITY_TOLERANCE):
        s.infeasible = True
        return
    threshold = (slack_up if is_le else min(slack_up, slack_dn)) + BOUND_TOLERANCE
    if s.row_maxroom[i] <= threshold:
        return
    cols, vals = d.row_cols[i], d.row_vals[i]
    max_room = 0.0
    for j, a in zip(cols, vals):
        room = abs(a) * (s.u[j] - s.l[j])
        if room > max_room:
            max_room = room
    s.row_maxroom[i] = max_room
    if is_le and max_room <= slack_up + BOUND_TOLERANCE:
        return
    for j, a in zip(cols, vals):
        if a > 0:
            _tighten_upper(s, j, s.l[j] + slack_up / a)
        else:
            _tighten_lower(s, j, s.u[j] + slack_up / a)
        if not is_le:
            if a > 0:
                _tighten_lower(s, j, s.u[j] - slack_dn / a)
            else:
                _tighten_upper(s, j, s.l[j] - slack_dn / a)


def propagate(s: PropagationState) -> int:
    """Propagate queued rows until the queue is empty or the budget is spent (src/propagation.jl:235-244)."""
    pops = 0
    while s.queue and pops < s.max_pops:
        i = s.queue.popleft()
        s.in_queue[i] = False
        _propagate_row(s, i)
        pops += 1
    return pops


def fix(s: PropagationState, j: int, value: float) -> bool:
    """Fix x_j = value and queue its rows (src/propagation.jl:252-274)."""
    if value < s.l[j] - BOUND_TOLERANCE or value > s.u[j] + BOUND_TOLERANCE:
        s.infeasible = True
        return False
    lo, hi = s.l[j], s.u[j]
    v = hi if value > hi else (lo if value < lo else value)
    l_old, u_old = lo, hi
    if abs(v - l_old) < BOUND_TOLERANCE and abs(v - u_old) < BOUND_TOLERANCE:
        return True
    s.l[j] = v
    s.u[j] = v
    s.tighten_lo[j] += 1
    s.tighten_hi[j] += 1
    dl = v - l_old
    du = v - u_old
    for i, a in zip(s.data.col_rows[j], s.data.col_vals[j]):
        if a > 0:
            s.L_min[i] += a * dl
            s.L_max[i] += a * du
        else:
            s.L_min[i] += a * du
            s.L_max[i] += a * dl
        _enqueue(s, i)
    return True


def is_fixed(s: PropagationState, j: int) -> bool:
    return abs(s.u[j] - s.l[j]) < BOUND_TOLERANCE


# ---- the rounding phases (src/rounding.jl:117-256) --------------------------------

def _round(v: float) -> float:
    """Julia ``round`` on a Float64: nearest, ties to even (Python's round is ties-to-even)."""
    return float(round(v))


def _clamp(x: float, lo: float, hi: float) -> float:
    return hi if x > hi else (lo if x < lo else x)


def _row_violation(d: PropagationData, i: int, activity: float) -> float:
    """src/rounding.jl:117-118"""
    return max(0.0, activity - d.b[i]) if d.is_le[i] else abs(activity - d.b[i])


def _guided_value(d: PropagationData, s: PropagationState, j: int, target: float, activity) -> float:
    """Violation-guided rounding (src/rounding.jl:123-141)."""
    if not s.u[j] - s.l[j] > BOUND_TOLERANCE:
        return target
    lo = float(math.ceil(s.l[j] - BOUND_TOLERANCE))
    hi = float(math.floor(s.u[j] + BOUND_TOLERANCE))
    if not hi > lo:
        return target
    rows, vals = d.col_rows[j], d.col_vals[j]

    def score(v):
        t = 0.0
        for i, a in zip(rows, vals):
            t += _row_violation(d, i, activity[i] + a * v) - _row_violation(d, i, activity[i])
        return t

    score_lo = score(lo)
    score_hi = score(hi)
    if score_lo < score_hi - 1e-12:
        return lo
    if score_hi < score_lo - 1e-12:
        return hi
    return target


def _add_activity(d: PropagationData, activity, j: int, v: float) -> None:
    for i, a in zip(d.col_rows[j], d.col_vals[j]):
        activity[i] += a * v


def _round_sequentially(d, s, xt, idx, x_star, direction, activity) -> None:
    """src/rounding.jl:152-174"""
    for j in idx:
        if is_fixed(s, j):
            xt[j] = s.l[j]
            continue
        target = _round(_clamp(x_star[j], s.l[j], s.u[j]))
        if target < s.l[j] - BOUND_TOLERANCE or target > s.u[j] + BOUND_TOLERANCE:
            other = _round(_clamp(x_star[j] + (1.0 if target < s.l[j] else -1.0), s.l[j], s.u[j]))
            target = _clamp(other, s.l[j], s.u[j])
        if direction is not None and direction[j]:
            target = _guided_value(d, s, j, target, activity)
        fix(s, j, target)
        propagate(s)
        if direction is not None:
            _add_activity(d, activity, j, target)
        xt[j] = target


def round_phases(d: PropagationData, x_star, first, batch_phase: bool, batch, after, int_idx,
                 direction, max_pops: int):
    """One rounding call, as pdfp_rounder_round: returns (xt, status) with status 2
    when the batch phase left the domains infeasible, else 1 / 0 for the final
    domains infeasible / not."""
    s = PropagationState(d, max_pops)
    xs = [float(v) for v in x_star]
    xt = list(xs)
    activity = None if direction is None else [0.0] * len(d.b)
    _round_sequentially(d, s, xt, first, xs, direction, activity)
    if batch_phase:
        for j in batch:
            if is_fixed(s, j):
                xt[j] = s.l[j]
                continue
            target = _round(_clamp(xs[j], s.l[j], s.u[j]))
            fix(s, j, target)
            if direction is not None:
                _add_activity(d, activity, j, target)
            xt[j] = target
        propagate(s)
        if s.infeasible:
            return xt, 2
    _round_sequentially(d, s, xt, after, xs, direction, activity)
    for j in int_idx:
        xt[j] = s.l[j] if is_fixed(s, j) else _round(_clamp(xs[j], s.l[j], s.u[j]))
    return xt, 1 if s.infeasible else 0
