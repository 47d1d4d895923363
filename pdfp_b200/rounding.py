"""Guarded two-phase CPR rounding (CPU), FP 2.0's constraint-propagation rounding.

Host-side restatement of src/rounding.jl:1-256.  The pump keeps rounding on
the CPU; the integer arithmetic (ties-to-even rounding, stable ranking sort,
bound tolerances) follows the reference line for line.  Random choices use the
``numpy.random.Generator`` handed in by the caller, not Julia's MersenneTwister,
so trajectories that reach the random swaps (iteration >= swap_iteration),
flips or perturbations differ from the reference's stream.
"""
from __future__ import annotations

import math
import time

import numpy as np

from .propagation import (BOUND_TOLERANCE, PropagationData, PropagationState, fix,
                          is_fixed, propagate)


def _round(v: float) -> float:
    """Julia ``round`` on a Float64: nearest, ties to even (Python's round is ties-to-even)."""
    return float(round(v))


def _clamp(x: float, lo: float, hi: float) -> float:
    return hi if x > hi else (lo if x < lo else x)


class BatchPolicy:
    """Online rule deciding per call whether to try the batch (src/rounding.jl:22-63)."""

    def __init__(self, xi: float = 0.3, nu: float = 0.9, reprobe: int = 20):
        self.xi = xi
        self.nu = nu
        self.reprobe = reprobe
        self.n_failed = 0.0
        self.n_held = 0.0
        self.s = math.nan
        self.h = math.nan
        self.w = math.nan
        self.skipped = 0

    def _ema(self, old: float, x: float) -> float:
        return x if math.isnan(old) else (1.0 - self.xi) * old + self.xi * x

    def wants_batch(self) -> bool:
        if self.skipped >= self.reprobe:
            return True
        if math.isnan(self.s) or self.n_failed == 0.0:
            return True
        h = 0.0 if math.isnan(self.h) else self.h
        p = self.n_failed / (self.n_failed + self.n_held)
        return p * (self.w + self.s) + (1.0 - p) * h < self.s

    def observe_batch(self, failed: bool, cost: float, wasted: float) -> None:
        self.n_failed *= self.nu
        self.n_held *= self.nu
        self.skipped = 0
        if failed:
            self.n_failed += 1.0
            self.w = self._ema(self.w, wasted)
            self.s = self._ema(self.s, max(cost - wasted, 0.0))
        else:
            self.n_held += 1.0
            self.h = self._ema(self.h, cost)

    def observe_skip(self, cost: float) -> None:
        self.s = self._ema(self.s, cost)
        self.skipped += 1


class Rounder:
    """Rounding state persisting across the calls of one pump run (src/rounding.jl:78-98)."""

    def __init__(self, milp, schedule: str = "all", max_pops: int = 2**62,
                 swap_iteration: int = 10, policy: BatchPolicy | None = "default"):
        self.milp = milp
        self.data = None
        self.schedule = schedule
        self.direction = None  # list[bool] over columns, or None
        self.max_pops = max_pops
        self.swap_iteration = swap_iteration
        self.policy = BatchPolicy() if policy == "default" else policy
        self.n_calls = 0
        self.n_batched = 0
        self.n_fallbacks = 0
        n = len(milp.c)
        self._is_binary = [False] * n
        for j in milp.int_idx.tolist():
            self._is_binary[j] = milp.l[j] == 0.0 and milp.u[j] == 1.0
        self._int_idx = milp.int_idx.tolist()

    def _new_state(self) -> PropagationState:
        if self.data is None:
            self.data = PropagationData(self.milp)
        return PropagationState(self.data, self.max_pops)

    def _ranking(self, x_star, rng, iteration: int) -> list:
        """Ascending fractionality, binaries first; random swaps from ``swap_iteration`` on
        (src/rounding.jl:105-115)."""
        keys = [abs(x_star[j] - _round(x_star[j])) - (10.0 if self._is_binary[j] else 0.0)
                for j in self._int_idx]
        order = sorted(range(len(keys)), key=keys.__getitem__)  # stable, like sortperm
        ranked = [self._int_idx[k] for k in order]
        if iteration >= self.swap_iteration and len(ranked) >= 10:
            L = len(ranked)
            for _ in range(max(1, L // 10)):
                a = int(rng.integers(0, L))
                b = int(rng.integers(0, L))
                ranked[a], ranked[b] = ranked[b], ranked[a]
        return ranked

    def _activity(self):
        return None if self.direction is None else [0.0] * len(self.milp.b)


def _row_violation(d: PropagationData, i: int, activity: float) -> float:
    """src/rounding.jl:117-118"""
    return max(0.0, activity - d.b[i]) if d.is_le[i] else abs(activity - d.b[i])


def _guided_value(r: Rounder, s: PropagationState, j: int, target: float, activity) -> float:
    """Violation-guided rounding (src/rounding.jl:123-141)."""
    if not s.u[j] - s.l[j] > BOUND_TOLERANCE:
        return target
    lo = float(math.ceil(s.l[j] - BOUND_TOLERANCE))
    hi = float(math.floor(s.u[j] + BOUND_TOLERANCE))
    if not hi > lo:
        return target
    d = r.data
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


def _add_activity(r: Rounder, activity, j: int, v: float) -> None:
    for i, a in zip(r.data.col_rows[j], r.data.col_vals[j]):
        activity[i] += a * v


def _round_sequentially(r: Rounder, s: PropagationState, xt, idx, x_star, activity) -> None:
    """src/rounding.jl:152-174"""
    for j in idx:
        if is_fixed(s, j):
            xt[j] = s.l[j]
            continue
        target = _round(_clamp(x_star[j], s.l[j], s.u[j]))
        if target < s.l[j] - BOUND_TOLERANCE or target > s.u[j] + BOUND_TOLERANCE:
            other = _round(_clamp(x_star[j] + (1.0 if target < s.l[j] else -1.0), s.l[j], s.u[j]))
            target = _clamp(other, s.l[j], s.u[j])
        if activity is not None and r.direction[j]:
            target = _guided_value(r, s, j, target, activity)
        fix(s, j, target)
        propagate(s)
        if activity is not None:
            _add_activity(r, activity, j, target)
        xt[j] = target


def _read_integers(r: Rounder, s: PropagationState, xt, x_star):
    for j in r._int_idx:
        xt[j] = s.l[j] if is_fixed(s, j) else _round(_clamp(x_star[j], s.l[j], s.u[j]))
    return xt


def round_sequential(r: Rounder, x_star, rng, iteration: int) -> np.ndarray:
    """FP 2.0's CPR of ``x_star`` (src/rounding.jl:191-197)."""
    s = r._new_state()
    xs = [float(v) for v in x_star]
    xt = list(xs)
    ranked = r._ranking(xs, rng, iteration)
    _round_sequentially(r, s, xt, ranked, xs, r._activity())
    return np.array(_read_integers(r, s, xt, xs))


def round_guarded(r: Rounder, x_star, rng, iteration: int) -> np.ndarray:
    """Guarded two-phase CPR (src/rounding.jl:205-256)."""
    r.n_calls += 1
    P = r.policy
    t0 = time.perf_counter_ns() if P is not None else 0
    if P is not None and not P.wants_batch():
        xt = round_sequential(r, x_star, rng, iteration)
        P.observe_skip((time.perf_counter_ns() - t0) / 1e9)
        return xt
    s = r._new_state()
    xs = [float(v) for v in x_star]
    xt = list(xs)
    activity = r._activity()
    ranked = r._ranking(xs, rng, iteration)

    def integral(j):
        return abs(xs[j] - _round(xs[j])) == 0.0

    if r.schedule == "regroup":
        last = 0
        for k in range(len(ranked), 0, -1):
            if integral(ranked[k - 1]):
                last = k
                break
        before = [ranked[k] for k in range(last) if not integral(ranked[k])]
        batch = [ranked[k] for k in range(last) if integral(ranked[k])]
        after = ranked[last:]
    else:
        before = []
        batch = [j for j in ranked if integral(j)]
        after = [j for j in ranked if not integral(j)]

    _round_sequentially(r, s, xt, before, xs, activity)
    for j in batch:
        if is_fixed(s, j):
            xt[j] = s.l[j]
            continue
        target = _round(_clamp(xs[j], s.l[j], s.u[j]))
        fix(s, j, target)
        if activity is not None:
            _add_activity(r, activity, j, target)
        xt[j] = target
    propagate(s)

    if s.infeasible:  # the guard: discard the batch
        r.n_fallbacks += 1
        wasted = 0.0 if P is None else (time.perf_counter_ns() - t0) / 1e9
        out = round_sequential(r, x_star, rng, iteration)
        if P is not None:
            P.observe_batch(True, (time.perf_counter_ns() - t0) / 1e9, wasted)
        return out
    r.n_batched += 1
    _round_sequentially(r, s, xt, after, xs, activity)
    _read_integers(r, s, xt, xs)
    if P is not None:
        P.observe_batch(False, (time.perf_counter_ns() - t0) / 1e9, 0.0)
    return np.array(xt)
