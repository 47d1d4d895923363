"""Guarded two-phase CPR rounding (CPU), FP 2.0's constraint-propagation rounding.

Host-side mirror of src/rounding.jl:1-256.  The pump keeps rounding on the CPU;
the propagation and the fixing phases run natively in libpdfp_b200.so
(pdfp_rounder_*, rounding.cpp: the reference's tolerances, queue and row classes,
its arithmetic in its order), while this module keeps the parts that involve the
caller's random stream and clock: the fractionality ranking with its random swaps
(stable sort, ties-to-even rounding) and the online batch policy.  Random choices
use the ``numpy.random.Generator`` handed in by the caller, not Julia's
MersenneTwister, so trajectories that reach the random swaps (iteration >=
swap_iteration), flips or perturbations differ from the reference's stream.
"""
from __future__ import annotations

import ctypes as C
import math
import time

import numpy as np
import scipy.sparse as sp

from . import _lib as L


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

    def _native(self) -> C.c_void_p:
        """The library's model part of the propagation (built on first use)."""
        if self.data is None:
            milp = self.milp
            A = sp.csr_matrix(milp.A, dtype=np.float64)
            A.sum_duplicates()
            A.sort_indices()
            csr, keep = L.make_csr(A)
            h = C.c_void_p()
            is_le = np.ascontiguousarray([s == "le" for s in milp.row_sense], dtype=np.uint8)
            is_int = np.zeros(len(milp.c), dtype=np.uint8)
            is_int[milp.int_idx] = 1
            b, lo, hi = L.f64(milp.b), L.f64(milp.l), L.f64(milp.u)
            L.check(L.lib().pdfp_rounder_create(C.byref(csr), L.dptr(b), L.uptr(is_le), L.dptr(lo),
                                                L.dptr(hi), L.uptr(is_int), C.byref(h)))
            self.data = h
            self._int_arr = np.ascontiguousarray(self._int_idx, dtype=np.int32)
        return self.data

    def __del__(self):
        try:
            if self.data is not None and self.data.value:
                L.lib().pdfp_rounder_destroy(self.data)
                self.data = None
        except Exception:  # noqa: BLE001 (interpreter shutdown)
            pass

    def _round_phases(self, x_star, first, batch_phase: bool, batch, after):
        """One native rounding call (pdfp_rounder_round): (xt, status); status 2: the
        batch phase left the domains infeasible (xt incomplete), 1: the final
        domains are infeasible, 0: not found infeasible."""
        h = self._native()
        xs = L.f64(x_star)
        xt = np.empty(len(xs))
        arr = [np.ascontiguousarray(v, dtype=np.int32) for v in (first, batch, after)]
        direction = None
        if self.direction is not None:
            direction = np.ascontiguousarray(self.direction, dtype=np.uint8)
        inf = C.c_int32()
        L.check(L.lib().pdfp_rounder_round(
            h, L.dptr(xs), L.iptr(arr[0]), len(arr[0]), 1 if batch_phase else 0, L.iptr(arr[1]),
            len(arr[1]), L.iptr(arr[2]), len(arr[2]), L.iptr(self._int_arr), len(self._int_arr),
            None if direction is None else L.uptr(direction), min(self.max_pops, 2**63 - 1),
            L.dptr(xt), C.byref(inf)))
        return xt, int(inf.value)

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



def round_sequential(r: Rounder, x_star, rng, iteration: int) -> np.ndarray:
    """FP 2.0's CPR of ``x_star`` (src/rounding.jl:191-197)."""
    xs = [float(v) for v in x_star]
    ranked = r._ranking(xs, rng, iteration)
    xt, _ = r._round_phases(x_star, ranked, False, [], [])
    return xt


def round_guarded(r: Rounder, x_star, rng, iteration: int) -> np.ndarray:
    """Guarded two-phase CPR (src/rounding.jl:205-256)."""
    r.n_calls += 1
    P = r.policy
    t0 = time.perf_counter_ns() if P is not None else 0
    if P is not None and not P.wants_batch():
        xt = round_sequential(r, x_star, rng, iteration)
        P.observe_skip((time.perf_counter_ns() - t0) / 1e9)
        return xt
    xs = [float(v) for v in x_star]
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

    xt, status = r._round_phases(x_star, before, True, batch, after)
    if status == 2:  # the guard: discard the batch
        r.n_fallbacks += 1
        wasted = 0.0 if P is None else (time.perf_counter_ns() - t0) / 1e9
        out = round_sequential(r, x_star, rng, iteration)
        if P is not None:
            P.observe_batch(True, (time.perf_counter_ns() - t0) / 1e9, wasted)
        return out
    r.n_batched += 1
    if P is not None:
        P.observe_batch(False, (time.perf_counter_ns() - t0) / 1e9, 0.0)
    return xt
