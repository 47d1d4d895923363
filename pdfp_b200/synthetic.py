"""Seeded synthetic models with the shapes of the benchmark configurations.

The reference is measured on MIPLIB instances that are not available here;
these generators stand in for them with the shapes, sizes and value
distributions the benchmark configurations specify.  Every generator is
deterministic in its seed (numpy PCG64).

* ``covering_p0201_like``  -- 133 x 201, 1923 nonzeros, binaries (config 0)
* ``general_integer``       -- 20k x 50k, Poisson(25) rows (config 1)
* ``zipf_lp``               -- 1M x 2M, 20M nonzeros, Zipf(1.5) rows (config 2)
* ``covering_packing_batch``-- 64 uneven covering/packing models (config 3)
* ``markshare_like``        -- 6 x (50 + 6), equality knapsacks (config 4)
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp

from .milp import MILP


def _rng(seed: int) -> np.random.Generator:
    return np.random.Generator(np.random.PCG64(seed))


def _covering_pattern(rng, m: int, n: int, nnz: int):
    """Distinct random positions, every row and every column holding at least one."""
    pos = set()
    for i in range(m):
        pos.add((i, int(rng.integers(0, n))))
    for j in range(n):
        pos.add((int(rng.integers(0, m)), j))
    while len(pos) < nnz:
        pos.add((int(rng.integers(0, m)), int(rng.integers(0, n))))
    rows = np.array([p[0] for p in pos], dtype=np.int64)
    cols = np.array([p[1] for p in pos], dtype=np.int64)
    order = np.lexsort((cols, rows))
    return rows[order], cols[order]


def covering_p0201_like(seed: int = 1, m: int = 133, n: int = 201, nnz: int = 1923) -> MILP:
    """Pure-binary covering model: rows -A x <= -b, A in {1..5}, b_i = 1 + floor(0.3 rowsum_i),
    so x = 1 is feasible; c in {1..100}; bounds [0, 1]."""
    rng = _rng(seed)
    rows, cols = _covering_pattern(rng, m, n, nnz)
    vals = rng.integers(1, 6, size=len(rows)).astype(np.float64)
    A = sp.csr_matrix((vals, (rows, cols)), shape=(m, n))
    rowsum = np.asarray(A.sum(axis=1)).ravel()
    b = 1.0 + np.floor(0.3 * rowsum)
    c = rng.integers(1, 101, size=n).astype(np.float64)
    return MILP(c, 0.0, -A, -b, ["le"] * m, np.zeros(n), np.ones(n), np.arange(n),
                name=f"covering_{m}x{n}_s{seed}")


def _csr_from_keys(key: np.ndarray, vals: np.ndarray, m: int, n: int) -> sp.csr_matrix:
    """CSR matrix from sorted unique row-major keys (row * n + col): no COO round trip."""
    rows = key // n
    indptr = np.zeros(m + 1, dtype=np.int64)
    np.cumsum(np.bincount(rows, minlength=m), out=indptr[1:])
    A = sp.csr_matrix((vals, (key - rows * n).astype(np.int32), indptr), shape=(m, n))
    A.has_sorted_indices = True
    A.has_canonical_format = True
    return A


def _sorted_unique(key: np.ndarray) -> np.ndarray:
    """Sorted distinct values (sort + adjacent difference; faster than np.unique here)."""
    key = np.sort(key)
    if len(key) == 0:
        return key
    keep = np.empty(len(key), dtype=bool)
    keep[0] = True
    np.not_equal(key[1:], key[:-1], out=keep[1:])
    return key[keep]


def _rows_with_lengths(rng, lengths: np.ndarray, n: int, band: int = 0):
    """Row index / distinct column index arrays for the given row lengths.  band > 0 draws
    row i's columns within +-band of its diagonal position i * n / m (wrapping)."""
    m = len(lengths)
    total = int(lengths.sum())
    rows = np.repeat(np.arange(m, dtype=np.int64), lengths)

    def draw(r):
        if band <= 0:
            return rng.integers(0, n, size=len(r), dtype=np.int64)
        return (r * n // m + rng.integers(-band, band + 1, size=len(r), dtype=np.int64)) % n

    cols = draw(rows)
    # make columns distinct within each row: sort, drop repeats, top up with fresh draws
    key = rows * n + cols
    key = _sorted_unique(key)
    missing = total - len(key)
    while missing > 0:
        extra_rows = rng.integers(0, m, size=missing, dtype=np.int64)
        key = _sorted_unique(np.concatenate([key, extra_rows * n + draw(extra_rows)]))
        missing = total - len(key)
    return key // n, key % n


def general_integer(seed: int = 1, m: int = 20000, n: int = 50000, m_eq: int = 5000,
                    mean_row: float = 25.0):
    """General-integer model: m rows (m - m_eq <=, m_eq =), n columns (90% integer in [0, 10],
    10% continuous in [0, 100]); Poisson(25) row lengths (zero redrawn); N(0, 1) coefficients
    rounded to 2 decimals (zero redrawn); b from an integer point x0 (b = A x0 on = rows,
    A x0 + U[0, 5] on <= rows); c ~ U[-1, 1].  Returns (milp, x0, target), target =
    clamp(x0 + U{-1, 0, 1}) on the integer columns."""
    rng = _rng(seed)
    lengths = rng.poisson(mean_row, size=m)
    while np.any(lengths == 0):
        z = lengths == 0
        lengths[z] = rng.poisson(mean_row, size=int(z.sum()))
    lengths = np.minimum(lengths, n)
    rows, cols = _rows_with_lengths(rng, lengths, n)
    vals = np.round(rng.normal(0.0, 1.0, size=len(rows)), 2)
    while np.any(vals == 0.0):
        z = vals == 0.0
        vals[z] = np.round(rng.normal(0.0, 1.0, size=int(z.sum())), 2)
    A = _csr_from_keys(rows * n + cols, vals, m, n)
    n_int = int(round(0.9 * n))
    perm = rng.permutation(n)
    int_idx = np.sort(perm[:n_int])
    is_int = np.zeros(n, dtype=bool)
    is_int[int_idx] = True
    l = np.zeros(n)
    u = np.where(is_int, 10.0, 100.0)
    x0 = np.where(is_int, rng.integers(0, 11, size=n), rng.integers(0, 101, size=n)).astype(np.float64)
    Ax0 = A @ x0
    sense = ["le"] * (m - m_eq) + ["eq"] * m_eq
    b = Ax0.copy()
    b[: m - m_eq] += rng.uniform(0.0, 5.0, size=m - m_eq)
    c = rng.uniform(-1.0, 1.0, size=n)
    milp = MILP(c, 0.0, A, b, sense, l, u, int_idx, name=f"general_{m}x{n}_s{seed}")
    target = x0.copy()
    step = rng.integers(-1, 2, size=n).astype(np.float64)
    target[is_int] = np.clip(x0[is_int] + step[is_int], l[is_int], u[is_int])
    return milp, x0, target


def zipf_lengths(rng, m: int, nnz: int, a: float = 1.5, cap: int = 10000) -> np.ndarray:
    """Zipf(a) row lengths capped at `cap`, rescaled to sum to exactly `nnz` (each >= 1)."""
    L = np.minimum(rng.zipf(a, size=m), cap).astype(np.float64)
    L = np.maximum(1, np.floor(L * (nnz / L.sum()))).astype(np.int64)
    L = np.minimum(L, cap)
    diff = nnz - int(L.sum())
    while diff != 0:
        if diff > 0:
            idx = rng.integers(0, m, size=diff)
            np.add.at(L, idx, 1)
            L = np.minimum(L, cap)
        else:
            cand = np.nonzero(L > 1)[0]
            idx = rng.choice(cand, size=min(-diff, len(cand)), replace=False)
            L[idx] -= 1
        diff = nnz - int(L.sum())
    return L


def zipf_lp(seed: int = 1, m: int = 1_000_000, n: int = 2_000_000, nnz: int = 20_000_000,
            band: int = 0):
    """LP relaxation for the bandwidth stress: n columns (first half binary, second half
    continuous in [0, 1]), Zipf(1.5) row lengths capped at 10,000 and rescaled to exactly `nnz`
    nonzeros, U[-1, 1] values, <= rows with b = A x_f + U[0, 1] for a random point x_f.
    band > 0: a variant with locality -- each row's columns within +-band of its diagonal
    position (band is raised to the longest row so that every row fits).
    Returns (milp, x_f)."""
    rng = _rng(seed)
    lengths = zipf_lengths(rng, m, nnz)
    lengths = np.minimum(lengths, n)
    if band > 0:
        band = min(max(band, int(lengths.max())), n // 2)
    rows, cols = _rows_with_lengths(rng, lengths, n, band)
    vals = rng.uniform(-1.0, 1.0, size=len(rows))
    A = _csr_from_keys(rows * n + cols, vals, m, n)
    n_bin = n // 2
    xf = np.concatenate([rng.integers(0, 2, size=n_bin).astype(np.float64),
                         rng.uniform(0.0, 1.0, size=n - n_bin)])
    b = A @ xf + rng.uniform(0.0, 1.0, size=m)
    c = np.zeros(n)
    milp = MILP(c, 0.0, A, b, ["le"] * m, np.zeros(n), np.ones(n), np.arange(n_bin),
                name=f"zipf_{m}x{n}_s{seed}")
    return milp, xf


def covering_packing_batch(seed: int = 1, k: int = 64, n_min: int = 1000, n_max: int = 200000,
                           row_min: int = 10, row_max: int = 40):
    """k binary models, n log-uniform in [n_min, n_max], m = 0.6 n, 10-40 nonzeros per row,
    coefficients in {1..5}; the first half covering (-A x <= -(1 + floor(0.3 rowsum))), the
    second half packing (A x <= floor(0.5 rowsum))."""
    rng = _rng(seed)
    out = []
    for p in range(k):
        n = int(np.exp(rng.uniform(np.log(n_min), np.log(n_max))))
        m = max(1, int(0.6 * n))
        lengths = rng.integers(row_min, row_max + 1, size=m)
        lengths = np.minimum(lengths, n)
        rows, cols = _rows_with_lengths(rng, lengths, n)
        vals = rng.integers(1, 6, size=len(rows)).astype(np.float64)
        A = _csr_from_keys(rows * n + cols, vals, m, n)
        rowsum = np.asarray(A.sum(axis=1)).ravel()
        if p < k // 2:
            milp = MILP(rng.integers(1, 101, size=n).astype(np.float64), 0.0, -A,
                        -(1.0 + np.floor(0.3 * rowsum)), ["le"] * m, np.zeros(n), np.ones(n),
                        np.arange(n), name=f"cover_{p}")
        else:
            milp = MILP(-rng.integers(1, 101, size=n).astype(np.float64), 0.0, A,
                        np.floor(0.5 * rowsum), ["le"] * m, np.zeros(n), np.ones(n),
                        np.arange(n), name=f"pack_{p}")
        out.append(milp)
    return out


def markshare_like(seed: int = 1, rows: int = 6, binaries: int = 50) -> MILP:
    """Equality knapsacks: sum_j a_ij x_j + s_i = floor(rowsum_i / 2), a in {0..99},
    x binary, slacks s_i in [0, 1000]; objective sum of slacks."""
    rng = _rng(seed)
    a = rng.integers(0, 100, size=(rows, binaries)).astype(np.float64)
    b = np.floor(a.sum(axis=1) / 2.0)
    A = sp.hstack([sp.csr_matrix(a), sp.eye(rows)]).tocsr()
    n = binaries + rows
    c = np.concatenate([np.zeros(binaries), np.ones(rows)])
    u = np.concatenate([np.ones(binaries), np.full(rows, 1000.0)])
    return MILP(c, 0.0, A, b, ["eq"] * rows, np.zeros(n), u, np.arange(binaries),
                name=f"markshare_{rows}x{binaries}_s{seed}")
