"""The library's native rounder (pdfp_rounder_*, rounding.cpp) against the
pure-Python restatement of src/propagation.jl and src/rounding.jl kept in
oracle/rounding_ref.py: every rounding call must give the same point and the same
infeasibility status, bit for bit.

Cases: the reference's example models (golden fixtures) and synthetic models with
equality, cardinality, knapsack and general rows, general-integer and continuous
columns and infinite bounds; random fractional and integral points; the three call
shapes the pump makes (sequential, guarded with and without the regrouping), with
and without violation-guided directions, and with small propagation budgets.  No
GPU is needed.
"""
import numpy as np
import pytest
import scipy.sparse as sp

from conftest import EXAMPLES, load_example
from oracle import rounding_ref as R
from pdfp_b200 import synthetic
from pdfp_b200.milp import MILP
from pdfp_b200.rounding import Rounder


def _mixed_model(seed):
    """Rows of every class: cardinality (all-one binaries), knapsack (positive
    binaries, <=), general rows over integers in [-3, 5], continuous columns, a few
    infinite bounds, equality rows."""
    rng = np.random.default_rng(seed)
    n_bin, n_int, n_cont = 30, 15, 10
    n = n_bin + n_int + n_cont
    rows, vals, b, sense = [], [], [], []
    for i in range(12):  # cardinality
        cols = rng.choice(n_bin, size=rng.integers(2, 8), replace=False)
        rows.append(cols)
        vals.append(np.ones(len(cols)))
        b.append(float(rng.integers(1, 3)))
        sense.append("eq" if i % 4 == 0 else "le")
    for _ in range(10):  # knapsack
        cols = rng.choice(n_bin, size=rng.integers(3, 10), replace=False)
        rows.append(cols)
        v = rng.integers(1, 20, size=len(cols)).astype(float)
        vals.append(v)
        b.append(float(np.floor(v.sum() / 2)))
        sense.append("le")
    for i in range(15):  # general
        cols = rng.choice(n, size=rng.integers(2, 9), replace=False)
        rows.append(cols)
        vals.append(np.round(rng.normal(size=len(cols)) * 3, 2))
        b.append(float(np.round(rng.normal() * 4, 1)))
        sense.append("eq" if i % 5 == 0 else "le")
    r = np.concatenate([np.full(len(c), i) for i, c in enumerate(rows)])
    c = np.concatenate(rows)
    A = sp.csr_matrix((np.concatenate(vals), (r, c)), shape=(len(rows), n))
    A.sum_duplicates()
    l = np.zeros(n)
    u = np.ones(n)
    l[n_bin:n_bin + n_int] = -3
    u[n_bin:n_bin + n_int] = 5
    l[n_bin + n_int:] = -10.0
    u[n_bin + n_int:] = 10.0
    l[-1], u[-2] = -np.inf, np.inf
    int_idx = np.arange(n_bin + n_int)
    return MILP(rng.normal(size=n), 0.0, A, np.array(b), sense, l, u, int_idx, name=f"mixed{seed}")


def _models():
    out = [load_example(name) for name in EXAMPLES]
    out += [synthetic.covering_p0201_like(3), synthetic.markshare_like(2)]
    out += [_mixed_model(s) for s in (1, 2, 3)]
    return out


def _points(milp, rng):
    n = len(milp.c)
    lo = np.where(np.isfinite(milp.l), milp.l, -5.0)
    hi = np.where(np.isfinite(milp.u), milp.u, 5.0)
    x1 = lo + rng.random(n) * (hi - lo)
    x2 = x1.copy()
    I = milp.int_idx
    k = len(I) // 2
    x2[I[:k]] = np.round(x2[I[:k]])  # half the integers already integral
    x3 = np.round(x1)                 # everything integral
    x4 = x1.copy()
    x4[I] = np.floor(x4[I]) + 0.5     # exact ties (ties to even)
    return [x1, x2, x3, x4]


def _check(milp, x, first, batch_phase, batch, after, direction, max_pops):
    d = R.PropagationData(milp)
    want_xt, want_st = R.round_phases(d, x, first, batch_phase, batch, after, milp.int_idx.tolist(),
                                      direction, max_pops)
    r = Rounder(milp, policy=None, max_pops=max_pops)
    r.direction = direction
    got_xt, got_st = r._round_phases(x, first, batch_phase, batch, after)
    assert got_st == want_st
    if want_st != 2:
        assert np.array_equal(got_xt, np.array(want_xt))


@pytest.mark.parametrize("k", range(len(_models())))
def test_native_rounder_equals_restatement(k):
    milp = _models()[k]
    rng = np.random.default_rng(100 + k)
    I = milp.int_idx.tolist()
    for x in _points(milp, rng):
        order = list(rng.permutation(I))
        integral = [j for j in order if abs(x[j] - round(x[j])) == 0.0]
        frac = [j for j in order if abs(x[j] - round(x[j])) != 0.0]
        direction = (rng.random(len(milp.c)) < 0.5).tolist()
        for dirn in (None, direction):
            for pops in (2**62, 3):
                _check(milp, x, order, False, [], [], dirn, pops)           # sequential
                _check(milp, x, [], True, integral, frac, dirn, pops)       # guarded
                cut = len(order) // 3                                       # regrouped
                _check(milp, x, [j for j in order[:cut] if j in frac], True,
                       [j for j in order[:cut] if j in integral], order[cut:], dirn, pops)


def test_native_rounder_rejects_bad_input():
    milp = load_example("p0201")
    r = Rounder(milp, policy=None)
    n = len(milp.c)
    with pytest.raises(Exception, match="out of range"):
        r._round_phases(np.zeros(n), [n + 5], False, [], [])
    with pytest.raises(Exception, match="out of range"):
        r._round_phases(np.zeros(n), [], True, [-1], [])
