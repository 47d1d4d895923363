"""The pump's column scaling on the device (pdfp_set_col_scale and the *_unscaled calls).

The pump feeds the projector x ./ D_c and x_tilde ./ D_c and reads back
D_c .* s.pdhg_x (src/pump.jl:305-306, 331, 338).  With the column scale held by
the handle, the division and the product run on the device; both are single
correctly rounded FP64 operations, so every result must equal the host
arithmetic bit for bit: the same iterate after the same solve, in both
precisions, for single handles and batch members.  Also checked: the argument
errors (no scale set, a scale entry that is not positive and finite, a NaN in the
target -- which must leave the handle's state untouched) and the page-locked
host arrays.
"""
import numpy as np
import pytest

from pdfp_b200 import gpu
from pdfp_b200 import synthetic
from pdfp_b200.params import SolverParameters

pytestmark = pytest.mark.gpu


def _problem(oracle, seed=3):
    milp = synthetic.covering_p0201_like(seed)
    sc, is_eq, is_int, w = oracle.projector_inputs(milp)
    rng = np.random.default_rng(seed)
    n = len(milp.c)
    xt = np.where(is_int, np.round(rng.random(n)), rng.random(n) * 3.0 - 1.0)
    x0 = np.clip(rng.normal(size=n), milp.l, milp.u)
    return milp, sc, is_eq, is_int, w, xt, x0


def _state(sc, is_eq, is_int, w, precision):
    return gpu.PDFPState(sc.A, sc.con_ub, is_eq, is_int, sc.var_lb, sc.var_ub, w, precision=precision)


PARAMS = SolverParameters(eps_optimal_relative=1e-5, eps_feasible_relative=1e-6,
                          iteration_limit=3000)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_unscaled_calls_equal_host_scaling(oracle, precision):
    milp, sc, is_eq, is_int, w, xt, x0 = _problem(oracle)
    host = _state(sc, is_eq, is_int, w, precision)
    dev = _state(sc, is_eq, is_int, w, precision)
    dev.set_col_scale(sc.D_c)
    host.set_x(x0 / sc.D_c)
    dev.set_x_unscaled(x0)
    assert np.array_equal(host.get("current_x"), dev.get("current_x"))
    host.set_target(xt / sc.D_c)
    dev.set_target_unscaled(xt)
    for name in ("current_x", "pdhg_x", "reflected_x"):
        assert np.array_equal(host.get(name), dev.get(name)), name
    r1 = host.solve(PARAMS, 1.0)
    r2 = dev.solve(PARAMS, 1.0)
    assert r1 == r2 and host.total_count == dev.total_count
    x_host = sc.D_c * host.pdhg_x
    x_dev = dev.get_unscaled("pdhg_x")
    assert np.array_equal(x_host, x_dev)
    assert np.array_equal(sc.D_c * host.get("current_x"), dev.get_unscaled("current_x"))
    # a second target through the same handles (warm start from the first)
    xt2 = xt.copy()
    xt2[np.flatnonzero(is_int)[:5]] = 1.0 - xt2[np.flatnonzero(is_int)[:5]]
    host.set_target(xt2 / sc.D_c)
    dev.set_target_unscaled(xt2)
    host.solve(PARAMS, 1.0)
    dev.solve(PARAMS, 1.0)
    assert np.array_equal(sc.D_c * host.pdhg_x, dev.get_unscaled("pdhg_x"))


def test_batch_members_scale_independently(oracle):
    probs, scs, xts = [], [], []
    for seed in (3, 4, 5):
        milp, sc, is_eq, is_int, w, xt, _ = _problem(oracle, seed)
        probs.append((sc.A, sc.con_ub, is_eq, is_int, sc.var_lb, sc.var_ub, w))
        scs.append(sc)
        xts.append(xt)
    host = gpu.PDFPBatch(probs, precision="mixed")
    dev = gpu.PDFPBatch(probs, precision="mixed")
    for p, sc in enumerate(scs):
        dev.set_col_scale(p, sc.D_c)
        host.set_target(p, xts[p] / sc.D_c)
        dev.set_target_unscaled(p, xts[p])
    host.solve(PARAMS, 1.0)
    dev.solve(PARAMS, 1.0)
    for p, sc in enumerate(scs):
        assert np.array_equal(sc.D_c * host.get(p, "pdhg_x"), dev.get_unscaled(p, "pdhg_x"))


def test_errors_leave_state_untouched(oracle):
    milp, sc, is_eq, is_int, w, xt, _ = _problem(oracle)
    s = _state(sc, is_eq, is_int, w, "fp64")
    with pytest.raises(Exception, match="no column scale"):
        s.set_target_unscaled(xt)
    with pytest.raises(Exception, match="no column scale"):
        s.get_unscaled("pdhg_x")
    for bad in (0.0, -1.0, np.nan, np.inf):
        d = sc.D_c.copy()
        d[7] = bad
        with pytest.raises(Exception, match="positive and finite"):
            s.set_col_scale(d)
    s.set_col_scale(sc.D_c)
    s.set_target_unscaled(xt)
    before = s.get("pdhg_x")
    bad = xt.copy()
    bad[11] = np.nan
    with pytest.raises(Exception, match="NaN in the target"):
        s.set_target_unscaled(bad)
    with pytest.raises(Exception, match="NaN in the target"):
        s.set_target(bad / sc.D_c)
    with pytest.raises(Exception, match="NaN in the start point"):
        s.set_x_unscaled(bad)
    with pytest.raises(Exception, match="unscaled form"):
        s.get_unscaled("pdhg_y")
    assert np.array_equal(before, s.get("pdhg_x"))
    # the handle still solves to the same point as a fresh one given the same target
    fresh = _state(sc, is_eq, is_int, w, "fp64")
    fresh.set_target(xt / sc.D_c)
    s.solve(PARAMS, 1.0)
    fresh.solve(PARAMS, 1.0)
    assert np.array_equal(s.pdhg_x, fresh.pdhg_x)


def test_pinned_arrays_round_trip(oracle):
    milp, sc, is_eq, is_int, w, xt, _ = _problem(oracle)
    n = len(xt)
    a = gpu.pinned_zeros(n)
    assert a.shape == (n,) and a.dtype == np.float64 and not a.any()
    a[:] = xt
    out = gpu.pinned_zeros(n)
    s = _state(sc, is_eq, is_int, w, "mixed")
    s.set_col_scale(sc.D_c)
    s.set_target_unscaled(a)
    s.solve(PARAMS, 1.0)
    got = s.get_unscaled("pdhg_x", out=out)
    assert got.base is not None and np.shares_memory(got, out)
    assert np.array_equal(got, sc.D_c * s.pdhg_x)
    with pytest.raises(ValueError):
        s.get_unscaled("pdhg_x", out=np.zeros(n - 1))
    del a, out, got  # frees the page-locked blocks


def test_set_device_selects_and_validates():
    from pdfp_b200 import _lib as L
    gpu.set_device(0)
    assert gpu.device_name()
    with pytest.raises(Exception, match="out of range"):
        gpu.set_device(4096)
    assert L.lib().pdfp_set_device(-1) != 0
