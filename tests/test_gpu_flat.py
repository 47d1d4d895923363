"""The flat step engine (flat_spmv.cuh) against the oracle and the tile engine.

PDFP_STEP_ENGINE fixes the engine of handles created while it is set.  FP64:
the flat engine takes the oracle's steps (same status and iteration count,
iterates within 1e-10).  Mixed: flat and tile engines agree (same status,
iteration counts within 5%, l1 distances within 1e-6 relative) on a matrix
with rows longer than a tile.
"""
import numpy as np
import pytest

from pdfp_b200 import gpu, synthetic
from pdfp_b200.params import SolverParameters

pytestmark = pytest.mark.gpu


def project(oracle, milp, xt, tol, precision, engine, monkeypatch):
    monkeypatch.setenv("PDFP_STEP_ENGINE", engine)
    sc, is_eq, is_int, w = oracle.projector_inputs(milp)
    s = gpu.PDFPState(sc.A, sc.con_ub, is_eq, is_int, sc.var_lb, sc.var_ub, w, precision=precision)
    tun = (gpu.C.c_int32 * 8)()
    gpu.L.check(gpu.L.lib().pdfp_get_tuning(s._h, tun))
    s.set_target(np.asarray(xt, dtype=np.float64) / sc.D_c)
    st = s.solve(SolverParameters(eps_optimal_relative=tol, eps_feasible_relative=tol), 1.0)
    return sc.D_c * s.pdhg_x, st, s.total_count, list(tun), sc, w


@pytest.mark.parametrize("engine", ["flat", "flat1"])
@pytest.mark.parametrize("name", ["p0201", "pk1", "gen-ip054"])
def test_flat_fp64_matches_oracle(oracle, examples, name, engine, monkeypatch):
    m = examples[name]
    xt = np.round(np.random.default_rng(4).random(len(m.c)) * (np.minimum(m.u, 3) - m.l) + m.l)
    x, st, cnt, tun, sc, w = project(oracle, m, xt, 1e-6, "fp64", engine, monkeypatch)
    assert tun[1] == 0 and tun[4] == 0  # both sides on the flat engine
    xo, so, o = oracle.project(m, xt, tol=1e-6)
    assert st == so and cnt == o.total_count
    assert np.abs(x - xo).max() <= 1e-10


def test_flat_and_tile_agree_mixed_with_long_rows(oracle, monkeypatch):
    milp, _ = synthetic.zipf_lp(seed=3, m=4000, n=20000, nnz=300_000)
    rng = np.random.default_rng(8)
    I = milp.int_idx
    xt = np.zeros(len(milp.c))
    xt[I] = np.round(rng.random(len(I)))
    assert np.diff(milp.A.indptr).max() > 2048  # some rows span several chunks
    res = {}
    for eng in ("tile", "flat", "flat1"):
        x, st, cnt, tun, sc, w = project(oracle, milp, xt, 1e-4, "mixed", eng, monkeypatch)
        l1 = float(np.sum(w[I] * np.abs(x[I] - xt[I]) / sc.D_c[I]))
        res[eng] = (st, cnt, l1)
    for eng in ("flat", "flat1"):
        assert res["tile"][0] == res[eng][0] == "OPTIMAL"
        assert abs(res["tile"][1] - res[eng][1]) <= 0.05 * res["tile"][1] + 64
        assert res[eng][2] == pytest.approx(res["tile"][2], rel=1e-3)
