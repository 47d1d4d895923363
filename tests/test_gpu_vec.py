"""The vec step engine (vec_spmv.cuh): rows read straight from the CSR arrays,
G lanes per row, long rows in pieces summed in FP64 by the warp that finishes
the row's last piece.

It runs the FP32 steps of the mixed form only.  Against the tile engine on a
matrix whose longest rows span several pieces: the same status, iteration
counts within 5% and l1 distances within 1e-3 relative for every choice of
nonzeros per lane and both gather cache policies; two solves agree bit for bit
(the pieces of a row are added in piece order whichever warp finishes last).
"""
import numpy as np
import pytest

from pdfp_b200 import gpu, synthetic
from pdfp_b200.params import SolverParameters

pytestmark = pytest.mark.gpu

PRM = SolverParameters(eps_optimal_relative=1e-4, eps_feasible_relative=1e-4)


@pytest.fixture(scope="module")
def zipf(oracle):
    milp, _ = synthetic.zipf_lp(seed=3, m=4000, n=20000, nnz=300_000)
    rng = np.random.default_rng(8)
    I = milp.int_idx
    xt = np.zeros(len(milp.c))
    xt[I] = np.round(rng.random(len(I)))
    assert np.diff(milp.A.indptr).max() > 2048  # rows of two pieces (2,048 nonzeros a piece)
    return milp, xt, oracle.projector_inputs(milp)


def solve(zipf, precision, prm=PRM):
    milp, xt, (sc, is_eq, is_int, w) = zipf
    s = gpu.PDFPState(sc.A, sc.con_ub, is_eq, is_int, sc.var_lb, sc.var_ub, w, precision=precision)
    s.set_target(xt / sc.D_c)
    st = s.solve(prm, 1.0)
    I = milp.int_idx
    l1 = float(np.sum(w[I] * np.abs(s.pdhg_x[I] - xt[I] / sc.D_c[I])))
    return s, st, l1


@pytest.fixture(scope="module")
def tile_answer(zipf):
    mp = pytest.MonkeyPatch()
    mp.setenv("PDFP_STEP_ENGINE", "tile")
    try:
        s, st, l1 = solve(zipf, "mixed")
        return st, s.total_count, l1
    finally:
        mp.undo()


@pytest.mark.parametrize("lane_nnz", [1, 2, 4, 8])
@pytest.mark.parametrize("policy", [0, 1])
def test_vec_agrees_with_tile(zipf, tile_answer, monkeypatch, lane_nnz, policy):
    monkeypatch.delenv("PDFP_STEP_ENGINE", raising=False)
    monkeypatch.setenv("PDFP_TUNING", f"{lane_nnz},32,{policy},{lane_nnz},32,{policy}")
    s, st, l1 = solve(zipf, "mixed")
    tun = s.tuning()
    assert (tun[0], tun[1], tun[3], tun[4], tun[6], tun[7]) == (lane_nnz, 32, lane_nnz, 32, policy, policy)
    assert tun[2] > 0 and tun[5] > 0  # items per side
    st0, cnt0, l10 = tile_answer
    assert st == st0 == "OPTIMAL"
    assert abs(s.total_count - cnt0) <= 0.05 * cnt0 + 64
    assert l1 == pytest.approx(l10, rel=1e-3)


def test_vec_is_deterministic(zipf, monkeypatch):
    monkeypatch.setenv("PDFP_STEP_ENGINE", "vec")
    prm = SolverParameters(eps_optimal_relative=1e-5, eps_feasible_relative=1e-5)
    out = []
    for _ in range(2):
        s, st, _ = solve(zipf, "mixed", prm)
        assert s.tuning()[1] == 32 and s.tuning()[4] == 32
        out.append((st, s.total_count, s.pdhg_x, s.get("pdhg_z"), s.get("current_y")))
    assert out[0][0] == out[1][0] == "OPTIMAL" and out[0][1] == out[1][1]
    for a, b in zip(out[0][2:], out[1][2:]):
        assert np.array_equal(a, b)


def test_vec_leaves_fp64_steps_on_the_tile_engine(zipf, oracle, monkeypatch):
    """PDFP_STEP_ENGINE=vec on an FP64 handle: its steps stay on an engine that
    takes the oracle's steps (same status and count, iterates within 1e-10)."""
    milp, xt, (sc, is_eq, is_int, w) = zipf
    monkeypatch.setenv("PDFP_STEP_ENGINE", "vec")
    prm = SolverParameters(eps_optimal_relative=1e-4, eps_feasible_relative=1e-4)
    s, st, _ = solve(zipf, "fp64", prm)
    assert s.tuning()[1] != 32 and s.tuning()[4] != 32
    o = oracle.OracleSolvers.PDFPState(sc.A, sc.con_ub, is_eq, is_int, sc.var_lb, sc.var_ub, w)
    o.set_target(xt / sc.D_c)
    assert st == o.solve(prm, 1.0) and s.total_count == o.total_count
    assert np.abs(s.pdhg_x - o.pdhg_x).max() <= 1e-10


@pytest.mark.parametrize("pin,msg", [("3,32,0,4,32,0", "nonzeros per lane"),
                                     ("4,32,2,4,32,0", "gather policy"),
                                     ("4,32,0,4,32,0,4,4,0,0,16,0", "no reducers")])
def test_vec_bad_pins(zipf, monkeypatch, pin, msg):
    monkeypatch.delenv("PDFP_STEP_ENGINE", raising=False)
    monkeypatch.setenv("PDFP_TUNING", pin)
    with pytest.raises(Exception, match=msg):
        solve(zipf, "mixed")


def window_form(s):
    out = gpu.C.c_int32()
    gpu.L.check(gpu.L.lib().pdfp_get_window_form(s._h, gpu.C.byref(out)))
    return out.value


@pytest.mark.parametrize("tol", [1e-4, 1e-5])
def test_vec_window_equals_per_step_launches(oracle, monkeypatch, tol):
    """PDFP_VEC_WINDOW=1: a window's minor steps in one cooperative launch of the vec
    engine (a grid barrier between the passes) take the same steps as two vec
    launches per step, bit for bit (every row's arithmetic is the same; each row's
    epilogue stays on one warp), on the 20k x 50k general-integer model."""
    milp, _, xt = synthetic.general_integer(1)
    sc, is_eq, is_int, w = oracle.projector_inputs(milp)
    prm = SolverParameters(eps_optimal_relative=tol, eps_feasible_relative=tol)
    monkeypatch.setenv("PDFP_STEP_ENGINE", "vec")
    out = {}
    for vw in ("0", "1"):
        monkeypatch.setenv("PDFP_VEC_WINDOW", vw)
        s = gpu.PDFPState(sc.A, sc.con_ub, is_eq, is_int, sc.var_lb, sc.var_ub, w, precision="mixed")
        assert window_form(s) == (2 if vw == "1" else 0)
        s.set_target(xt / sc.D_c)
        st = s.solve(prm, 1.0)
        out[vw] = (st, s.total_count, s.pdhg_x, s.get("pdhg_z"), s.get("current_y"))
    assert out["0"][0] == out["1"][0] == "OPTIMAL"
    assert out["0"][1] == out["1"][1]
    for a, b in zip(out["0"][2:], out["1"][2:]):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("lane_nnz", [2, 8])
def test_vec_batch_members_equal_single_handles(oracle, monkeypatch, lane_nnz):
    """A batch handle on the vec engine (both sides pinned; PDFP_TINY=0 so that the step
    kernels run instead of the one-block path): five uneven covering/packing members,
    which stop at different iterations.  Each member takes exactly the steps of its own
    single handle: the same status, iteration count and iterates bit for bit.  A row's
    sum does not depend on which work item holds it (nor on the larger items the A'
    side takes when the handle has enough of them), a warp's step parameters are
    recomputed when its item belongs to another member, and the items of members that
    have stopped are skipped."""
    monkeypatch.setenv("PDFP_TUNING", f"{lane_nnz},32,0,{lane_nnz},32,1")
    monkeypatch.setenv("PDFP_TINY", "0")
    models = synthetic.covering_packing_batch(seed=7, k=5, n_min=2000, n_max=20000)
    rng = np.random.default_rng(21)
    probs, targets, dcs = [], [], []
    for m in models:
        sc, is_eq, is_int, w = oracle.projector_inputs(m)
        probs.append((sc.A, sc.con_ub, is_eq, is_int, sc.var_lb, sc.var_ub, w))
        targets.append(np.round(rng.random(len(m.c))) / sc.D_c)
        dcs.append(sc.D_c)
    prm = SolverParameters(eps_optimal_relative=1e-4, eps_feasible_relative=1e-5)
    b = gpu.PDFPBatch(probs, precision="mixed")
    assert b.tuning()[1] == 32 and b.tuning()[4] == 32  # both sides on the vec engine
    for p, xt in enumerate(targets):
        b.set_target(p, xt)
    st = b.solve(prm, 1.0)
    counts = [r["total_count"] for r in b.results]
    assert len(set(counts)) > 1  # members stop at different iterations
    for p, pr in enumerate(probs):
        s = gpu.PDFPState(*pr, precision="mixed")
        s.set_target(targets[p])
        assert s.solve(prm, 1.0) == st[p], p
        assert s.total_count == counts[p], p
        assert np.array_equal(s.pdhg_x, b.get(p, "pdhg_x")), p
