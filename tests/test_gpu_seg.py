"""The A side's long rows by column segment (seg_spmv.cuh) against the tile engine.

PDFP_SEG="n,l" regroups the rows of at least l nonzeros into n column segments:
one block per segment gathers from its segment of x_bar in shared memory, a
second launch adds each row's partials in segment order and runs the z update,
and the tile engine takes the other rows.  Mixed form (FP32 steps): the same
status, iteration counts within 5% and l1 distances within 1e-3 relative as the
plain tile engine, for several segmentations (one segment; segments too narrow
for some rows, which then stay on the tile engine); two solves agree bit for
bit; a batch handle with the form agrees member by member.
"""
import numpy as np
import pytest

from pdfp_b200 import gpu, synthetic
from pdfp_b200.params import SolverParameters

pytestmark = pytest.mark.gpu

PRM = SolverParameters(eps_optimal_relative=1e-4, eps_feasible_relative=1e-4)


def model(seed=3, m=4000, n=20000, nnz=300_000):
    milp, _ = synthetic.zipf_lp(seed=seed, m=m, n=n, nnz=nnz)
    rng = np.random.default_rng(seed + 5)
    I = milp.int_idx
    xt = np.zeros(len(milp.c))
    xt[I] = np.round(rng.random(len(I)))
    return milp, xt


@pytest.fixture(scope="module")
def zipf(oracle):
    milp, xt = model()
    assert (np.diff(milp.A.indptr) >= 256).sum() > 50
    return milp, xt, oracle.projector_inputs(milp)


def solve(zipf, prm=PRM):
    milp, xt, (sc, is_eq, is_int, w) = zipf
    s = gpu.PDFPState(sc.A, sc.con_ub, is_eq, is_int, sc.var_lb, sc.var_ub, w, precision="mixed")
    s.set_target(xt / sc.D_c)
    st = s.solve(prm, 1.0)
    I = milp.int_idx
    l1 = float(np.sum(w[I] * np.abs(s.pdhg_x[I] - xt[I] / sc.D_c[I])))
    return s, st, l1


def seg_of(s):
    out = (gpu.C.c_int32 * 2)()
    gpu.L.check(gpu.L.lib().pdfp_get_tuning_seg(s._h, out))
    return list(out)


@pytest.fixture(scope="module")
def tile_answer(zipf):
    mp = pytest.MonkeyPatch()
    mp.setenv("PDFP_STEP_ENGINE", "tile")
    mp.setenv("PDFP_SEG", "0")
    try:
        s, st, l1 = solve(zipf)
        assert seg_of(s) == [0, 0]
        return st, s.total_count, l1
    finally:
        mp.undo()


@pytest.mark.parametrize("seg", ["1,256", "16,256", "148,512", "296,128", "2000,64"])
def test_seg_agrees_with_tile(zipf, tile_answer, monkeypatch, seg):
    monkeypatch.setenv("PDFP_STEP_ENGINE", "tile")
    monkeypatch.setenv("PDFP_SEG", seg)
    s, st, l1 = solve(zipf)
    n, l = map(int, seg.split(","))
    assert seg_of(s) == [n, l]
    st0, cnt0, l10 = tile_answer
    assert st == st0 == "OPTIMAL"
    assert abs(s.total_count - cnt0) <= 0.05 * cnt0 + 64
    assert l1 == pytest.approx(l10, rel=1e-3)


def test_seg_is_deterministic(zipf, monkeypatch):
    monkeypatch.setenv("PDFP_STEP_ENGINE", "tile")
    monkeypatch.setenv("PDFP_SEG", "148,256")
    prm = SolverParameters(eps_optimal_relative=1e-5, eps_feasible_relative=1e-5)
    out = []
    for _ in range(2):
        s, st, _ = solve(zipf, prm)
        out.append((st, s.total_count, s.pdhg_x, s.get("pdhg_z"), s.get("current_y")))
    assert out[0][0] == out[1][0] == "OPTIMAL" and out[0][1] == out[1][1]
    for a, b in zip(out[0][2:], out[1][2:]):
        assert np.array_equal(a, b)


def test_seg_in_a_batch(oracle, monkeypatch):
    """Three zipf members in one handle: long rows of every member in the same
    segments of the packed columns; each member's answer as without the form."""
    members = [model(seed=s, m=2000, n=8000, nnz=120_000) for s in (11, 12, 13)]
    probs = []
    for milp, xt in members:
        sc, is_eq, is_int, w = oracle.projector_inputs(milp)
        probs.append((sc, is_eq, is_int, w, milp, xt))
    res = {}
    monkeypatch.setenv("PDFP_STEP_ENGINE", "tile")
    for seg in ("0", "64,128"):
        monkeypatch.setenv("PDFP_SEG", seg)
        b = gpu.PDFPBatch([(sc.A, sc.con_ub, is_eq, is_int, sc.var_lb, sc.var_ub, w)
                           for sc, is_eq, is_int, w, _, _ in probs], precision="mixed")
        got = seg_of(b)
        assert got == ([0, 0] if seg == "0" else [64, 128])
        for p, (sc, _, _, _, milp, xt) in enumerate(probs):
            b.set_target(p, xt / sc.D_c)
        sts = b.solve(PRM, 1.0)
        res[seg] = [(st, r["total_count"], b.get(p, "pdhg_x")) for p, (st, r) in
                    enumerate(zip(sts, b.results))]
    for p, (sc, is_eq, is_int, w, milp, xt) in enumerate(probs):
        (s0, c0, x0), (s1, c1, x1) = res["0"][p], res["64,128"][p]
        assert s0 == s1 == "OPTIMAL"
        assert abs(c0 - c1) <= 0.05 * c0 + 64
        I = milp.int_idx
        l0 = np.sum(w[I] * np.abs(x0[I] - xt[I] / sc.D_c[I]))
        l1 = np.sum(w[I] * np.abs(x1[I] - xt[I] / sc.D_c[I]))
        assert l1 == pytest.approx(l0, rel=1e-3)


@pytest.mark.parametrize("bad", ["abc", "5", "0,3", "-1,4"])
def test_seg_bad_env(zipf, monkeypatch, bad):
    monkeypatch.setenv("PDFP_SEG", bad)
    with pytest.raises(Exception, match="PDFP_SEG"):
        solve(zipf)


def test_seg_off_by_default_and_tune_accepted(zipf, monkeypatch):
    """Unset, the long rows stay on the step engine; PDFP_SEG=tune hands the choice
    to the autotuner (which tries segmentations on handles of at least 2^22 nonzeros
    only, so this smaller handle keeps the plain form)."""
    monkeypatch.delenv("PDFP_STEP_ENGINE", raising=False)
    monkeypatch.delenv("PDFP_SEG", raising=False)
    s, st, _ = solve(zipf)
    assert st == "OPTIMAL" and seg_of(s) == [0, 0]
    monkeypatch.setenv("PDFP_SEG", "tune")
    s, st, _ = solve(zipf)
    assert st == "OPTIMAL" and seg_of(s) == [0, 0]
