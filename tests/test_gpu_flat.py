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


def test_tuning_pin_and_bad_pin(oracle, examples, monkeypatch):
    m = examples["pk1"]
    xt = np.round(np.random.default_rng(2).random(len(m.c)))
    monkeypatch.delenv("PDFP_STEP_ENGINE", raising=False)
    monkeypatch.setenv("PDFP_TUNING", "12288,128,0,0,0,1")
    sc, is_eq, is_int, w = oracle.projector_inputs(m)
    s = gpu.PDFPState(sc.A, sc.con_ub, is_eq, is_int, sc.var_lb, sc.var_ub, w, precision="mixed")
    tun = (gpu.C.c_int32 * 8)()
    gpu.L.check(gpu.L.lib().pdfp_get_tuning(s._h, tun))
    assert (tun[0], tun[1], tun[4], tun[6], tun[7]) == (12288, 128, 0, 0, 1)
    s.set_target(xt / sc.D_c)
    assert s.solve(SolverParameters(eps_optimal_relative=1e-4, eps_feasible_relative=1e-4), 1.0) == "OPTIMAL"
    monkeypatch.setenv("PDFP_TUNING", "100,128,0,0,0,1")
    with pytest.raises(Exception, match="stage bytes"):
        gpu.PDFPState(sc.A, sc.con_ub, is_eq, is_int, sc.var_lb, sc.var_ub, w, precision="mixed")


def test_small_mixed_handles_compute_in_fp64(oracle, examples, monkeypatch):
    """Below 2^18 nonzeros a mixed handle is an FP64 handle (same steps, same
    answer); PDFP_MIXED_MIN_NNZ=0 keeps FP32."""
    m = examples["p0201"]
    xt = np.round(np.random.default_rng(6).random(len(m.c)))
    sc, is_eq, is_int, w = oracle.projector_inputs(m)
    prm = SolverParameters(eps_optimal_relative=1e-4, eps_feasible_relative=1e-4)
    out = {}
    for label, prec, env in [("fp64", "fp64", None), ("auto", "mixed", None), ("fp32", "mixed", "0")]:
        if env is None:
            monkeypatch.delenv("PDFP_MIXED_MIN_NNZ", raising=False)
        else:
            monkeypatch.setenv("PDFP_MIXED_MIN_NNZ", env)
        s = gpu.PDFPState(sc.A, sc.con_ub, is_eq, is_int, sc.var_lb, sc.var_ub, w, precision=prec)
        s.set_target(xt / sc.D_c)
        s.solve(prm, 1.0)
        out[label] = (s.last["precision"], s.total_count, s.pdhg_x)
    assert out["auto"][0] == gpu.L.FP64 and out["fp32"][0] == gpu.L.MIXED
    assert out["auto"][1] == out["fp64"][1] and np.array_equal(out["auto"][2], out["fp64"][2])


@pytest.mark.parametrize("name", ["p0201", "pk1", "markshare2"])
def test_one_launch_minor_steps(oracle, examples, name, monkeypatch):
    """Small members run a window's minor steps in one launch.  FP64: the oracle's
    steps (status, iteration count, iterates within 1e-10); mixed: the two-launch
    form's answer (same status, counts within 5%, l1 distance within 1e-6 relative)."""
    m = examples[name]
    xt = np.round(np.random.default_rng(8).random(len(m.c)) * (np.minimum(m.u, 2) - m.l) + m.l)
    sc, is_eq, is_int, w = oracle.projector_inputs(m)
    prm = SolverParameters(eps_optimal_relative=1e-6, eps_feasible_relative=1e-6)
    monkeypatch.setenv("PDFP_TINY", "1")
    s = gpu.PDFPState(sc.A, sc.con_ub, is_eq, is_int, sc.var_lb, sc.var_ub, w, precision="fp64")
    s.set_target(xt / sc.D_c)
    st = s.solve(prm, 1.0)
    o = oracle.OracleSolvers.PDFPState(sc.A, sc.con_ub, is_eq, is_int, sc.var_lb, sc.var_ub, w)
    o.set_target(xt / sc.D_c)
    assert st == o.solve(prm, 1.0) and s.total_count == o.total_count
    assert np.abs(s.pdhg_x - o.pdhg_x).max() <= 1e-10
    res = {}
    for tiny in ("0", "1"):
        monkeypatch.setenv("PDFP_TINY", tiny)
        s = gpu.PDFPState(sc.A, sc.con_ub, is_eq, is_int, sc.var_lb, sc.var_ub, w, precision="mixed")
        s.set_target(xt / sc.D_c)
        st = s.solve(SolverParameters(eps_optimal_relative=1e-4, eps_feasible_relative=1e-4), 1.0)
        I = m.int_idx
        res[tiny] = (st, s.total_count, float(np.sum(w[I] * np.abs(s.pdhg_x[I] - xt[I] / sc.D_c[I]))))
    assert res["0"][0] == res["1"][0]
    assert abs(res["0"][1] - res["1"][1]) <= 0.05 * res["0"][1] + 200
    assert res["1"][2] == pytest.approx(res["0"][2], rel=1e-6, abs=1e-9)


@pytest.mark.parametrize("pin", ["12288,128,{p},16384,128,{p},4,3", "24576,128,{p},24576,256,{p},2,4"])
def test_async_gathers_equal_register_gathers(oracle, monkeypatch, pin):
    """Gather policy 2 (per-thread async copies into the stage; the reducers form the
    products) computes every product and sum with the same roundings in the same
    order as the register gathers: the solves must agree bit for bit, long rows
    spanning several chunks included."""
    milp, _ = synthetic.zipf_lp(seed=3, m=4000, n=20000, nnz=300_000)
    rng = np.random.default_rng(8)
    I = milp.int_idx
    xt = np.zeros(len(milp.c))
    xt[I] = np.round(rng.random(len(I)))
    monkeypatch.delenv("PDFP_STEP_ENGINE", raising=False)
    sc, is_eq, is_int, w = oracle.projector_inputs(milp)
    out = {}
    for policy in (0, 2):
        monkeypatch.setenv("PDFP_TUNING", pin.format(p=policy))
        s = gpu.PDFPState(sc.A, sc.con_ub, is_eq, is_int, sc.var_lb, sc.var_ub, w, precision="mixed")
        tun = (gpu.C.c_int32 * 8)()
        gpu.L.check(gpu.L.lib().pdfp_get_tuning(s._h, tun))
        assert (tun[6], tun[7]) == (policy, policy)
        s.set_target(xt / sc.D_c)
        st = s.solve(SolverParameters(eps_optimal_relative=1e-5, eps_feasible_relative=1e-5), 1.0)
        out[policy] = (st, s.total_count, s.pdhg_x, s.get("pdhg_z"), s.get("current_y"))
    assert out[0][0] == out[2][0] == "OPTIMAL"
    assert out[0][1] == out[2][1]
    for a, b in zip(out[0][2:], out[2][2:]):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_overlapped_step_launches_change_nothing(oracle, monkeypatch, precision):
    """Consecutive step launches overlap one grid's drain with the next one's staging
    (programmatic dependent launch); every read of the previous grid's output waits
    for it, so the solves with and without the overlap agree bit for bit."""
    milp, _ = synthetic.zipf_lp(seed=5, m=3000, n=12000, nnz=150_000)
    rng = np.random.default_rng(9)
    I = milp.int_idx
    xt = np.zeros(len(milp.c))
    xt[I] = np.round(rng.random(len(I)))
    monkeypatch.delenv("PDFP_STEP_ENGINE", raising=False)
    monkeypatch.setenv("PDFP_AUTOTUNE", "0")
    sc, is_eq, is_int, w = oracle.projector_inputs(milp)
    out = {}
    for ov in ("0", "1"):
        monkeypatch.setenv("PDFP_STEP_OVERLAP", ov)
        s = gpu.PDFPState(sc.A, sc.con_ub, is_eq, is_int, sc.var_lb, sc.var_ub, w, precision=precision)
        s.set_target(xt / sc.D_c)
        st = s.solve(SolverParameters(eps_optimal_relative=1e-5, eps_feasible_relative=1e-5), 1.0)
        out[ov] = (st, s.total_count, s.pdhg_x, s.get("pdhg_z"), s.get("current_y"))
    assert out["0"][0] == out["1"][0] == "OPTIMAL"
    assert out["0"][1] == out["1"][1]
    for a, b in zip(out["0"][2:], out["1"][2:]):
        assert np.array_equal(a, b)


def test_blocks_per_sm_cap_changes_nothing(oracle, monkeypatch):
    """A cap on resident blocks per SM (with the launch's shared-memory carveout
    sized for it) changes only where the tiles run: the same solve bit for bit."""
    milp, _ = synthetic.zipf_lp(seed=3, m=4000, n=20000, nnz=300_000)
    rng = np.random.default_rng(8)
    I = milp.int_idx
    xt = np.zeros(len(milp.c))
    xt[I] = np.round(rng.random(len(I)))
    monkeypatch.delenv("PDFP_STEP_ENGINE", raising=False)
    sc, is_eq, is_int, w = oracle.projector_inputs(milp)
    out = {}
    for cap in (0, 2):
        monkeypatch.setenv("PDFP_TUNING", f"12288,128,0,24576,128,1,3,2,{cap},{cap}")
        s = gpu.PDFPState(sc.A, sc.con_ub, is_eq, is_int, sc.var_lb, sc.var_ub, w, precision="mixed")
        blk = (gpu.C.c_int32 * 2)()
        gpu.L.check(gpu.L.lib().pdfp_get_tuning_blocks(s._h, blk))
        assert list(blk) == [cap, cap]
        s.set_target(xt / sc.D_c)
        st = s.solve(SolverParameters(eps_optimal_relative=1e-5, eps_feasible_relative=1e-5), 1.0)
        out[cap] = (st, s.total_count, s.pdhg_x, s.get("pdhg_z"))
    assert out[0][0] == out[2][0] == "OPTIMAL" and out[0][1] == out[2][1]
    for a, b in zip(out[0][2:], out[2][2:]):
        assert np.array_equal(a, b)
    monkeypatch.setenv("PDFP_TUNING", "12288,128,0,24576,128,1,3,2,9,0")
    with pytest.raises(Exception, match="blocks per SM"):
        gpu.PDFPState(sc.A, sc.con_ub, is_eq, is_int, sc.var_lb, sc.var_ub, w, precision="mixed")


def test_half_size_reducer_role_agrees(oracle, monkeypatch):
    """256 gatherers with 128 reducers: the row sums group lanes by the reducer count,
    so roundings may differ from the 256/256 kernel; the projection agrees within the
    mixed-form tolerances (same status, iteration counts within 5%, l1 distances within
    1e-3 relative), long rows spanning several chunks included."""
    milp, _ = synthetic.zipf_lp(seed=3, m=4000, n=20000, nnz=300_000)
    rng = np.random.default_rng(8)
    I = milp.int_idx
    xt = np.zeros(len(milp.c))
    xt[I] = np.round(rng.random(len(I)))
    monkeypatch.delenv("PDFP_STEP_ENGINE", raising=False)
    sc, is_eq, is_int, w = oracle.projector_inputs(milp)
    res = {}
    for red in (256, 128):
        monkeypatch.setenv("PDFP_TUNING", f"16384,256,0,24576,256,1,3,2,0,0,{red},{red}")
        s = gpu.PDFPState(sc.A, sc.con_ub, is_eq, is_int, sc.var_lb, sc.var_ub, w, precision="mixed")
        r = (gpu.C.c_int32 * 2)()
        gpu.L.check(gpu.L.lib().pdfp_get_tuning_reducers(s._h, r))
        assert list(r) == [red, red]
        s.set_target(xt / sc.D_c)
        st = s.solve(SolverParameters(eps_optimal_relative=1e-4, eps_feasible_relative=1e-4), 1.0)
        x = sc.D_c * s.pdhg_x
        res[red] = (st, s.total_count, float(np.sum(w[I] * np.abs(x[I] - xt[I]) / sc.D_c[I])))
    assert res[256][0] == res[128][0] == "OPTIMAL"
    assert abs(res[256][1] - res[128][1]) <= 0.05 * res[256][1] + 64
    assert res[128][2] == pytest.approx(res[256][2], rel=1e-3)
    monkeypatch.setenv("PDFP_TUNING", "16384,256,0,24576,256,1,3,2,0,0,96,0")
    with pytest.raises(Exception, match="reducers"):
        gpu.PDFPState(sc.A, sc.con_ub, is_eq, is_int, sc.var_lb, sc.var_ub, w, precision="mixed")


@pytest.mark.parametrize("name", ["p0201", "pk1", "gen-ip054"])
def test_medium_path_fp64_matches_oracle(oracle, examples, name, monkeypatch):
    """A window's minor steps in one cooperative launch (one block per SM over
    nonzero-balanced row ranges, grid barriers between the passes), forced on the
    example models: the FP64 form takes the oracle's steps (same status and
    iteration count, iterates within 1e-10)."""
    monkeypatch.setenv("PDFP_TINY", "0")
    monkeypatch.setenv("PDFP_MEDIUM", "1")
    m = examples[name]
    xt = np.round(np.random.default_rng(4).random(len(m.c)) * (np.minimum(m.u, 3) - m.l) + m.l)
    x, st, cnt, tun, sc, w = project(oracle, m, xt, 1e-6, "fp64", "tile", monkeypatch)
    xo, so, o = oracle.project(m, xt, tol=1e-6)
    assert st == so and cnt == o.total_count
    assert np.abs(x - xo).max() <= 1e-10


def test_medium_path_agrees_with_tile_engine_mixed(oracle, monkeypatch):
    """The cooperative path against the per-step launches on a matrix with rows longer
    than a block's share of work, in the mixed form, batch of two members: same
    status, iteration counts within 5%, l1 distances within 1e-3 relative."""
    milp, _ = synthetic.zipf_lp(seed=3, m=4000, n=20000, nnz=300_000)
    rng = np.random.default_rng(8)
    I = milp.int_idx
    sc, is_eq, is_int, w = oracle.projector_inputs(milp)
    xts = []
    for _ in range(2):
        xt = np.zeros(len(milp.c))
        xt[I] = np.round(rng.random(len(I)))
        xts.append(xt)
    res = {}
    for med in ("0", "1"):
        monkeypatch.setenv("PDFP_MEDIUM", med)
        b = gpu.PDFPBatch([(sc.A, sc.con_ub, is_eq, is_int, sc.var_lb, sc.var_ub, w)] * 2,
                          precision="mixed")
        for p in range(2):
            b.set_target(p, xts[p] / sc.D_c)
        b.solve(SolverParameters(eps_optimal_relative=1e-4, eps_feasible_relative=1e-4), 1.0)
        out = []
        for p in range(2):
            x = sc.D_c * b.get(p, "pdhg_x")
            out.append((b.results[p]["status"], b.results[p]["total_count"],
                        float(np.sum(w[I] * np.abs(x[I] - xts[p][I]) / sc.D_c[I]))))
        res[med] = out
        b.close()
    for p in range(2):
        assert res["0"][p][0] == res["1"][p][0] == "OPTIMAL"
        assert abs(res["0"][p][1] - res["1"][p][1]) <= 0.05 * res["0"][p][1] + 64
        assert res["1"][p][2] == pytest.approx(res["0"][p][2], rel=1e-3)
