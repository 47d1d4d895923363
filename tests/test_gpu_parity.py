"""GPU parity of the projector, the preconditioner and the power iteration.

Every test calls libpdfp_b200.so through its C ABI (pdfp_b200.gpu) and compares
with the CPU oracle (oracle/) on the same seeded inputs.  Tolerances:

* scale_problem: bit-identical factors and scaled values (the reference's
  ascending-order sums are reproduced exactly).
* power iteration: identical estimate to 1e-12 relative, same iteration count.
* FP64 projector: the same termination reason and iteration count as the
  oracle, iterates within 1e-10 absolute (only reductions differ in order).
* Mixed projector: the reference's GPU-vs-CPU test (test/runtests.jl:81-88,
  l1 distance within rtol 1e-4); solved tightly (1e-7) its l1 distance is
  within 1e-6 relative of the oracle's; its KKT residuals re-evaluated in FP64
  on the host are within the requested tolerance.
"""
import numpy as np
import pytest
import scipy.sparse as sp

from pdfp_b200 import gpu
from pdfp_b200.milp import MILP
from pdfp_b200.params import SolverParameters
from pdfp_b200 import synthetic

pytestmark = pytest.mark.gpu


def proj_inputs(oracle, milp):
    return oracle.projector_inputs(milp)


def gpu_project(oracle, milp, x_tilde, tol, precision, primal_weight=1.0, iteration_limit=1_000_000,
                eps_feas=None):
    sc, is_eq, is_int, w = proj_inputs(oracle, milp)
    s = gpu.PDFPState(sc.A, sc.con_ub, is_eq, is_int, sc.var_lb, sc.var_ub, w, precision=precision)
    s.set_target(np.asarray(x_tilde, dtype=np.float64) / sc.D_c)
    p = SolverParameters(eps_optimal_relative=tol,
                         eps_feasible_relative=tol if eps_feas is None else eps_feas,
                         iteration_limit=iteration_limit)
    status = s.solve(p, primal_weight)
    return sc.D_c * s.pdhg_x, status, s, sc


def kkt(sc, is_eq, is_int, w, xt_scaled, s, row_unscale=None):
    """compute_residual! (src/pdfp.jl:200-218) in FP64 on the host from the GPU's vectors."""
    x, y, z, ds = s.get("pdhg_x"), s.get("pdhg_y"), s.get("pdhg_z"), s.get("dual_slack")
    A, b = sc.A, sc.con_ub
    d = A @ x - b
    viol = np.where(is_eq, np.abs(d), np.maximum(d, 0.0))
    if row_unscale is not None:
        viol = viol * row_unscale
        bnorm = np.linalg.norm(b * row_unscale)
    else:
        bnorm = np.linalg.norm(b)
    rel_p = np.linalg.norm(viol) / (1.0 + bnorm)
    rel_d = np.linalg.norm(A.T @ z - y - ds) / (1.0 + np.linalg.norm(np.where(is_int, w, 0.0)))
    l1 = np.sum(np.where(is_int, w * np.abs(x - xt_scaled), 0.0))
    yt = np.sum(np.where(is_int, y * (xt_scaled - x), 0.0))
    gap = abs(yt + z @ d - l1) / (1.0 + np.sum(np.where(is_int, w * np.abs(xt_scaled), 0.0)))
    return rel_p, rel_d, gap


# ---- preconditioner and power iteration -------------------------------------------


@pytest.mark.parametrize("name", ["p0201", "pk1", "gen-ip054", "markshare2"])
@pytest.mark.parametrize("rescale", [False, True])
def test_scale_problem_bit_identical(oracle, examples, name, rescale):
    m = examples[name]
    con_lb = np.where(m.is_eq, m.b, -np.inf)
    g = gpu.scale_problem(m.A, m.c, m.l, m.u, con_lb, m.b, bound_objective_rescaling=rescale)
    o = oracle.scale_problem(m.A, m.c, m.l, m.u, con_lb, m.b, bound_objective_rescaling=rescale)
    assert np.array_equal(g.A.data, o.A.data)
    assert np.array_equal(g.D_r, o.D_r) and np.array_equal(g.D_c, o.D_c)
    for a, b in [(g.c, o.c), (g.var_lb, o.var_lb), (g.var_ub, o.var_ub), (g.con_lb, o.con_lb),
                 (g.con_ub, o.con_ub)]:
        assert np.allclose(a, b, rtol=1e-14, atol=0, equal_nan=True)
    assert g.bound_scale == pytest.approx(o.bound_scale, rel=1e-14)
    assert g.objective_scale == pytest.approx(o.objective_scale, rel=1e-14)


def test_scale_problem_synthetic_general_integer(oracle):
    milp, _, _ = synthetic.general_integer(1, m=2000, n=5000, m_eq=500)
    con_lb = np.where(milp.is_eq, milp.b, -np.inf)
    g = gpu.scale_problem(milp.A, milp.c, milp.l, milp.u, con_lb, milp.b)
    o = oracle.scale_problem(milp.A, milp.c, milp.l, milp.u, con_lb, milp.b)
    assert np.array_equal(g.A.data, o.A.data)
    assert np.array_equal(g.D_r, o.D_r) and np.array_equal(g.D_c, o.D_c)


@pytest.mark.parametrize("name", ["p0201", "pk1"])
def test_power_iteration_matches_oracle(oracle, examples, name):
    sc, *_ = proj_inputs(oracle, examples[name])
    sg, ig = gpu.estimate_max_singular_value(sc.A)
    so, io = oracle.estimate_max_singular_value(sc.A)
    assert sg == pytest.approx(so, rel=1e-12)
    assert ig == io


def test_power_iteration_empty_and_tiny():
    assert gpu.estimate_max_singular_value(sp.csr_matrix(np.array([[3.0]])))[0] == pytest.approx(3.0)
    s, _ = gpu.estimate_max_singular_value(sp.csr_matrix(np.array([[1.0, 0.0], [0.0, 2.0]])))
    assert s == pytest.approx(2.0, rel=1e-4)


# ---- projector known answers (test/runtests.jl:40-55) ---------------------------------


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_toy_projection(oracle, precision):
    m = MILP([0.0, 0.0], 0.0, sp.csr_matrix(np.array([[1.0, 1.0]])), [1.0], ["le"], [0.0, 0.0],
             [1.0, 1.0], [0, 1])
    x, status, s, _ = gpu_project(oracle, m, [1.0, 1.0], 1e-8, precision)
    assert status == "OPTIMAL"
    assert abs(np.abs(x - 1.0).sum() - 1.0) <= 1e-5
    assert x.sum() <= 1.0 + 1e-6


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_general_integer_toy(oracle, precision):
    m = MILP([0.0, 0.0], 0.0, sp.csr_matrix(np.array([[1.0, 1.0]])), [2.0], ["eq"], [0.0, 0.0],
             [5.0, np.inf], [0])
    x, status, _, _ = gpu_project(oracle, m, [3.0, 0.0], 1e-8, precision)
    assert status == "OPTIMAL"
    assert abs(x[0] - 2.0) <= 1e-5


def test_fp64_toys_follow_the_oracle_exactly(oracle):
    m = MILP([0.0, 0.0], 0.0, sp.csr_matrix(np.array([[1.0, 1.0]])), [2.0], ["eq"], [0.0, 0.0],
             [5.0, np.inf], [0])
    xg, sg, s, _ = gpu_project(oracle, m, [3.0, 0.0], 1e-8, "fp64")
    xo, so, o = oracle.project(m, [3.0, 0.0], tol=1e-8)
    assert sg == so and s.total_count == o.total_count
    assert np.abs(xg - xo).max() <= 1e-12


# ---- the reference's GPU parity test (test/runtests.jl:81-88) ----------------------


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_pk1_gpu_vs_cpu_distance(oracle, examples, precision):
    m = examples["pk1"]
    xt = np.round(np.random.default_rng(4).random(len(m.c)))
    I = m.int_idx
    xo, _, o = oracle.project(m, xt, tol=1e-8)
    xg, status, s, _ = gpu_project(oracle, m, xt, 1e-8, precision)
    dg = np.abs(xg[I] - xt[I]).sum()
    do = np.abs(xo[I] - xt[I]).sum()
    assert status == "OPTIMAL"
    assert dg == pytest.approx(do, rel=1e-4, abs=1e-9)


# ---- FP64 projections follow the oracle ---------------------------------------------


@pytest.mark.parametrize("name,tol", [("p0201", 1e-2), ("p0201", 1e-4), ("pk1", 1e-4),
                                      ("gen-ip054", 1e-4), ("markshare2", 1e-3)])
def test_fp64_projection_matches_oracle(oracle, examples, name, tol):
    m = examples[name]
    rng = np.random.default_rng(7)
    xt = m.l.copy()
    I = m.int_idx
    xt[I] = np.round(np.clip(rng.uniform(m.l[I], np.minimum(m.u[I], m.l[I] + 3)), m.l[I], m.u[I]))
    xt[~m.is_int] = np.where(np.isfinite(m.u[~m.is_int]), m.u[~m.is_int], m.l[~m.is_int])
    xo, so, o = oracle.project(m, xt, tol=tol)
    xg, sg, s, _ = gpu_project(oracle, m, xt, tol, "fp64")
    assert sg == so
    assert s.total_count == o.total_count
    assert np.abs(xg - xo).max() <= 1e-10 * max(1.0, np.abs(xo).max())


def test_config0_projection_mixed_and_fp64(oracle):
    milp = synthetic.covering_p0201_like(1)
    rng = np.random.default_rng(11)
    xt = np.round(rng.random(len(milp.c)))
    I = milp.int_idx
    xo, so, o = oracle.project(milp, xt, tol=1e-7)
    do = np.abs(xo[I] - xt[I]).sum()
    for precision in ("fp64", "mixed"):
        xg, sg, s, _ = gpu_project(oracle, milp, xt, 1e-7, precision)
        assert sg == "OPTIMAL"
        dg = np.abs(xg[I] - xt[I]).sum()
        assert dg == pytest.approx(do, rel=1e-6)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_config1_projection_kkt_and_distance(oracle, precision):
    """20k x 50k general-integer model at the benchmark tolerance (1e-4 gap, 1e-5 residual)."""
    milp, x0, xt = synthetic.general_integer(1)
    sc, is_eq, is_int, w = proj_inputs(oracle, milp)
    s = gpu.PDFPState(sc.A, sc.con_ub, is_eq, is_int, sc.var_lb, sc.var_ub, w, precision=precision)
    xts = xt / sc.D_c
    s.set_target(xts)
    status = s.solve(SolverParameters(eps_optimal_relative=1e-4, eps_feasible_relative=1e-5,
                                      iteration_limit=200_000), 1.0)
    assert status == "OPTIMAL"
    rel_p, rel_d, gap = kkt(sc, is_eq, is_int, w, xts, s)
    assert rel_p <= 1e-5 * 1.01 and rel_d <= 1e-4 * 1.01 and gap <= 1e-4 * 1.01
    # the device's FP64 evaluation agrees with the host's
    assert s.last["rel_primal"] == pytest.approx(rel_p, rel=1e-6, abs=1e-12)
    assert s.last["rel_gap"] == pytest.approx(gap, rel=1e-6, abs=1e-12)
    if precision == "fp64":
        o = oracle.OraclePDFP(sc.A, sc.con_ub, is_eq, is_int, sc.var_lb, sc.var_ub, w)
        o.set_target(xts)
        oracle_status = o.solve(oracle.default_params(eps_optimal_relative=1e-4,
                                                       eps_feasible_relative=1e-5,
                                                       iteration_limit=200_000), 1.0)
        assert oracle_status == status and o.total_count == s.total_count
        I = milp.int_idx
        dg = np.abs(sc.D_c[I] * s.pdhg_x[I] - xt[I]).sum()
        do = np.abs(sc.D_c[I] * o.pdhg_x[I] - xt[I]).sum()
        assert dg == pytest.approx(do, rel=1e-9)


# ---- batching ------------------------------------------------------------------------


@pytest.mark.parametrize("path", ["default", "cooperative"])
def test_batch_equals_single_handles(oracle, monkeypatch, path):
    """Each member of a batch takes exactly its single-handle steps; "cooperative"
    forces the one-launch-per-window cooperative path (grid barriers) on both."""
    if path == "cooperative":
        monkeypatch.setenv("PDFP_TINY", "0")
        monkeypatch.setenv("PDFP_MEDIUM", "1")
    milps = [synthetic.covering_p0201_like(s) for s in (1, 2, 3)]
    targets = [np.round(np.random.default_rng(s).random(len(m.c))) for s, m in zip((5, 6, 7), milps)]
    probs, singles = [], []
    for m, xt in zip(milps, targets):
        sc, is_eq, is_int, w = proj_inputs(oracle, m)
        probs.append((sc.A, sc.con_ub, is_eq, is_int, sc.var_lb, sc.var_ub, w))
        x, st, s, _ = gpu_project(oracle, m, xt, 1e-6, "fp64")
        singles.append((sc.D_c, x, st, s.total_count))
    b = gpu.PDFPBatch(probs, precision="fp64")
    for p, xt in enumerate(targets):
        b.set_target(p, xt / singles[p][0])
    st = b.solve(SolverParameters(eps_optimal_relative=1e-6, eps_feasible_relative=1e-6,
                                  iteration_limit=1_000_000), 1.0)
    for p in range(3):
        D_c, x, status, count = singles[p]
        assert st[p] == status and b.results[p]["total_count"] == count
        assert np.abs(D_c * b.get(p, "pdhg_x") - x).max() <= 1e-10


def test_batch_members_terminate_independently(oracle):
    """A tiny and a larger member with different tolerances: each stops on its own test."""
    m1 = synthetic.covering_p0201_like(1)
    m2, _, xt2 = synthetic.general_integer(2, m=3000, n=6000, m_eq=500)
    xt1 = np.round(np.random.default_rng(1).random(len(m1.c)))
    probs, scs = [], []
    for m in (m1, m2):
        sc, is_eq, is_int, w = proj_inputs(oracle, m)
        scs.append(sc)
        probs.append((sc.A, sc.con_ub, is_eq, is_int, sc.var_lb, sc.var_ub, w))
    b = gpu.PDFPBatch(probs, precision="mixed")
    b.set_target(0, xt1 / scs[0].D_c)
    b.set_target(1, xt2 / scs[1].D_c)
    params = [SolverParameters(eps_optimal_relative=1e-2, eps_feasible_relative=1e-3),
              SolverParameters(eps_optimal_relative=1e-4, eps_feasible_relative=1e-5)]
    st = b.solve(params, [1.0, 1.0])
    assert st == ["OPTIMAL", "OPTIMAL"]
    assert b.results[0]["total_count"] < b.results[1]["total_count"]
    assert b.results[0]["rel_gap"] <= 1e-2 and b.results[1]["rel_gap"] <= 1e-4


# ---- limits, warm starts and errors ------------------------------------------------------


def test_iteration_limit_zero_and_time_limit(oracle, examples):
    m = examples["p0201"]
    xt = np.round(np.random.default_rng(3).random(len(m.c)))
    x, status, s, _ = gpu_project(oracle, m, xt, 1e-12, "fp64", iteration_limit=0)
    assert status == "ITERATION_LIMIT" and s.total_count == 0
    x, status, s, _ = gpu_project(oracle, m, xt, 1e-12, "fp64", iteration_limit=400)
    assert status == "ITERATION_LIMIT" and s.total_count == 400
    sc, is_eq, is_int, w = proj_inputs(oracle, m)
    s = gpu.PDFPState(sc.A, sc.con_ub, is_eq, is_int, sc.var_lb, sc.var_ub, w)
    s.set_target(xt / sc.D_c)
    status = s.solve(SolverParameters(eps_optimal_relative=1e-14, eps_feasible_relative=1e-14,
                                      time_limit=0.0), 1.0)
    assert status == "TIME_LIMIT" and s.total_count == 200


def test_warm_start_continues_from_current_iterate(oracle, examples):
    m = examples["pk1"]
    xt = np.round(np.random.default_rng(4).random(len(m.c)))
    sc, is_eq, is_int, w = proj_inputs(oracle, m)
    p = SolverParameters(eps_optimal_relative=1e-6, eps_feasible_relative=1e-6)
    s = gpu.PDFPState(sc.A, sc.con_ub, is_eq, is_int, sc.var_lb, sc.var_ub, w)
    s.set_target(xt / sc.D_c)
    s.solve(p, 1.0)
    first = s.total_count
    s.set_target(xt / sc.D_c)  # same target: warm start from the converged iterate
    s.solve(p, 1.0)
    assert s.total_count <= first
    o = oracle.OraclePDFP(sc.A, sc.con_ub, is_eq, is_int, sc.var_lb, sc.var_ub, w)
    o.set_target(xt / sc.D_c)
    o.solve(oracle.default_params(eps_optimal_relative=1e-6, eps_feasible_relative=1e-6), 1.0)
    o.set_target(xt / sc.D_c)
    o.solve(oracle.default_params(eps_optimal_relative=1e-6, eps_feasible_relative=1e-6), 1.0)
    assert o.total_count == s.total_count


def _raw_create(rp, ci, v, m, n, b, is_eq, is_int, lb, ub, w):
    """pdfp_create straight through the C ABI (no host-side clean-up of the CSR)."""
    import ctypes as C
    from pdfp_b200 import _lib as L
    arrs = [np.asarray(rp, np.int32), np.asarray(ci, np.int32), np.asarray(v, np.float64)]
    csr = L.Csr(m, n, L.iptr(arrs[0]), L.iptr(arrs[1]), L.dptr(arrs[2]))
    vecs = [L.f64(b), np.asarray(is_eq, np.uint8), np.asarray(is_int, np.uint8), L.f64(lb),
            L.f64(ub), L.f64(w)]
    h = C.c_void_p()
    rc = L.lib().pdfp_create(C.byref(csr), L.dptr(vecs[0]), L.uptr(vecs[1]), L.uptr(vecs[2]),
                             L.dptr(vecs[3]), L.dptr(vecs[4]), L.dptr(vecs[5]), None, 0, C.byref(h))
    if rc == 0:
        L.lib().pdfp_destroy(h)
    return rc


def test_invalid_inputs_are_rejected():
    from pdfp_b200 import _lib as L
    from pdfp_b200._lib import LibraryError
    ok = dict(b=[1.0], is_eq=[0], is_int=[1, 1], lb=[0.0, 0.0], ub=[1.0, 1.0], w=[1.0, 1.0])
    assert _raw_create([0, 2], [0, 1], [1.0, 1.0], 1, 2, **ok) == 0
    assert _raw_create([0, 2], [1, 0], [1.0, 1.0], 1, 2, **ok) == L.E_INVALID   # unsorted row
    assert _raw_create([0, 1], [5], [1.0], 1, 2, **ok) == L.E_INVALID          # column out of range
    assert _raw_create([0, 3], [0, 1], [1.0, 1.0], 1, 2, **ok) == L.E_INVALID  # row_ptr beyond data
    assert _raw_create([1, 2], [0, 1], [1.0, 1.0], 1, 2, **ok) == L.E_INVALID  # row_ptr[0] != 0
    assert _raw_create([0, 2], [0, 1], [1.0, np.inf], 1, 2, **ok) == L.E_INVALID
    bad = dict(ok, b=[np.nan])
    assert _raw_create([0, 2], [0, 1], [1.0, 1.0], 1, 2, **bad) == L.E_INVALID
    A = sp.csr_matrix(np.array([[1.0, 1.0]]))
    s = gpu.PDFPState(A, [1.0], [0], [1, 1], [0.0, 0.0], [1.0, 1.0], [1.0, 1.0])
    with pytest.raises(LibraryError):
        s.set_target([np.nan, 0.0])
    with pytest.raises(LibraryError):
        s.solve(SolverParameters(termination_evaluation_frequency=0), 1.0)
    with pytest.raises(LibraryError):
        s.solve(SolverParameters(), -1.0)


def test_empty_constraint_set(oracle):
    """No rows: the projection is the clamp of the target (step size 1, src/pdfp.jl:222-223)."""
    A = sp.csr_matrix((0, 3))
    s = gpu.PDFPState(A, np.zeros(0), np.zeros(0, bool), np.array([1, 1, 0], bool),
                      np.zeros(3), np.array([1.0, 2.0, 1.0]), np.ones(3))
    s.set_target(np.array([0.5, 3.0, 0.2]))
    st = s.solve(SolverParameters(eps_optimal_relative=1e-8, eps_feasible_relative=1e-8), 1.0)
    assert st == "OPTIMAL"
    x = s.pdhg_x
    assert x[0] == pytest.approx(0.5, abs=1e-6) and x[1] == pytest.approx(2.0, abs=1e-6)


def test_uneven_batch_members_follow_the_oracle(oracle):
    """Config-3 shape at test scale: 12 covering/packing models, n log-uniform in
    [300, 6000], one FP64 batch handle; every member takes the oracle's steps."""
    models = synthetic.covering_packing_batch(seed=5, k=12, n_min=300, n_max=6000)
    probs, targets, scs = [], [], []
    rng = np.random.default_rng(12)
    for m in models:
        sc, is_eq, is_int, w = proj_inputs(oracle, m)
        probs.append((sc.A, sc.con_ub, is_eq, is_int, sc.var_lb, sc.var_ub, w))
        targets.append(np.round(rng.random(len(m.c))))
        scs.append(sc)
    b = gpu.PDFPBatch(probs, precision="fp64")
    for p, xt in enumerate(targets):
        b.set_target(p, xt / scs[p].D_c)
    prm = SolverParameters(eps_optimal_relative=1e-4, eps_feasible_relative=1e-5)
    st = b.solve(prm, 1.0)
    for p, m in enumerate(models):
        sc, is_eq, is_int, w = proj_inputs(oracle, m)
        twin = oracle.OracleSolvers.PDFPState(sc.A, sc.con_ub, is_eq, is_int, sc.var_lb,
                                               sc.var_ub, w)
        twin.set_target(targets[p] / sc.D_c)
        status = twin.solve(prm, 1.0)
        assert st[p] == status and b.results[p]["total_count"] == twin.total_count, p
        assert np.abs(b.get(p, "pdhg_x") - twin.pdhg_x).max() <= 1e-10, p


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_whole_window_kernel_staged_equals_unstaged(oracle, monkeypatch, precision):
    """Small members run whole windows in one launch, with their vectors and matrix
    copied into shared memory for the launch or read in place (PDFP_TINY_STAGE=0): the
    same arithmetic, so bit-identical iterates and the same iteration counts."""
    milps = [synthetic.covering_p0201_like(s) for s in (1, 2)] + [synthetic.markshare_like(3)]
    targets = [np.round(np.random.default_rng(s).random(len(m.c))) for s, m in zip((5, 6, 7), milps)]
    out = {}
    for stage in ("1", "0"):
        monkeypatch.setenv("PDFP_TINY_STAGE", stage)
        probs, dcs = [], []
        for m in milps:
            sc, is_eq, is_int, w = proj_inputs(oracle, m)
            probs.append((sc.A, sc.con_ub, is_eq, is_int, sc.var_lb, sc.var_ub, w))
            dcs.append(sc.D_c)
        b = gpu.PDFPBatch(probs, precision=precision)
        for p, xt in enumerate(targets):
            b.set_target(p, xt / dcs[p])
        b.solve(SolverParameters(eps_optimal_relative=1e-6, eps_feasible_relative=1e-6,
                                 iteration_limit=100_000), 1.0)
        single = gpu.PDFPState(*probs[0], precision=precision)
        single.set_target(targets[0] / dcs[0])
        single.solve(SolverParameters(eps_optimal_relative=1e-6, eps_feasible_relative=1e-6), 1.0)
        out[stage] = ([r["total_count"] for r in b.results], [b.get(p, "pdhg_x") for p in range(3)],
                      single.total_count, single.pdhg_x)
    (c1, x1, s1, y1), (c0, x0, s0, y0) = out["1"], out["0"]
    assert c1 == c0 and s1 == s0
    for a, bb in zip(x1, x0):
        assert np.array_equal(a, bb)
    assert np.array_equal(y1, y0)
