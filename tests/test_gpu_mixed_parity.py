"""The mixed projector's FP32 path -- the one the benchmark times -- against the FP64 oracle.

The mixed form runs the PDHG iterates and sparse products in FP32 and the
evaluation in FP64; under a tolerance tighter than the FP32 floor (1e-6) the
FP64 polish finishes the solve.  These tests run it through the C ABI on three
shapes and compare with the oracle's FP64 PDHG (the reference's CPU path,
src/pdfp.jl:252-288) on the same targets:

* zipf-4k: synthetic.zipf_lp(seed=3, m=4000, n=20000, nnz=300_000) -- Zipf(1.5)
  row lengths whose longest rows span several shared-memory chunks of the tile
  engine, as on the 1M x 2M benchmark matrix;
* zipf-100k: the benchmark's generator at a tenth of its size (100k x 200k,
  2M nonzeros), a cold projection and then the benchmark's step: the next
  target with 5% of the integer targets flipped, warm-started;
* config1: the 20k x 50k general-integer model (500k nonzeros).

Bars (the reference's own GPU-vs-CPU test is test/runtests.jl:81-88, the l1
distance of src/pdfp.jl:210-217):

* tight tolerance (1e-8; 1e-7 on config1): the FP32 phase and the FP64 polish both run;
  the l1 distance is within 1e-6 relative of the oracle's at the same
  tolerance; the KKT residuals re-evaluated in FP64 on the host meet it;
* benchmark tolerance (gap and dual 1e-4, primal 1e-5): the solve stays in FP32;
  the host FP64 KKT residuals meet the tolerance; the l1 distance differs from
  the oracle's by at most twice the gap tolerance's share, 2e-4 (1 + sum_I w|x~|)
  -- the most two solutions within that gap tolerance can differ by.  The
  measured relative difference is printed (pytest -s).
"""
import numpy as np
import pytest

from conftest import host_kkt
from pdfp_b200 import gpu
from pdfp_b200 import synthetic
from pdfp_b200.params import SolverParameters

pytestmark = pytest.mark.gpu

BENCH_TOL = (1e-4, 1e-5)  # eps_optimal_relative, eps_feasible_relative


def flip(xt, milp, rng, frac=0.05):
    """The benchmark's next target: 5% of the integer targets moved by one inside the bounds."""
    I = milp.int_idx
    xt = xt.copy()
    idx = I[rng.choice(len(I), size=max(1, int(frac * len(I))), replace=False)]
    up = np.minimum(xt[idx] + 1, milp.u[idx])
    dn = np.maximum(xt[idx] - 1, milp.l[idx])
    xt[idx] = np.where(up != xt[idx], up, dn)
    return xt


def case(name):
    """(milp, [targets]) in the model's own units."""
    if name == "zipf-4k":
        milp, _ = synthetic.zipf_lp(seed=3, m=4000, n=20000, nnz=300_000)
        rng = np.random.default_rng(3)
        xt = np.zeros(len(milp.c))
        xt[milp.int_idx] = np.round(rng.random(len(milp.int_idx)))
        return milp, [xt]
    if name == "zipf-100k":
        milp, _ = synthetic.zipf_lp(seed=5, m=100_000, n=200_000, nnz=2_000_000)
        rng = np.random.default_rng(5)
        xt = np.zeros(len(milp.c))
        xt[milp.int_idx] = np.round(rng.random(len(milp.int_idx)))
        return milp, [xt, flip(xt, milp, rng)]
    milp, _, xt = synthetic.general_integer(1)
    return milp, [xt]


_ORACLE_RUNS = {}  # the oracle's answers by case and tolerance


def run_both(oracle, milp, targets, eps_opt, eps_feas, polish=None, key=None):
    """Project the targets in sequence (each warm-started from the last) with the mixed
    GPU handle and with the oracle; per projection: (gpu result, gpu host KKT, oracle
    result, oracle host KKT, D).  `key` caches the oracle's side."""
    sc, is_eq, is_int, w = oracle.projector_inputs(milp)
    g = gpu.PDFPState(sc.A, sc.con_ub, is_eq, is_int, sc.var_lb, sc.var_ub, w, precision="mixed")
    if polish is not None:
        g.set_polish(*polish)
    p = SolverParameters(eps_optimal_relative=eps_opt, eps_feasible_relative=eps_feas,
                         iteration_limit=400_000)
    if key is None or key not in _ORACLE_RUNS:
        o = oracle.OraclePDFP(sc.A, sc.con_ub, is_eq, is_int, sc.var_lb, sc.var_ub, w)
        op = oracle.default_params(eps_optimal_relative=eps_opt, eps_feasible_relative=eps_feas,
                                   iteration_limit=400_000)
        ores = []
        for xt in targets:
            xts = xt / sc.D_c
            o.set_target(xts)
            assert o.solve(op, 1.0) == "OPTIMAL"
            ores.append((dict(o.last), host_kkt(sc, is_eq, is_int, w, xts, o.get)))
        if key is not None:
            _ORACLE_RUNS[key] = ores
    else:
        ores = _ORACLE_RUNS[key]
    out = []
    for xt, (olast, okkt) in zip(targets, ores):
        xts = xt / sc.D_c
        g.set_target(xts)
        assert g.solve(p, 1.0) == "OPTIMAL"
        D = 1.0 + np.sum(np.where(is_int, w * np.abs(xts), 0.0))
        out.append((dict(g.last), host_kkt(sc, is_eq, is_int, w, xts, g.get), olast, okkt, D))
    return out



@pytest.mark.parametrize("name,tol", [("zipf-4k", 1e-8), ("zipf-100k", 1e-8), ("config1", 1e-7)])
def test_mixed_tight_matches_oracle(oracle, name, tol):
    milp, targets = case(name)
    for r, (gp, gd, gg, gl1), ro, (op_, od, og, ol1), D in run_both(oracle, milp, targets, tol, tol,
                                                                    key=(name, tol)):
        # both phases ran: FP32 iterations first, then the FP64 polish to the tolerance
        assert r["polished"] == 1
        assert 0 < r["fp64_iterations"] < r["total_count"]
        assert gp <= tol * 1.01 and gd <= tol * 1.01 and gg <= tol * 1.01
        assert op_ <= tol * 1.01 and od <= tol * 1.01 and og <= tol * 1.01
        # the device's FP64 distance is the host's
        assert r["objective_value"] == pytest.approx(gl1, rel=1e-9)
        rel = abs(gl1 - ol1) / ol1
        print(f"\n[{name} tol {tol:g}] l1 gpu {gl1:.10g} oracle {ol1:.10g} rel {rel:.3e}; "
              f"iterations {r['total_count']} ({r['fp64_iterations']} FP64) vs oracle "
              f"{ro['total_count']}")
        assert rel <= 1e-6


@pytest.mark.parametrize("name", ["zipf-4k", "zipf-100k", "config1"])
def test_mixed_at_bench_tolerance_stays_fp32(oracle, name):
    eps_opt, eps_feas = BENCH_TOL
    milp, targets = case(name)
    for r, (gp, gd, gg, gl1), ro, (_, _, _, ol1), D in run_both(oracle, milp, targets, eps_opt,
                                                                eps_feas, key=(name, "bench")):
        assert r["polished"] == 0 and r["fp64_iterations"] == 0
        assert r["precision"] == 1  # PDFP_MIXED at termination
        assert gp <= eps_feas * 1.01 and gd <= eps_opt * 1.01 and gg <= eps_opt * 1.01
        diff = abs(gl1 - ol1)
        print(f"\n[{name} bench tol] l1 gpu {gl1:.10g} oracle {ol1:.10g} rel {diff / ol1:.3e} "
              f"(bound {2 * eps_opt * D / ol1:.3e}); iterations {r['total_count']} vs oracle "
              f"{ro['total_count']}")
        assert diff <= 2.0 * eps_opt * D


def test_forced_polish_after_the_first_window(oracle):
    """An FP32 floor of 0.99 ends the FP32 phase at the first evaluation: exactly one
    window (200 iterations) in FP32, the rest in FP64, the oracle's answer at 1e-8."""
    milp, targets = case("zipf-4k")
    ((r, (gp, gd, gg, gl1), ro, (_, _, _, ol1), D),) = run_both(oracle, milp, targets, 1e-8, 1e-8,
                                                                polish=(10, 0.99))
    assert r["polished"] == 1
    assert r["total_count"] - r["fp64_iterations"] == 200
    assert gp <= 1.01e-8 and gd <= 1.01e-8 and gg <= 1.01e-8
    assert abs(gl1 - ol1) <= 1e-6 * ol1


def test_polish_on_stall(oracle):
    """With no FP32 floor to reach (1e-12), the polish takes over when the FP32 phase
    stalls (one evaluation without a 10% KKT improvement)."""
    milp, targets = case("zipf-4k")
    ((r, (gp, gd, gg, gl1), ro, (_, _, _, ol1), D),) = run_both(oracle, milp, targets, 1e-8, 1e-8,
                                                                polish=(1, 1e-12))
    assert r["polished"] == 1 and 0 < r["fp64_iterations"] < r["total_count"]
    assert gp <= 1.01e-8 and gd <= 1.01e-8 and gg <= 1.01e-8
    assert abs(gl1 - ol1) <= 1e-6 * ol1


def test_polish_off_runs_tight_tolerances_in_fp64(oracle):
    milp, targets = case("zipf-4k")
    ((r, (gp, gd, gg, gl1), ro, (_, _, _, ol1), D),) = run_both(oracle, milp, targets, 1e-8, 1e-8,
                                                                polish=(0, 1e-6))
    assert r["polished"] == 0 and r["fp64_iterations"] == r["total_count"]
    assert r["precision"] == 0
    assert abs(gl1 - ol1) <= 1e-6 * ol1


def test_set_polish_rejects_bad_arguments():
    milp, _ = synthetic.zipf_lp(seed=3, m=400, n=2000, nnz=10_000)
    from oracle import oracle as O
    sc, is_eq, is_int, w = O.projector_inputs(milp)
    g = gpu.PDFPState(sc.A, sc.con_ub, is_eq, is_int, sc.var_lb, sc.var_ub, w, precision="mixed")
    from pdfp_b200 import _lib as L
    assert L.lib().pdfp_set_polish(g._h, -1, 1e-6) == L.E_INVALID
    assert L.lib().pdfp_set_polish(g._h, 10, 0.0) == L.E_INVALID
    assert L.lib().pdfp_set_polish(g._h, 10, 1.0) == L.E_INVALID
    assert L.lib().pdfp_set_polish(None, 10, 1e-6) == L.E_INVALID


@pytest.mark.parametrize("name", ["zipf-4k", "zipf-100k"])
def test_vec_engine_matches_oracle(oracle, name, monkeypatch):
    """The same bars with the FP32 steps on the vec engine (vec_spmv.cuh): tight
    tolerance through the FP64 polish, and the benchmark tolerance in FP32."""
    monkeypatch.setenv("PDFP_STEP_ENGINE", "vec")
    test_mixed_tight_matches_oracle(oracle, name, 1e-8)
    test_mixed_at_bench_tolerance_stays_fp32(oracle, name)


@pytest.mark.parametrize("name,seg", [("zipf-4k", "64,256"), ("zipf-100k", "148,512")])
def test_segmented_long_rows_match_oracle(oracle, name, seg, monkeypatch):
    """The same bars with the A side's long rows by column segment (seg_spmv.cuh)."""
    monkeypatch.setenv("PDFP_STEP_ENGINE", "tile")
    monkeypatch.setenv("PDFP_SEG", seg)
    test_mixed_tight_matches_oracle(oracle, name, 1e-8)
    test_mixed_at_bench_tolerance_stays_fp32(oracle, name)
