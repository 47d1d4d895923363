"""GPU root LP (pdlp_solve_relaxation) against the oracle's solve_lp_relaxation.

FP64: the same termination reason and iteration count as the oracle, the same
objective to 1e-9 relative and primal points within 1e-8 (only reduction orders
differ).  Mixed: OPTIMAL with the objective within the solve's tolerance.
cuPDLPx termination (models with continuous columns) uses residuals in original
units and detects infeasibility (src/pdlp.jl:247-290): tested on small infeasible
and unbounded LPs against the oracle.
"""
import numpy as np
import pytest
import scipy.sparse as sp

from pdfp_b200 import gpu, synthetic
from pdfp_b200.milp import MILP, num_continuous

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["p0201", "pk1", "gen-ip054", "markshare2"])
def test_root_lp_matches_oracle(oracle, examples, name):
    m = examples[name]
    cup = num_continuous(m) > 0
    xo, dso, so, io, ro = oracle.solve_lp_relaxation(m, 1e-2, 60.0, cup)
    xg, dsg, sg, ig, rg = gpu.solve_lp_relaxation(m, 1e-2, 60.0, cup, return_result=True)
    assert sg == so == "OPTIMAL"
    assert ig == io
    assert rg["objective_value"] == pytest.approx(ro["objective_value"], rel=1e-9, abs=1e-12)
    assert np.abs(xg - xo).max() <= 1e-8 * max(1.0, np.abs(xo).max())
    assert np.array_equal(np.sign(np.round(dsg, 12)), np.sign(np.round(dso, 12)))


def test_p0201_root_lp_is_the_published_600_iterations(examples):
    x, ds, status, iters = gpu.solve_lp_relaxation(examples["p0201"], 1e-2, 60.0, False)
    assert status == "OPTIMAL" and iters == 600  # README.md:39


@pytest.mark.parametrize("name", ["p0201", "pk1"])
def test_root_lp_mixed_precision(oracle, examples, name):
    m = examples[name]
    cup = num_continuous(m) > 0
    xo, _, so, _, ro = oracle.solve_lp_relaxation(m, 1e-4, 60.0, cup)
    xg, _, sg, ig, rg = gpu.solve_lp_relaxation(m, 1e-4, 60.0, cup, precision="mixed",
                                               return_result=True)
    assert sg == "OPTIMAL"
    assert rg["rel_gap"] <= 1e-4 and rg["rel_primal"] <= 1e-4 and rg["rel_dual"] <= 1e-4
    assert rg["objective_value"] == pytest.approx(ro["objective_value"], rel=1e-3, abs=1e-6)


def _lp(A, b, c, l, u, sense):
    return MILP(np.asarray(c, float), 0.0, sp.csr_matrix(np.asarray(A, float)), b, sense, l, u, [])


@pytest.mark.parametrize("case", ["infeasible", "unbounded"])
def test_cupdlpx_infeasibility_detection(oracle, case):
    if case == "infeasible":   # x1 + x2 <= -1, x >= 0
        m = _lp([[1.0, 1.0]], [-1.0], [1.0, 1.0], [0.0, 0.0], [np.inf, np.inf], ["le"])
    else:                      # min -x1 s.t. x1 - x2 <= 0, x >= 0 (unbounded)
        m = _lp([[1.0, -1.0]], [0.0], [-1.0, 0.0], [0.0, 0.0], [np.inf, np.inf], ["le"])
    _, _, so, io, _ = oracle.solve_lp_relaxation(m, 1e-4, 30.0, True)
    _, _, sg, ig = gpu.solve_lp_relaxation(m, 1e-4, 30.0, True)
    assert sg == so
    assert ig == io
    assert sg in ("PRIMAL_INFEASIBLE", "DUAL_INFEASIBLE", "ITERATION_LIMIT", "TIME_LIMIT", "OPTIMAL")


def test_config1_root_lp(oracle):
    from pdfp_b200 import synthetic
    milp, _, _ = synthetic.general_integer(1, m=2000, n=5000, m_eq=500)
    xo, _, so, io, ro = oracle.solve_lp_relaxation(milp, 1e-3, 120.0, True)
    xg, _, sg, ig, rg = gpu.solve_lp_relaxation(milp, 1e-3, 120.0, True, return_result=True)
    assert sg == so and ig == io
    assert rg["objective_value"] == pytest.approx(ro["objective_value"], rel=1e-8)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_small_lp_staged_equals_unstaged(monkeypatch, precision):
    """A small LP runs whole windows in one launch, its data copied into shared memory or
    read in place (PDFP_TINY_STAGE=0): bit-identical solutions and iteration counts, with
    (markshare-shaped, continuous slacks) and without (p0201-shaped) the cuPDLPx ray passes."""
    for milp, cupdlpx in [(synthetic.covering_p0201_like(2), False), (synthetic.markshare_like(3), True)]:
        out = {}
        for stage in ("1", "0"):
            monkeypatch.setenv("PDFP_TINY_STAGE", stage)
            x, ds, status, iters = gpu.solve_lp_relaxation(milp, tolerance=1e-4,
                                                           cupdlpx_termination=cupdlpx,
                                                           precision=precision)
            out[stage] = (x, ds, status, iters)
        assert out["1"][2] == out["0"][2] and out["1"][3] == out["0"][3]
        assert np.array_equal(out["1"][0], out["0"][0]) and np.array_equal(out["1"][1], out["0"][1])
