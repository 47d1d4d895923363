"""pdfp_solve_batch_any: a batched solve that returns once any running member stops.

A member that is still running when the call returns stops at an evaluation-window
boundary with its whole state on the device; resumed by later calls, it takes
exactly the steps of one uninterrupted solve.  Checked on two members of one
batch, the first with a loose tolerance (it stops first), the second with a
tight one (left running, then resumed call after call): each member's status,
PDHG count and pdhg_x equal those of an uninterrupted pdfp_solve_batch, bit for
bit.  Small members run the one-launch window kernel (which leaves at a window
boundary once another member has stopped), the zipf member the captured window
graph; the mixed cases include the FP64 polish.
"""
import numpy as np
import pytest

from pdfp_b200 import gpu, synthetic
from pdfp_b200.params import SolverParameters

pytestmark = pytest.mark.gpu

LOOSE = SolverParameters(eps_optimal_relative=1e-2, eps_feasible_relative=1e-2)
TIGHT = SolverParameters(eps_optimal_relative=1e-7, eps_feasible_relative=1e-7)
IDLE = SolverParameters(iteration_limit=0)


def model(examples, name):
    if name == "zipf-4k":
        milp, _ = synthetic.zipf_lp(seed=3, m=4000, n=20000, nnz=300_000)
        return milp
    return examples[name]


def make_batch(oracle, milp, precision):
    sc, is_eq, is_int, w = oracle.projector_inputs(milp)
    b = gpu.PDFPBatch([(sc.A, sc.con_ub, is_eq, is_int, sc.var_lb, sc.var_ub, w)] * 2,
                      precision=precision)
    rng = np.random.default_rng(7)
    xts = []
    for p in range(2):
        xt = np.zeros(len(milp.c))
        I = milp.int_idx
        xt[I] = np.round(rng.random(len(I)) * (np.minimum(milp.u[I], 2) - milp.l[I]) + milp.l[I])
        b.set_target(p, xt / sc.D_c)
        xts.append(xt)
    return b


@pytest.mark.parametrize("name,precision", [("p0201", "fp64"), ("pk1", "fp64"),
                                            ("gen-ip054", "mixed"), ("zipf-4k", "fp64"),
                                            ("zipf-4k", "mixed")])
def test_resumed_member_takes_the_uninterrupted_steps(oracle, examples, name, precision,
                                                     monkeypatch):
    # the same step kernels in both handles: the autotuner times its candidates, so two
    # tuned handles may pick differently chunked tilings (long rows summed otherwise)
    monkeypatch.setenv("PDFP_AUTOTUNE", "0")
    milp = model(examples, name)
    ref = make_batch(oracle, milp, precision)
    ref_status = ref.solve([LOOSE, TIGHT], 1.0)
    ref_res = [dict(r) for r in ref.results]
    ref_x = [ref.get(p, "pdhg_x").copy() for p in range(2)]

    b = make_batch(oracle, milp, precision)
    st = b.solve_any([LOOSE, TIGHT], 1.0)
    assert st[0] == ref_status[0] and st[1] == "RUNNING"
    assert b.results[0]["total_count"] == ref_res[0]["total_count"]
    assert np.array_equal(b.get(0, "pdhg_x"), ref_x[0])
    calls = 1
    while st[1] == "RUNNING":
        st = b.solve_any([IDLE, TIGHT], 1.0, resume=[False, True])
        calls += 1
        assert calls < 10_000
    assert calls >= 2
    assert st[1] == ref_status[1]
    assert b.results[1]["total_count"] == ref_res[1]["total_count"]
    assert b.results[1]["restarts"] == ref_res[1]["restarts"]
    assert np.array_equal(b.get(1, "pdhg_x"), ref_x[1])


def test_resume_needs_a_running_member(oracle, examples):
    b = make_batch(oracle, examples["p0201"], "fp64")
    with pytest.raises(Exception, match="cannot resume"):
        b.solve_any([LOOSE, TIGHT], 1.0, resume=[False, True])
    st = b.solve_any([LOOSE, TIGHT], 1.0)
    assert st[1] == "RUNNING"
    with pytest.raises(Exception, match="cannot resume"):  # member 0 has stopped
        b.solve_any([LOOSE, TIGHT], 1.0, resume=[True, True])
    b.warm_start(1)  # a new projection for member 1: it can no longer resume
    with pytest.raises(Exception, match="cannot resume"):
        b.solve_any([IDLE, TIGHT], 1.0, resume=[False, True])
