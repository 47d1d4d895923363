"""The library's bounded device waits give up, report PDFP_E_TIMEOUT and leave the
GPU usable (pdfp_selftest_bounded_wait).

Every spin of the library's kernels -- the tile engine's mbarrier waits and the
cooperative window's grid barrier -- gives up after a limit.  No correct solve
reaches it, so the self-test runs the same wait code in a kernel whose wait
cannot complete (an mbarrier phase one arrival short, a grid barrier expecting
one block more than launched) with a 50 ms limit: nothing faults or traps, the
wait just ends.  Afterwards a handle created before the timeout and a new one
both solve.  (The reference's loop ends only on its own time and iteration
limits, src/pdfp.jl:279-282.)
"""
import time

import numpy as np
import pytest

from pdfp_b200 import _lib as L
from pdfp_b200 import gpu, synthetic
from pdfp_b200.params import SolverParameters

pytestmark = pytest.mark.gpu


def _handle(oracle, seed):
    milp = synthetic.covering_p0201_like(seed)
    sc, is_eq, is_int, w = oracle.projector_inputs(milp)
    s = gpu.PDFPState(sc.A, sc.con_ub, is_eq, is_int, sc.var_lb, sc.var_ub, w, precision="fp64")
    xt = np.round(np.random.default_rng(seed).random(len(milp.c)))
    return s, xt / sc.D_c


@pytest.mark.parametrize("which", [0, 1])
def test_bounded_wait_gives_up_and_the_gpu_stays_usable(oracle, which):
    before, xt_b = _handle(oracle, 1)
    t = time.perf_counter()
    rc = gpu.selftest_bounded_wait(which, 0.05)
    dt = time.perf_counter() - t
    assert rc == L.E_TIMEOUT
    assert b"bounded device wait gave up" in L.lib().pdfp_last_error()
    assert 0.05 <= dt < 3.0
    p = SolverParameters(eps_optimal_relative=1e-4, eps_feasible_relative=1e-4)
    before.set_target(xt_b)
    assert before.solve(p, 1.0) == "OPTIMAL"
    after, xt_a = _handle(oracle, 2)
    after.set_target(xt_a)
    assert after.solve(p, 1.0) == "OPTIMAL"


def test_selftest_rejects_bad_arguments():
    assert gpu.selftest_bounded_wait(2, 0.05) == L.E_INVALID
    assert gpu.selftest_bounded_wait(0, 0.0) == L.E_INVALID
    assert gpu.selftest_bounded_wait(0, 5.0) == L.E_INVALID
