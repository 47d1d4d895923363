"""The device constraint check (pdfp_checker_*): max_violation (src/milp.jl:102-114)
on the GPU equals the host evaluation bit for bit."""
import ctypes as C

import numpy as np
import pytest
import scipy.sparse as sp

from pdfp_b200 import _lib as L
from pdfp_b200 import gpu, synthetic
from pdfp_b200.milp import MILP, max_violation


def test_checker_rejects_null_arguments():
    h = C.c_void_p()
    assert L.lib().pdfp_checker_create(None, None, None, C.byref(h)) == L.E_INVALID
    assert L.lib().pdfp_checker_max_violation(None, None, None) == L.E_INVALID


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["p0201", "pk1", "gen-ip054", "markshare2"])
def test_checker_equals_host_on_examples(examples, name):
    m = examples[name]
    ck = gpu.ConstraintChecker(m)
    rng = np.random.default_rng(3)
    n = len(m.c)
    for trial in range(6):
        if trial % 2:
            x = np.round(rng.random(n) * np.minimum(m.u - m.l, 5) + m.l)
        else:
            x = rng.normal(size=n) * 10.0 ** rng.integers(-3, 4)
        assert ck.max_violation(x) == max_violation(m, x)


@pytest.mark.gpu
def test_checker_equals_host_large_with_empty_rows():
    milp, _, _ = synthetic.general_integer(4, m=20000, n=50000, m_eq=5000)
    A = milp.A.tolil()
    A[17, :] = 0.0  # an empty row
    A = sp.csr_matrix(A)
    A.eliminate_zeros()
    m2 = MILP(milp.c, milp.c0, A, milp.b, milp.row_sense, milp.l, milp.u, milp.int_idx)
    ck = gpu.ConstraintChecker(m2)
    rng = np.random.default_rng(9)
    for _ in range(3):
        x = rng.random(A.shape[1]) * 10
        assert ck.max_violation(x) == max_violation(m2, x)
    with pytest.raises(ValueError):
        ck.max_violation(np.zeros(3))


@pytest.mark.gpu
def test_pump_with_device_check_takes_the_same_steps(examples, monkeypatch):
    """The pump's decisions do not depend on where max_violation runs."""
    import pdfp_b200.pump as P
    m = examples["pk1"]
    runs = []
    for threshold in (1 << 40, 0):  # host check, then device check
        monkeypatch.setattr(P, "DEVICE_CHECK_MIN_NNZ", threshold)
        r = P.feasibility_pump(m, time_limit=120.0, precision="fp64", seed=5, batch_policy="always")
        runs.append(r)
    a, b = runs
    assert (a.found, a.iterations, a.perturbations, a.pdhg_iterations) == \
        (b.found, b.iterations, b.perturbations, b.pdhg_iterations)
    assert np.array_equal(a.x, b.x)
