"""The CPU oracle pinned against the reference's own known answers.

Pins (the reference's tests and published log, read as text):
* test/runtests.jl:41-47  toy projection: OPTIMAL, l1 distance 1, x1 + x2 <= 1
* test/runtests.jl:49-54  general integer with a continuous partner: x1 = 2
* test/runtests.jl:30-38  MPS reader: p0201 sizes and types, pk1 has 31 continuous columns
* test/runtests.jl:73-79  the pump finds a feasible point on the four examples
* README.md:36-48         the p0201 log: root LP OPTIMAL after 600 iterations at 1e-2; the
                          first rounding violates by 9; pump iteration 1 has distance
                          8.08613, violation 1 and 600 PDHG iterations at gap 1e-2
"""
import json
import os

import numpy as np
import pytest
import scipy.sparse as sp

from conftest import GOLDEN, REF_EXAMPLES
from pdfp_b200.milp import MILP, is_feasible, num_continuous


def test_toy_projection_distance_one(oracle):
    m = MILP([0.0, 0.0], 0.0, sp.csr_matrix(np.array([[1.0, 1.0]])), [1.0], ["le"], [0.0, 0.0],
             [1.0, 1.0], [0, 1])
    x, status, _ = oracle.project(m, [1.0, 1.0])
    assert status == "OPTIMAL"
    assert abs(np.abs(x - 1.0).sum() - 1.0) <= 1e-5
    assert x.sum() <= 1.0 + 1e-6


def test_general_integer_projection(oracle):
    m = MILP([0.0, 0.0], 0.0, sp.csr_matrix(np.array([[1.0, 1.0]])), [2.0], ["eq"], [0.0, 0.0],
             [5.0, np.inf], [0])
    x, status, _ = oracle.project(m, [3.0, 0.0])
    assert status == "OPTIMAL"
    assert abs(x[0] - 2.0) <= 1e-5


def test_mps_reader_sizes(examples):
    m = examples["p0201"]
    assert len(m.c) == 201 and len(m.int_idx) == 201
    assert np.all(m.l[m.int_idx] == 0) and np.all(m.u[m.int_idx] == 1)
    assert set(m.row_sense) <= {"le", "eq"}
    assert num_continuous(examples["pk1"]) == 31


@pytest.mark.skipif(not (REF_EXAMPLES and os.path.isdir(REF_EXAMPLES)),
                    reason="no reference checkout (PDFP_REFERENCE_DIR)")
def test_mps_reader_matches_fixtures():
    from pdfp_b200.milp import read_mps
    from conftest import load_example
    for name in ["p0201", "pk1"]:
        a = read_mps(os.path.join(REF_EXAMPLES, f"{name}.mps.gz"))
        b = load_example(name)
        assert (a.A != b.A).nnz == 0 and np.array_equal(a.b, b.b) and np.array_equal(a.int_idx, b.int_idx)


def test_readme_root_lp_and_first_pump_iteration(oracle, examples, capsys):
    """The p0201 log printed by the reference (README.md:36-48)."""
    log = json.load(open(os.path.join(GOLDEN, "reference_log.json")))["p0201"]
    m = examples["p0201"]
    x, ds, status, iters, _ = oracle.solve_lp_relaxation(m, 1e-2, 60.0, False)
    assert status == log["root_lp"]["status"] and iters == log["root_lp"]["iterations"]
    from pdfp_b200.pump import feasibility_pump
    feasibility_pump(m, solvers=oracle.OracleSolvers(), verbose=True, time_limit=60.0)
    out = capsys.readouterr().out.splitlines()
    assert any(l.startswith("root LP     OPTIMAL after 600 iterations") for l in out)
    assert any(f"first rounding violates by {log['first_rounding_violation']})" in l for l in out)
    first = [l for l in out if l.strip().startswith("1 ")][0].split()
    it1 = log["iterations"][0]
    assert float(first[1]) == pytest.approx(it1["distance"], rel=1e-5)
    assert int(first[2]) == it1["violation"] and int(first[3]) == it1["pdhg"]
    assert first[5] == it1["action"]


@pytest.mark.parametrize("name", ["p0201", "gen-ip054", "pk1", "markshare2"])
def test_pump_finds_feasible_on_examples(oracle, examples, name):
    from pdfp_b200.pump import feasibility_pump
    m = examples[name]
    r = feasibility_pump(m, solvers=oracle.OracleSolvers(), time_limit=120.0)
    assert r.found
    assert is_feasible(m, r.x)
    assert r.objective == pytest.approx(float(np.dot(m.c, r.x) + m.c0))


def test_scaling_is_ruiz_then_pock_chambolle(oracle, examples):
    """Structural checks of scale_problem (src/preconditioner.jl:26-99)."""
    m = examples["pk1"]
    n = len(m.c)
    con_lb = np.where(m.is_eq, m.b, -np.inf)
    s = oracle.scale_problem(m.A, m.c, m.l, m.u, con_lb, m.b)
    # A_scaled = D_r A D_c exactly as products of the factors
    As = sp.diags(s.D_r) @ m.A @ sp.diags(s.D_c)
    assert np.allclose(As.toarray(), s.A.toarray(), rtol=1e-14, atol=0)
    # Pock-Chambolle with alpha = 1 bounds the spectral norm of the scaled matrix by 1
    assert np.linalg.norm(s.A.toarray(), 2) <= 1.0 + 1e-12
    assert 0 < s.bound_scale <= 1 and 0 < s.objective_scale <= 1
    assert np.allclose(s.c, m.c * s.D_c * s.objective_scale)


def test_power_iteration_matches_dense_norm(oracle, examples):
    sc, *_ = oracle.projector_inputs(examples["p0201"])
    s, it = oracle.estimate_max_singular_value(sc.A)
    assert s == pytest.approx(np.linalg.norm(sc.A.toarray(), 2), rel=1e-4)
    assert 0 < it < 5000


def test_oracle_thread_count_does_not_change_results(oracle, examples):
    m = examples["pk1"]
    xt = np.round(np.random.default_rng(4).random(len(m.c)))
    oracle.set_threads(1)
    a, _, _ = oracle.project(m, xt, tol=1e-6)
    oracle.set_threads(4)
    b, _, _ = oracle.project(m, xt, tol=1e-6)
    oracle.set_threads(1)
    assert np.array_equal(a, b)
