"""The CPU rounder (src/rounding.jl) on the reference's own rounding tests
(test/runtests.jl:57-70)."""
import numpy as np

from pdfp_b200.rounding import BatchPolicy, Rounder, round_guarded, round_sequential
from pdfp_b200.milp import is_feasible


def test_lp_integral_feasible_point_rounds_to_itself(oracle, examples):
    from pdfp_b200.pump import feasibility_pump
    m = examples["p0201"]
    r = feasibility_pump(m, solvers=oracle.OracleSolvers(), time_limit=60.0)
    assert r.found and is_feasible(m, r.x)
    rng = np.random.Generator(np.random.PCG64(1))
    assert np.array_equal(round_guarded(Rounder(m), r.x, rng, 0), r.x)


def test_guarded_equals_sequential_without_integral_coordinates(examples):
    m = examples["p0201"]
    x = np.full(len(m.c), 0.5) + 0.01 * np.random.default_rng(2).random(len(m.c))
    a = round_guarded(Rounder(m, policy=None), x, np.random.Generator(np.random.PCG64(3)), 20)
    b = round_sequential(Rounder(m, policy=None), x, np.random.Generator(np.random.PCG64(3)), 20)
    assert np.array_equal(a, b)
    assert np.all(a == np.round(a))


def test_batch_policy_tries_batch_until_a_failure():
    P = BatchPolicy()
    assert P.wants_batch()
    P.observe_batch(False, 1.0, 0.0)
    assert P.wants_batch()  # no failure seen yet
    P.observe_batch(True, 2.0, 1.5)
    P.observe_skip(0.1)
    # cheap sequential calls, costly failures: skip the batch
    assert not P.wants_batch() or P.skipped >= P.reprobe
    for _ in range(P.reprobe):
        P.observe_skip(0.1)
    assert P.wants_batch()  # re-probe after `reprobe` skips
