"""Batched pump driver: trajectories as members of one projector batch.

CPU tests run the driver on the oracle's solvers; the GPU tests run it on the
library and compare trajectory by trajectory with the oracle run.  Step-by-step
comparisons use batch_policy="always": the "cost" policy decides from measured
wall-clock costs (src/rounding.jl:22-63), so two runs may round differently.
"""
import numpy as np
import pytest

from pdfp_b200 import is_feasible, synthetic
from pdfp_b200.pump import feasibility_pump, feasibility_pump_batched

EXAMPLES = ["p0201", "pk1", "gen-ip054", "markshare2"]


@pytest.mark.parametrize("name,seed", [("p0201", 101), ("pk1", 201), ("markshare2", 7)])
def test_one_trajectory_equals_single_pump(examples, oracle, name, seed):
    """K = 1: the batched driver takes exactly the single pump's steps."""
    m = examples[name]
    single = feasibility_pump(m, solvers=oracle.OracleSolvers(), time_limit=120, seed=seed,
                              batch_policy="always")
    res, trajs = feasibility_pump_batched(m, solvers=oracle.OracleSolvers(), time_limit=120,
                                          seeds=(seed,), batch_policy="always")
    assert res.found == single.found
    assert res.iterations == single.iterations
    assert res.pdhg_iterations == single.pdhg_iterations
    assert res.perturbations == single.perturbations
    assert np.array_equal(res.x, single.x)
    assert trajs[0].found == single.found


def test_first_trajectory_to_succeed_wins(examples, oracle):
    """Two seeds in lockstep: the winner is the one the single pumps find first."""
    m = examples["p0201"]
    singles = {s: feasibility_pump(m, solvers=oracle.OracleSolvers(), time_limit=120, seed=s,
                                   batch_policy="always")
               for s in (101, 201)}
    res, trajs = feasibility_pump_batched(m, solvers=oracle.OracleSolvers(), time_limit=120,
                                          seeds=(101, 201), batch_policy="always")
    assert res.found and is_feasible(m, res.x)
    first = min(singles.values(), key=lambda r: r.iterations).iterations
    assert res.iterations == first
    winners = [t for t in trajs if t.found]
    assert len(winners) == 1
    assert singles[winners[0].seed].iterations == first
    assert all(t.iterations == first for t in trajs)


def test_batched_markshare_like(oracle):
    m = synthetic.markshare_like(5)
    res, trajs = feasibility_pump_batched(m, solvers=oracle.OracleSolvers(), time_limit=60,
                                          seeds=(101, 201))
    assert res.found and is_feasible(m, res.x)
    assert len(trajs) == 2 and [t.seed for t in trajs] == [101, 201]


def test_batched_rejects_bad_arguments(examples, oracle):
    with pytest.raises(ValueError):
        feasibility_pump_batched(examples["p0201"], solvers=oracle.OracleSolvers(), seeds=())
    with pytest.raises(ValueError):
        feasibility_pump_batched(examples["p0201"], solvers=oracle.OracleSolvers(),
                                 batch_policy="sometimes")


@pytest.mark.gpu
@pytest.mark.parametrize("name", EXAMPLES)
def test_gpu_batched_pump_matches_single_gpu_pumps(examples, name):
    """FP64 batch on the GPU: the two trajectories take the steps of the two
    single-trajectory GPU pumps with the same seeds, and the first to succeed wins."""
    m = examples[name]
    singles = {s: feasibility_pump(m, time_limit=120, seed=s, precision="fp64",
                                   batch_policy="always") for s in (101, 201)}
    res, trajs = feasibility_pump_batched(m, time_limit=120, seeds=(101, 201), precision="fp64",
                                          batch_policy="always")
    assert res.found and is_feasible(m, res.x)
    first = min(r.iterations for r in singles.values() if r.found)
    assert res.iterations == first
    assert all(t.iterations == first for t in trajs)
    for t in trajs:
        if t.found:
            assert singles[t.seed].iterations == first
            assert np.array_equal(res.x, singles[t.seed].x)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["pk1", "gen-ip054"])
def test_gpu_batched_pump_matches_oracle(examples, oracle, name):
    """Against the oracle's solvers, trajectory by trajectory, on models without
    symmetric columns (see test_gpu_pump for why p0201 is left out)."""
    m = examples[name]
    res_o, tr_o = feasibility_pump_batched(m, solvers=oracle.OracleSolvers(), time_limit=120,
                                           seeds=(101, 201), batch_policy="always")
    res_g, tr_g = feasibility_pump_batched(m, time_limit=120, seeds=(101, 201), precision="fp64",
                                           batch_policy="always")
    assert res_g.found and is_feasible(m, res_g.x)
    assert [(t.seed, t.found, t.iterations, t.perturbations) for t in tr_g] == \
        [(t.seed, t.found, t.iterations, t.perturbations) for t in tr_o]
    I = m.int_idx
    assert np.array_equal(res_g.x[I], res_o.x[I])
    assert np.allclose(res_g.x, res_o.x, rtol=1e-9, atol=1e-9)


@pytest.mark.gpu
@pytest.mark.parametrize("name", EXAMPLES)
def test_gpu_batched_pump_mixed_finds_feasible(examples, name):
    m = examples[name]
    res, trajs = feasibility_pump_batched(m, time_limit=120, seeds=(101, 201), precision="mixed")
    assert res.found and is_feasible(m, res.x)
    assert sum(t.found for t in trajs) == 1


@pytest.mark.parametrize("name", ["p0201", "pk1", "markshare2"])
def test_asynchronous_equals_lockstep_on_oracle(examples, oracle, name):
    """The asynchronous driver with the oracle's solvers (every member's projection
    ends within each call): the same trajectories, step for step, as lockstep."""
    m = examples[name]
    kw = dict(solvers=oracle.OracleSolvers(), time_limit=120, seeds=(101, 201),
              batch_policy="always")
    res_l, tr_l = feasibility_pump_batched(m, **kw)
    res_a, tr_a = feasibility_pump_batched(m, asynchronous=True, **kw)
    assert res_a.found == res_l.found
    assert (res_a.iterations, res_a.pdhg_iterations, res_a.perturbations) == \
        (res_l.iterations, res_l.pdhg_iterations, res_l.perturbations)
    assert np.array_equal(res_a.x, res_l.x)
    assert [(t.seed, t.found) for t in tr_a] == [(t.seed, t.found) for t in tr_l]


@pytest.mark.gpu
@pytest.mark.parametrize("name", EXAMPLES)
def test_gpu_asynchronous_pump_trajectories_match_single_pumps(examples, name):
    """FP64 batch on the GPU, asynchronous: each trajectory advances at its own pace
    and takes exactly the steps of the single-trajectory pump with its seed; the
    winner's result is that pump's result."""
    m = examples[name]
    singles = {s: feasibility_pump(m, time_limit=120, seed=s, precision="fp64",
                                   batch_policy="always") for s in (101, 201)}
    res, trajs = feasibility_pump_batched(m, time_limit=120, seeds=(101, 201), precision="fp64",
                                          batch_policy="always", asynchronous=True)
    assert res.found and is_feasible(m, res.x)
    winners = [t for t in trajs if t.found]
    assert len(winners) == 1
    w = singles[winners[0].seed]
    assert w.found
    assert (res.iterations, res.pdhg_iterations, res.perturbations) == \
        (w.iterations, w.pdhg_iterations, w.perturbations)
    assert np.array_equal(res.x, w.x)
    for t in trajs:  # the others stopped somewhere along their own single pump's path
        assert t.iterations <= singles[t.seed].iterations or not singles[t.seed].found


@pytest.mark.gpu
@pytest.mark.parametrize("name", EXAMPLES)
def test_gpu_asynchronous_pump_mixed_finds_feasible(examples, name):
    m = examples[name]
    res, trajs = feasibility_pump_batched(m, time_limit=120, seeds=(101, 201), precision="mixed",
                                          asynchronous=True)
    assert res.found and is_feasible(m, res.x)
    assert sum(t.found for t in trajs) == 1
