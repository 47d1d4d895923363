"""Instances and trajectories over several ranks (gloo, world size 2, on the CPU).

The ranks use the oracle's solvers so the host-side logic -- the
longest-processing-time deal, the host gather, the per-iteration stop flag --
runs without a GPU; the GPU library plugs into the same ``solvers`` seam.
"""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

from pdfp_b200.shard import lpt_partition

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_lpt_partition_balances_and_covers():
    costs = [50, 10, 40, 30, 30, 20, 5, 5]
    parts = lpt_partition(costs, 3)
    assert sorted(i for p in parts for i in p) == list(range(len(costs)))
    loads = [sum(costs[i] for i in p) for p in parts]
    assert max(loads) - min(loads) <= max(costs)
    assert parts[0][0] == 0  # the largest item goes to rank 0
    assert lpt_partition(costs, 1) == [list(range(len(costs)))]
    assert lpt_partition([], 2) == [[], []]
    with pytest.raises(ValueError):
        lpt_partition(costs, 0)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime

    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    try:
        from conftest import load_example
        from oracle import oracle as O
        from pdfp_b200 import synthetic
        from pdfp_b200.params import SolverParameters
        from pdfp_b200.shard import feasibility_pump_sharded, solve_batch_sharded
        models = [synthetic.covering_p0201_like(s) for s in (1, 2, 3, 4, 5)]
        probs, targets = [], []
        for s, m in enumerate(models):
            sc, is_eq, is_int, w = O.projector_inputs(m)
            probs.append((sc.A, sc.con_ub, is_eq, is_int, sc.var_lb, sc.var_ub, w))
            targets.append(np.round(np.random.default_rng(s).random(len(m.c))) / sc.D_c)
        prm = SolverParameters(eps_optimal_relative=1e-6, eps_feasible_relative=1e-6)
        xs, rs = solve_batch_sharded(probs, targets, prm, solvers=O.OracleSolvers())
        res, trajs = feasibility_pump_sharded(load_example("p0201"), (101, 201, 7, 11),
                                              solvers=O.OracleSolvers(), time_limit=120,
                                              batch_policy="always")
        out.put((rank, [x.tolist() for x in xs], [r["total_count"] for r in rs],
                 (res.found, res.iterations, res.x.tolist()),
                 [(t.seed, t.found, t.iterations) for t in trajs]))
    finally:
        dist.destroy_process_group()


def test_sharded_batch_and_pump_two_ranks(oracle, examples):
    from pdfp_b200 import synthetic
    from pdfp_b200.params import SolverParameters
    from pdfp_b200.pump import feasibility_pump
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = [q.get(timeout=300) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    got.sort(key=lambda g: g[0])
    (_, xs0, it0, res0, tr0), (_, xs1, it1, res1, tr1) = got
    # every rank holds the whole gathered answer
    assert xs0 == xs1 and it0 == it1 and res0 == res1 and tr0 == tr1
    # ... and it is the one-process batch's answer
    probs, targets = [], []
    for s, m in enumerate(synthetic.covering_p0201_like(k) for k in (1, 2, 3, 4, 5)):
        sc, is_eq, is_int, w = oracle.projector_inputs(m)
        probs.append((sc.A, sc.con_ub, is_eq, is_int, sc.var_lb, sc.var_ub, w))
        targets.append(np.round(np.random.default_rng(s).random(len(m.c))) / sc.D_c)
    b = oracle.OracleSolvers.PDFPBatch(probs)
    for p, t in enumerate(targets):
        b.set_target(p, t)
    b.solve([SolverParameters(eps_optimal_relative=1e-6, eps_feasible_relative=1e-6)] * 5, 1.0)
    for p in range(5):
        assert np.array_equal(np.asarray(xs0[p]), b.get(p, "pdhg_x"))
        assert it0[p] == b.results[p]["total_count"]
    # the pump: the first success over all four seeds, every rank stopped with it
    m = examples["p0201"]
    singles = {s: feasibility_pump(m, solvers=oracle.OracleSolvers(), time_limit=120, seed=s,
                                   batch_policy="always") for s in (101, 201, 7, 11)}
    first = min(r.iterations for r in singles.values() if r.found)
    found, iters, x = res0
    assert found and iters == first
    assert [t[0] for t in tr0] == [101, 201, 7, 11]
    assert all(t[2] == first for t in tr0)
    winners = [t for t in tr0 if t[1]]
    assert winners and all(singles[t[0]].iterations == first for t in winners)
