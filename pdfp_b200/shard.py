"""Independent projections and pump trajectories spread over the GPUs of a node.

One process per GPU (``torch.distributed``).  Projections of different
instances and pump trajectories are independent, so nothing crosses between
GPUs inside a solve: instances are dealt to ranks by nonzeros with the
longest-processing-time rule, every rank solves its share in one batch handle
on its own GPU, and the results are gathered on the host at the end.  Pump
trajectories on different ranks agree once per pump iteration on a single flag
("some rank found a feasible point, or the time ran out").

This replaces the reference's process-per-trajectory launcher
(scripts/solve.jl:121-148), which runs independent pump processes and keeps the
first to finish.  Each rank should select its GPU before solving
(``pdfp_b200.gpu.set_device(local_rank)``, as ``torch.cuda.set_device`` does for
torch).
"""
from __future__ import annotations

import heapq


def lpt_partition(costs, world: int):
    """Deal items to ``world`` ranks, largest cost first, each to the least loaded
    rank (lowest rank on ties).  Returns one ascending index list per rank."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    heap = [(0.0, r) for r in range(world)]
    parts = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        parts[r].append(i)
        heapq.heappush(heap, (load + float(costs[i]), r))
    return [sorted(p) for p in parts]


def _world(group):
    import torch.distributed as dist  # noqa: PLC0415
    if not dist.is_available() or not dist.is_initialized():
        return 1, 0
    return dist.get_world_size(group), dist.get_rank(group)


def solve_batch_sharded(problems, targets, params, primal_weight: float = 1.0, *,
                        precision: str = "fp64", solvers=None, group=None,
                        initial_x=None):
    """Project ``targets[p]`` for every problem, the problems shared out over the ranks.

    ``problems`` are the 7- or 8-tuples ``PDFPBatch`` takes (scaled data), the same
    list on every rank; ``params`` one ``SolverParameters`` or one per problem.
    Each rank builds one batch of the problems ``lpt_partition`` gives it (cost =
    nonzeros + rows + columns) and solves it; the host then gathers.  Returns
    ``(x, results)`` in problem order on every rank.
    """
    import torch.distributed as dist  # noqa: PLC0415
    if solvers is None:
        from . import gpu as solvers  # noqa: PLC0415
    world, rank = _world(group)
    k = len(problems)
    if len(targets) != k:
        raise ValueError("one target per problem is required")
    plist = params if isinstance(params, (list, tuple)) else [params] * k
    costs = [pr[0].nnz + pr[0].shape[0] + pr[0].shape[1] for pr in problems]
    mine = lpt_partition(costs, world)[rank]
    local = {}
    if mine:
        batch = solvers.PDFPBatch([problems[i] for i in mine], precision=precision)
        for q, i in enumerate(mine):
            if initial_x is not None:
                batch.set_x(q, initial_x[i])
            batch.set_target(q, targets[i])
        batch.solve([plist[i] for i in mine], primal_weight)
        for q, i in enumerate(mine):
            local[i] = (batch.get(q, "pdhg_x"), dict(batch.results[q]))
        if hasattr(batch, "close"):
            batch.close()
    if world > 1:
        gathered = [None] * world
        dist.all_gather_object(gathered, local, group=group)
        for part in gathered:
            local.update(part)
    return [local[i][0] for i in range(k)], [local[i][1] for i in range(k)]


def feasibility_pump_sharded(milp, seeds, *, group=None, solvers=None, **kwargs):
    """Pump trajectories dealt round-robin to the ranks, each rank's share batched.

    Every rank runs ``feasibility_pump_batched`` on ``seeds[rank::world]``; at the
    head of each pump iteration the ranks all-reduce one flag (found or out of
    time) and stop together.  Returns, on every rank, the winner's
    ``PumpResult`` -- the successful trajectory with the fewest pump iterations,
    lowest rank on ties; trajectory 0 of rank 0 when none succeeded -- and all
    ranks' ``TrajectoryResult`` lists in seed order.
    """
    import torch
    import torch.distributed as dist  # noqa: PLC0415

    from .pump import feasibility_pump_batched  # noqa: PLC0415
    world, rank = _world(group)
    mine = list(seeds)[rank::world]
    if not mine:
        raise ValueError("need at least one pump seed per rank")

    def stop(done: bool) -> bool:
        if world == 1:
            return done
        flag = torch.tensor([1 if done else 0], dtype=torch.int32)
        dist.all_reduce(flag, op=dist.ReduceOp.MAX, group=group)
        return bool(flag.item())

    res, trajs = feasibility_pump_batched(milp, seeds=mine, solvers=solvers, stop=stop, **kwargs)
    gathered = [(res, trajs)]
    if world > 1:
        gathered = [None] * world
        dist.all_gather_object(gathered, (res, trajs), group=group)
    winners = [(r.iterations, q) for q, (r, _) in enumerate(gathered) if r.found]
    best = gathered[min(winners)[1]][0] if winners else gathered[0][0]
    by_seed = {t.seed: t for _, ts in gathered for t in ts}
    return best, [by_seed[s] for s in seeds]
