"""Multi-GPU execution of batched solves: one process per GPU, independent shards.

The reference solves each system in one process (OpenMP threads only); systems
of a batch are independent, so a multi-GPU run partitions them across ranks by
estimated work, solves each shard with one rsg_batch per GPU (no collective on
the data path), and gathers solutions and statistics to rank 0 once at the end
through torch.distributed (NCCL between GPUs, gloo for CPU tests).
"""
from __future__ import annotations

import heapq

import numpy as np


def estimated_cost(nnz: int, n: int) -> float:
    """Work estimate of one Jacobi-PCG solve: nnz per iteration x iterations ~ n^(1/3) (3-D Poisson-type)."""
    return float(nnz) * max(float(n), 1.0) ** (1.0 / 3.0)


def shard_systems(costs, world: int) -> list[list[int]]:
    """Longest-processing-time-first assignment of systems to ranks (deterministic).

    Returns, for every rank, the ascending list of system indexes it owns."""
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    heap = [(0.0, r) for r in range(world)]
    shards = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        shards[r].append(i)
        heapq.heappush(heap, (load + costs[i], r))
    return [sorted(s) for s in shards]


def solve_sharded(systems, rhs, rank: int, world: int, solve_local, group=None):
    """Solve independent systems across ranks.

    systems: list of (row_ptr, col_idx, values); rhs: list of right-hand sides.
    solve_local(list_of_systems, list_of_rhs) -> (list_of_x, list_of_stats_dicts) runs on this rank
    (rsg.Batch on a GPU).  Returns (all x, all stats) on rank 0 and (None, None) elsewhere.
    """
    import torch.distributed as dist
    costs = [estimated_cost(len(ci), len(rp) - 1) for rp, ci, _ in systems]
    shards = shard_systems(costs, world)
    mine = shards[rank]
    xs, stats = solve_local([systems[i] for i in mine], [rhs[i] for i in mine]) if mine else ([], [])
    payload = (mine, [np.asarray(x) for x in xs], stats)
    gathered = [None] * world if rank == 0 else None
    dist.gather_object(payload, gathered, dst=0, group=group)
    if rank != 0:
        return None, None
    x_all = [None] * len(systems)
    s_all = [None] * len(systems)
    for idxs, xl, sl in gathered:
        for i, x, s in zip(idxs, xl, sl):
            x_all[i] = x
            s_all[i] = s
    return x_all, s_all


def gpu_batch_solver(ctx, conf):
    """solve_local for solve_sharded backed by rsg.Batch on this rank's GPU."""
    import rsg

    def run(systems, rhs):
        batch = rsg.Batch(ctx, systems)
        x, per, _ = batch.solve(np.concatenate(rhs), conf=conf)
        out = batch.split(x), [st.as_dict() for st in per]
        batch.close()
        return out
    return run
