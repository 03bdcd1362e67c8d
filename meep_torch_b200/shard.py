"""Sharding a batch of independent 2D structures across ranks (one process per GPU).

A batch of structures (the batched-variants workload) needs no exchange while stepping:
each rank advances its own share with one plan, and the monitor accumulators are gathered
once at the end. Shares are balanced by longest-processing-time-first bin packing on the
per-step cost (cells), which keeps the slowest rank -- the one the job waits for -- within
4/3 of the optimum.
"""
from __future__ import annotations

import heapq
from typing import Callable, Sequence


def lpt_partition(costs: Sequence[float], n_parts: int) -> list[list[int]]:
    """Indices of ``costs`` split into ``n_parts`` lists: largest cost first, each to the
    currently lightest part (ties: lower part index, then lower item index). Every part
    keeps its items in ascending index order."""
    if n_parts < 1:
        raise ValueError("n_parts must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    heap = [(0.0, p) for p in range(n_parts)]
    parts: list[list[int]] = [[] for _ in range(n_parts)]
    for i in order:
        load, p = heapq.heappop(heap)
        parts[p].append(i)
        heapq.heappush(heap, (load + float(costs[i]), p))
    return [sorted(q) for q in parts]


def part_loads(costs: Sequence[float], parts: list[list[int]]) -> list[float]:
    return [sum(float(costs[i]) for i in q) for q in parts]


def run_sharded(costs: Sequence[float], run_share: Callable[[list[int]], list], *,
                rank: int = 0, world: int = 1, group=None, dst: int = 0):
    """Run this rank's LPT share and gather every structure's results on ``dst``.

    ``run_share(indices)`` advances the structures ``indices`` (this rank's share) and
    returns one result per index (e.g. its list of accumulators as CPU tensors). On
    ``dst`` the return value is the list of all results in the batch's own order; on the
    other ranks it is None. With world == 1 no collective is called."""
    parts = lpt_partition(costs, world)
    mine = parts[rank]
    local = run_share(mine)
    if len(local) != len(mine):
        raise ValueError("run_share must return one result per index")
    if world == 1:
        return list(local)
    import torch.distributed as dist
    gathered = [None] * world if rank == dst else None
    dist.gather_object(list(zip(mine, local)), gathered, dst=dst, group=group)
    if rank != dst:
        return None
    out = [None] * len(costs)
    for share in gathered:
        for i, res in share:
            out[i] = res
    return out
