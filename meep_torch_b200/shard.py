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


def distributed_gradient(term_grad: Callable[[list[int]], tuple], n_terms: int, *,
                         rank: int = 0, world: int = 1, group=None, costs=None):
    """Objective and design gradient of a sum of independent terms, split across ranks.

    Design objectives are often sums of terms that each need their own forward + adjoint
    FDTD pair: one per narrowband wavelength, per excitation, or per fabrication scenario
    (nominal / eroded / dilated) of a robust design. ``term_grad(indices)`` evaluates the
    terms ``indices`` on this rank and returns (sum of their objective values, sum of their
    gradients as one tensor). The terms are split by LPT on ``costs`` (default: equal), and
    one all-reduce sums the objectives and gradients, so every rank returns the same
    (J, dJ/drho). A rank with no term contributes zeros (it still joins the collective)."""
    import torch
    parts = lpt_partition(costs if costs is not None else [1.0] * n_terms, world)
    mine = parts[rank]
    J, g = term_grad(mine) if mine else (0.0, None)
    if world == 1:
        return float(J), g
    import torch.distributed as dist
    # the gradient's shape is the same on every rank; ranks without a term learn it here
    shape = torch.tensor(list(g.shape) if g is not None else [], dtype=torch.int64)
    meta = [None] * world
    dist.all_gather_object(meta, (tuple(shape.tolist()), str(g.dtype) if g is not None
                                  else None), group=group)
    ref_shape, ref_dtype = next(m for m in meta if m[1] is not None)
    dev = g.device if g is not None else torch.device("cpu")
    flat = torch.zeros(1 + int(torch.tensor(ref_shape).prod()), dtype=torch.float64,
                       device=dev)
    flat[0] = float(J)
    if g is not None:
        flat[1:] = g.detach().reshape(-1).to(torch.float64)
    dist.all_reduce(flat, op=dist.ReduceOp.SUM, group=group)
    out_dtype = getattr(torch, ref_dtype.replace("torch.", ""))
    return float(flat[0]), flat[1:].reshape(ref_shape).to(out_dtype)
