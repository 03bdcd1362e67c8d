"""Batch sharding across ranks (meep_torch_b200.shard): the LPT partition and the
end-of-run gather, with two gloo ranks on CPU (the data path has no collective; the
per-rank step is stubbed here and runs on the GPU through Engine2D in the bench)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from meep_torch_b200.shard import lpt_partition, part_loads, run_sharded


def test_lpt_partition_covers_and_balances():
    from meep_torch_b200 import workloads as W
    costs = [s["nx"] * s["ny"] for s in W.cfg2_specs(256)]
    for world in (1, 2, 3, 4, 8):
        parts = lpt_partition(costs, world)
        flat = sorted(i for q in parts for i in q)
        assert flat == list(range(len(costs)))
        loads = part_loads(costs, parts)
        # LPT bound: max load <= 4/3 OPT, and OPT >= max(total / world, max item)
        lower = max(sum(costs) / world, max(costs))
        assert max(loads) <= 4.0 / 3.0 * lower + 1e-9
        assert max(loads) / (sum(costs) / world) < 1.01        # 256 items: nearly even


def test_lpt_partition_small_cases():
    assert lpt_partition([5, 4, 3, 3], 2) == [[0, 3], [1, 2]]
    assert lpt_partition([1, 1, 1], 4) == [[0], [1], [2], []]
    with pytest.raises(ValueError):
        lpt_partition([1], 0)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, costs, q):
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        seen = []

        def run_share(idx):
            seen.extend(idx)
            # a deterministic per-structure "accumulator"
            return [torch.full((2, 3), float(i) * 10 + rank * 0) + torch.arange(3.0)
                    for i in idx]

        out = run_sharded(costs, run_share, rank=rank, world=world)
        q.put((rank, seen, None if out is None else [t.tolist() for t in out]))
    finally:
        dist.destroy_process_group()


def test_run_sharded_gathers_in_batch_order_two_ranks():
    costs = list(np.random.default_rng(3).integers(1, 100, size=11))
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, costs, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = {}
    for _ in range(world):
        rank, seen, out = q.get(timeout=120)
        res[rank] = (seen, out)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    parts = lpt_partition(costs, world)
    assert res[0][0] == parts[0] and res[1][0] == parts[1]
    assert res[1][1] is None
    out = res[0][1]
    assert len(out) == len(costs)
    for i, t in enumerate(out):
        assert t == [[i * 10 + c for c in range(3)]] * 2


def test_run_sharded_single_rank_needs_no_collective():
    out = run_sharded([3, 1, 2], lambda idx: [i * 2 for i in idx])
    assert out == [0, 2, 4]


def _term(i):
    """A stand-in objective term i and its gradient over a 4 x 5 design."""
    import torch
    rho = torch.linspace(0, 1, 20, dtype=torch.float64).reshape(4, 5)
    return float((i + 1) * rho.sum()), (i + 1) * torch.cos(rho + i)


def _grad_worker(rank, world, port, n_terms, q):
    import torch
    import torch.distributed as dist

    from meep_torch_b200.shard import distributed_gradient
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        seen = []

        def term_grad(idx):
            seen.extend(idx)
            J, g = 0.0, torch.zeros(4, 5, dtype=torch.float64)
            for i in idx:
                a, b = _term(i)
                J, g = J + a, g + b
            return J, g

        J, g = distributed_gradient(term_grad, n_terms, rank=rank, world=world)
        q.put((rank, seen, J, g.tolist()))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,n_terms", [(2, 3), (3, 2)])
def test_distributed_gradient_sums_terms_across_ranks(world, n_terms):
    """Objective terms (wavelengths / scenarios) split over gloo ranks: every rank ends with
    the single-process sum of objectives and gradients, each term evaluated exactly once;
    a rank without a term (3 ranks, 2 terms) still joins the all-reduce."""
    import torch
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_grad_worker, args=(r, world, port, n_terms, q))
             for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    J_ref = sum(_term(i)[0] for i in range(n_terms))
    g_ref = sum(_term(i)[1] for i in range(n_terms))
    assert sorted(i for r in res for i in r[1]) == list(range(n_terms))
    for rank, seen, J, g in res:
        assert abs(J - J_ref) < 1e-12 * abs(J_ref)
        assert torch.allclose(torch.tensor(g, dtype=torch.float64), g_ref, rtol=1e-14)
