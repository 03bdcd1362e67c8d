"""Data-parallel surrogate training and sharded data generation with two gloo ranks on
CPU: shard ranges, the global target scale, the broadcast of rank 0's parameters and the
per-step gradient all-reduce (train_fno under torch.distributed)."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from meep_torch_b200 import surrogate as S


def test_shard_range_covers():
    for n in (0, 1, 7, 20000, 20256):
        for world in (1, 2, 3, 8):
            parts = [S.shard_range(n, r, world) for r in range(world)]
            assert parts[0][0] == 0 and parts[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(parts, parts[1:]))
            sizes = [b - a for a, b in parts]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        S.shard_range(4, 2, 2)


def _data(n=16):
    g = torch.Generator().manual_seed(7)
    x = torch.rand(n, 1, 16, 16, generator=g)
    y = torch.randn(n, 6, 16, 16, generator=g) * (1.0 + torch.arange(n).view(n, 1, 1, 1))
    return x, y


def _flat(model):
    return torch.cat([(torch.view_as_real(p.detach()) if p.is_complex() else p.detach())
                      .reshape(-1) for p in model.parameters()]).double().numpy()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, mode, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        torch.manual_seed(100 + rank)                      # different inits: rank 0's wins
        m = S.FNO2d(width=8, modes=4, layers=2)
        x, y = _data()
        if mode == "same":
            xs, ys = x[:8], y[:8]
        else:
            a, b = S.shard_range(x.shape[0] - 1, rank, world)   # 8 and 7 designs
            xs, ys = x[a:b], y[a:b]
        scale, _ = S.train_fno(m, xs, ys, epochs=2, batch=4, lr=1e-2)
        q.put((rank, scale, _flat(m).tolist()))
    finally:
        dist.destroy_process_group()


def _run(mode):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, 2, port, mode, q)) for r in range(2)]
    for p in ps:
        p.start()
    out = dict((r, (s, np.array(v))) for r, s, v in (q.get(timeout=300) for _ in ps))
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    return out


def test_data_parallel_identical_shards_equal_single_process():
    """With the same shard on both ranks the mean gradient is each rank's own, so the
    two-rank run equals a one-process run from rank 0's initial parameters."""
    out = _run("same")
    torch.manual_seed(100)
    m = S.FNO2d(width=8, modes=4, layers=2)
    x, y = _data()
    scale, _ = S.train_fno(m, x[:8], y[:8], epochs=2, batch=4, lr=1e-2)
    for r in (0, 1):
        assert out[r][0] == pytest.approx(scale, rel=1e-12)
        np.testing.assert_allclose(out[r][1], _flat(m), rtol=1e-5, atol=1e-7)


def test_data_parallel_shards_stay_in_sync():
    """Different shards (8 and 7 designs): the ranks share one global scale, take the
    smaller shard's step count and end with identical parameters."""
    out = _run("split")
    x, y = _data()
    rms = float(y[:15].double().pow(2).mean().sqrt())
    assert out[0][0] == pytest.approx(rms, rel=1e-6) and out[1][0] == out[0][0]
    np.testing.assert_array_equal(out[0][1], out[1][1])
    torch.manual_seed(100)
    assert not np.allclose(out[0][1], _flat(S.FNO2d(width=8, modes=4, layers=2)))
