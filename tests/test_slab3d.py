"""x-slab decomposition of one 3D grid (meep_torch_b200.slab3d) on CPU.

The slab steppers here are the numpy oracle split into its H and E halves
(oracle/fdtd.py step_3d_h / step_3d_e), so these tests check the decomposition itself
-- slab bounds, cropping of state, coefficients, sources and monitors, the halo
exchanges (in-process copies and gloo point-to-point between two ranks), and the
assembly of accumulators and state -- against the whole-grid oracle run, bit for bit
in float64. The same driver runs the library's slab plans on the GPU
(test_gpu_parity.py)."""
import math
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from meep_torch_b200 import slab3d as SL
from meep_torch_b200.core.monitors_3d import DFTFieldsMonitor3D, FluxMonitor3D
from oracle import fdtd as O

NX, NY, NZ, NPML, STEPS = 15, 10, 9, 3, 24
FREQS = [0.35, 0.5]


def _amp(t):
    return math.cos(0.37 * t) * math.exp(-((t - 8.0) / 5.0) ** 2)


class _Src:
    """A source object in the reference's form (``src`` and ``amplitude``)."""

    def __init__(self, src):
        self.src = src

    def amplitude(self, t):
        return _amp(t)


class OracleSlab:
    """A slab stepper with the library plan's interface (begin / half / plane / accs /
    state), stepping the oracle's two halves on numpy arrays."""
    acc_dtype = torch.float64
    device = torch.device("cpu")

    def __init__(self, state, coeffs, source, parts, sl, point_sign=1, **_):
        self.s = {k: v.copy() for k, v in state.items() if v is not None}
        self.c = coeffs
        self.src = None if source is None else source.src
        self.sign = point_sign
        self.mons = [p.monitor for p in parts if p is not None]
        self.accs_np = [None] * len(self.mons)
        self.h = None

    def begin(self, t0, k):
        self.t = t0

    def half(self, part):
        if part == 0:
            self.h = O.step_3d_h(self.s, self.c)
            return
        e = O.step_3d_e(self.s, self.c, self.h, _amp(self.t) if self.src else 0.0, self.src,
                        point_sign=self.sign)
        self.s.update(self.h)
        self.s.update(e)
        for m, mon in enumerate(self.mons):
            smp = _sample(mon, self.s, self.t, self.c["dt"])
            self.accs_np[m] = smp if self.accs_np[m] is None else self.accs_np[m] + smp
        self.t += 1

    def plane(self, comp, i, nxt=False):
        return (self.h if nxt else self.s)[comp][i]

    @property
    def accs(self):
        return [torch.from_numpy(a) for a in self.accs_np]

    def state(self):
        return {k: torch.from_numpy(v) for k, v in self.s.items()}

    def close(self):
        pass


def _sample(mon, s, t, dt):
    if type(mon).__name__ == "FluxMonitor3D":
        return O.flux3d_sample(s, t, dt, FREQS, mon.normal, int(mon.idx),
                               getattr(mon, "win", None), int(getattr(mon, "ap", 0)))
    axis, idx = mon.plane
    sl = [slice(None)] * 3
    sl[axis] = int(idx)
    F = s[mon.component][tuple(sl)]
    w = getattr(mon, "win", None)
    if w is not None:
        F = F[w[0]:w[1], w[2]:w[3]]
    return O.dft_sample(F, t, dt, FREQS, mon.component, np.float64)


def _problem(mask_source=False):
    rng = np.random.default_rng(7)
    eps = 1.0 + 3.0 * rng.random((NX, NY, NZ))
    c = O.coeffs_3d(NX, NY, NZ, 0.1, eps=eps, npml=NPML)
    s = O.state_3d(c)
    if mask_source:
        m = np.zeros((NX, NY, NZ - 1))
        m[4:11, 5, 3:6] = rng.random((7, 3)) + 0.5       # crosses slab boundaries
        src = ("Ez", m)
    else:
        src = ("Ez", 6, 5, 4)
    dt = c["dt"]
    mons = [FluxMonitor3D(dt, FREQS, normal="x", idx=7, ap=1),
            FluxMonitor3D(dt, FREQS, normal="x", idx=5, win=(1, 8, 2, 7)),
            FluxMonitor3D(dt, FREQS, normal="y", idx=4, win=(2, 12, 1, 7)),
            FluxMonitor3D(dt, FREQS, normal="z", idx=5, ap=2),
            DFTFieldsMonitor3D(dt, FREQS, component="Ez", plane=(1, 3)),
            DFTFieldsMonitor3D(dt, FREQS, component="Hy", plane=(0, 10))]
    return s, c, _Src(src), mons


def _whole(s, c, src, mons):
    mfn = [lambda st, t, m=m: _sample(m, st, t, c["dt"]) for m in mons]
    return O.run_3d(s, c, STEPS, amp_fn=_amp, src=src.src, monitors=mfn)


def test_slab_bounds_cover_and_halo():
    for nx, n in ((15, 1), (15, 2), (15, 4), (256, 8), (17, 8)):
        sl = SL.slab_bounds(nx, n)
        assert sl[0].x0 == 0 and sl[-1].x1 == nx
        for a, b in zip(sl, sl[1:]):
            assert a.x1 == b.x0
        widths = [q.x1 - q.x0 for q in sl]
        assert max(widths) - min(widths) <= 1 and min(widths) >= 2
        for q in sl:
            assert q.lo == max(q.x0 - 1, 0) and q.hi == min(q.x1 + 1, nx)
            a, b = q.own_local
            assert (a, b) == (q.x0 - q.lo, q.x1 - q.lo)
    with pytest.raises(ValueError):
        SL.slab_bounds(5, 3)


@pytest.mark.parametrize("n_slabs", [1, 2, 3, 5])
@pytest.mark.parametrize("mask_source", [False, True])
def test_local_slabs_match_whole_grid(n_slabs, mask_source):
    s, c, src, mons = _problem(mask_source)
    ref_s, ref_acc = _whole(s, c, src, mons)
    st, accs = SL.run_3d_slabs({k: v for k, v in s.items()}, c, STEPS, source=src,
                               monitors=mons, n_slabs=n_slabs, make_engine=OracleSlab)
    for a, r in zip(accs, ref_acc):
        assert a.shape == r.shape
        assert np.array_equal(a.numpy(), r)
    for k, v in ref_s.items():
        assert np.array_equal(st[k].numpy(), v), k


def _free_port():
    q = socket.socket()
    q.bind(("127.0.0.1", 0))
    port = q.getsockname()[1]
    q.close()
    return port


def _worker(rank, world, port, mask_source, out_q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        s, c, src, mons = _problem(mask_source)
        st, accs = SL.run_3d_distributed(s, c, STEPS, source=src, monitors=mons, rank=rank,
                                         world=world, make_engine=OracleSlab)
        sl = SL.slab_bounds(NX, world)[rank]
        own = {k: (r0, n, st[k][r0 - sl.lo: r0 - sl.lo + n].numpy())
               for k, (r0, n) in SL.owned_rows(st, sl).items()}
        out_q.put((rank, own, None if accs is None else [a.numpy() for a in accs]))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_distributed_slabs_gloo_match_whole_grid(world):
    s, c, src, mons = _problem(True)
    ref_s, ref_acc = _whole(s, c, src, mons)
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, True, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = {}
    for _ in range(world):
        rank, own, accs = q.get(timeout=180)
        res[rank] = (own, accs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for a, r in zip(res[0][1], ref_acc):
        assert np.array_equal(a, r)
    assert all(res[r][1] is None for r in range(1, world))
    covered = {k: np.zeros(v.shape[0], dtype=int) for k, v in ref_s.items()}
    for r in range(world):
        for k, (r0, n, rows) in res[r][0].items():
            assert np.array_equal(rows, ref_s[k][r0:r0 + n]), (r, k)
            covered[k][r0:r0 + n] += 1
    for k, cov in covered.items():
        # every row owned exactly once (psi_Hz_x / psi_Hy_x start at box plane 1)
        assert np.all(cov == 1), k
