"""One 3D grid split along x into slabs, one slab per rank (one process per GPU).

The reference advances the whole grid in one process (``run_3d``, core/monitors_3d.py:
192-210). Here rank r owns the x planes [x0, x1) and holds [lo, hi) = [x0 - 1, x1 + 1)
clipped to the grid: one halo plane on each side that has a neighbour. Every array of
the reference state has an x extent nx - c (c = 0, 1, 2), and box plane i of the
library's layout is global plane lo + i, so a slab is the global problem cropped to
[lo, hi) with updates restricted to the owned planes (``mtb_yee3d_set_slab``).

One step is two exchanges of two components each (the only x derivatives of the
Yee update):

- H(n+1/2) at plane x1-1 needs Ey, Ez(n) at plane x1: after each E update, rank r
  sends Ey, Ez of its first owned plane x0 to rank r-1 (its right halo);
- E(n+1) at plane x0 needs Hy, Hz(n+1/2) at plane x0-1: after each H update, rank r
  sends Hy, Hz of its last owned plane x1-1 to rank r+1 (its left halo).

Halo planes are contiguous in the box layout (ny x zpitch floats), so they travel as
they are: torch.distributed point-to-point (NCCL over NVLink on GPUs, gloo on CPU)
between ranks, a device copy between slabs of one process. Monitors are cropped to
the owned planes; their accumulators are summed onto rank 0 once at the end.
"""
from __future__ import annotations

import copy
from dataclasses import dataclass

import numpy as np
import torch

from .engine3d import FIELDS, PSI, PSI_OFF, field_shapes, flux_window

__all__ = ["Slab", "slab_bounds", "slice_state", "slice_coeffs", "slice_source",
           "slice_monitors", "LocalHalo", "DistHalo", "SlabDriver", "run_3d_slabs",
           "run_3d_distributed"]

# x offset of each state array's row 0 in box planes (psi_Hz_x, psi_Hy_x cover the
# interior of x)
X_OFF = {k: 0 for k in FIELDS}
X_OFF.update({k: PSI_OFF[q][0] for q, k in enumerate(PSI)})


@dataclass(frozen=True)
class Slab:
    """Rank ``r`` of ``n``: owned planes [x0, x1), held planes [lo, hi) of ``nx``."""
    r: int
    n: int
    nx: int
    x0: int
    x1: int

    @property
    def lo(self) -> int:
        return self.x0 - 1 if self.x0 > 0 else 0

    @property
    def hi(self) -> int:
        return self.x1 + 1 if self.x1 < self.nx else self.nx

    @property
    def nx_local(self) -> int:
        return self.hi - self.lo

    @property
    def own_local(self) -> tuple[int, int]:
        return self.x0 - self.lo, self.x1 - self.lo


def slab_bounds(nx: int, n: int) -> list[Slab]:
    """``n`` contiguous slabs of near-equal width (the first nx % n one plane wider)."""
    if n < 1:
        raise ValueError("n must be >= 1")
    if nx < 2 * n:
        raise ValueError(f"nx = {nx} too small for {n} slabs (>= 2 planes each)")
    base, rem = divmod(nx, n)
    out, x = [], 0
    for r in range(n):
        w = base + (1 if r < rem else 0)
        out.append(Slab(r, n, nx, x, x + w))
        x += w
    return out


def _rows(t, nx: int, sl: Slab):
    """Rows [lo, hi - c) of an array whose x extent is nx - c."""
    c = nx - t.shape[0]
    if c < 0 or c > 2:
        raise ValueError(f"x extent {t.shape[0]} of a grid with nx = {nx}")
    return t[sl.lo: sl.hi - c]


def _copy(x):
    return x.clone() if isinstance(x, torch.Tensor) else x.copy()


def _stack(parts, like):
    return torch.stack(parts) if isinstance(like, torch.Tensor) else np.stack(parts)


def _slice_any(k, v, sl: Slab):
    """Rows of a state array; a pole stack (P*: one plane per pole) along its dim 1."""
    if v is None:
        return None
    if k.startswith("P"):
        if v.shape[0] == 0:
            return _copy(v[:, sl.lo: sl.hi - (sl.nx - v.shape[1])])
        return _stack([_copy(_rows(p, sl.nx, sl)) for p in v], v)
    return _copy(_rows(v, sl.nx, sl))


def slice_state(state, sl: Slab):
    """The slab's part of a State3D (or dict): every array cropped to planes [lo, hi)
    (pole stacks along their x axis, dim 1)."""
    g = state if isinstance(state, dict) else state._asdict()
    out = {k: _slice_any(k, v, sl) for k, v in g.items()}
    return out if isinstance(state, dict) else type(state)(**out)


def slice_coeffs(coeffs, sl: Slab):
    """Coeffs3D (or the oracle's dict) cropped to [lo, hi): eps, full-grid damping pairs
    and the x CPML profiles (half nodes "hx" n-1, interior nodes "ex" n-2)."""
    g = coeffs if isinstance(coeffs, dict) else coeffs._asdict()
    nx = sl.nx
    cp = dict(g["cpml"])
    for key in ("hx", "ex"):
        cp[key] = tuple(_rows(v, nx, sl) for v in cp[key])
    out = dict(g)
    out["cpml"] = cp
    out["eps"] = g["eps"][sl.lo: sl.hi]
    pols = g.get("pols")
    if isinstance(pols, dict):                           # c3 stacks along their dim 1
        out["pols"] = {k: (c1, c2, _stack([_rows(p, nx, sl) for p in c3], c3))
                       for k, (c1, c2, c3) in pols.items()}
    damp = g.get("damp")
    if isinstance(damp, dict):
        out["damp"] = {k: tuple(_rows(v, nx, sl) if getattr(v, "ndim", 0) == 3 else v
                                for v in pair) for k, pair in damp.items()}
    if "dims" in out:
        out["dims"] = (sl.nx_local,) + tuple(out["dims"][1:])
    return out if isinstance(coeffs, dict) else type(coeffs)(**out)


def slice_source(source, sl: Slab):
    """The slab's share of a 3D soft current (a copy of the source with its ``src``
    moved to local planes), or None when no source cell is owned. Point and
    plane-indexed forms go to the owner of their plane; a mask keeps its owned planes."""
    if source is None:
        return None
    src = source.src
    comp = src[0]
    if getattr(src[1], "ndim", 0) == 3:                  # (comp, mask)
        m = _copy(_rows(src[1], sl.nx, sl))
        a, b = sl.own_local
        m[:a] = 0
        m[b:] = 0
        if not bool((m != 0).any()):
            return None
        new = (comp, m)
    else:
        i = int(src[1])
        if not (sl.x0 <= i < sl.x1):
            return None
        new = (comp, i - sl.lo) + tuple(src[2:])
    out = copy.copy(source)
    out.src = new
    return out


@dataclass
class MonitorPart:
    """Where a slab's accumulator goes in the global one: rows [row0, row0 + rows) of
    dim 2, or the whole accumulator (row0 = 0 and rows = all)."""
    monitor: object          # the slab-local monitor
    row0: int
    rows: int


def _plane_shape(mon, nx, ny, nz):
    axis, idx = mon.plane
    shp = field_shapes(nx, ny, nz)[mon.component]
    a0, a1 = [a for a in range(3) if a != axis]
    return axis, int(idx), shp[a0], shp[a1]


def global_acc_shape(mon, nx, ny, nz):
    nf = len(mon.freqs)
    if type(mon).__name__ == "FluxMonitor3D":
        _, w = flux_window(mon.normal, int(mon.idx), nx, ny, nz, getattr(mon, "win", None),
                           int(getattr(mon, "ap", 0)))
        return (nf, 8, max(0, w[1] - w[0]), max(0, w[3] - w[2]))
    _, _, m0, m1 = _plane_shape(mon, nx, ny, nz)
    return (nf, 2, m0, m1)


def slice_monitors(monitors, sl: Slab, ny: int, nz: int) -> list[MonitorPart | None]:
    """Each monitor's slab-local copy (plane index and window in local planes) with its
    place in the global accumulator, or None when the slab owns none of it. An
    x-normal plane belongs to the owner of its plane; y- and z-normal planes are split
    by their x rows. H samples one plane below an x-normal plane (core/monitors_3d.py:
    124-162), which is the left halo when the plane is x0: it holds H(n+1/2) of that
    plane when the samples are taken."""
    nx = sl.nx
    out = []
    for mon in monitors:
        kind = type(mon).__name__
        if kind == "FluxMonitor3D":
            idx = int(mon.idx)
            _, w = flux_window(mon.normal, idx, nx, ny, nz, getattr(mon, "win", None),
                               int(getattr(mon, "ap", 0)))
            l0, h0, l1, h1 = w
            loc = copy.copy(mon)
            loc.ap = 0
            if mon.normal == "x":
                if not (sl.x0 <= idx < sl.x1) or h0 <= l0 or h1 <= l1:
                    out.append(None)
                    continue
                loc.idx = idx - sl.lo
                loc.win = (l0, h0, l1, h1)
                out.append(MonitorPart(loc, 0, h0 - l0))
            else:                                        # rows of the window are x
                r0, r1 = max(l0, sl.x0), min(h0, sl.x1)
                if r1 <= r0 or h1 <= l1:
                    out.append(None)
                    continue
                loc.win = (r0 - sl.lo, r1 - sl.lo, l1, h1)
                out.append(MonitorPart(loc, r0 - l0, r1 - r0))
        elif kind == "DFTFieldsMonitor3D":
            axis, idx, m0, m1 = _plane_shape(mon, nx, ny, nz)
            w = getattr(mon, "win", None) or (0, m0, 0, m1)
            loc = copy.copy(mon)
            if axis == 0:
                if not (sl.x0 <= idx < sl.x1):
                    out.append(None)
                    continue
                loc.plane = (0, idx - sl.lo)
                loc.win = tuple(w)
                out.append(MonitorPart(loc, 0, w[1] - w[0]))
            else:
                r0, r1 = max(w[0], sl.x0), min(w[1], sl.x1)
                if r1 <= r0:
                    out.append(None)
                    continue
                loc.win = (r0 - sl.lo, r1 - sl.lo, w[2], w[3])
                out.append(MonitorPart(loc, r0 - w[0], r1 - r0))
        else:
            raise NotImplementedError(f"3D monitor {kind} on x slabs")
    return out


def _t(x):
    """A torch view of a plane (numpy planes of the CPU oracle engines share memory)."""
    return x if isinstance(x, torch.Tensor) else torch.from_numpy(x)


class LocalHalo:
    """All slabs in one process: halo planes move by copies on the current stream."""

    def __init__(self, engines, slabs):
        self.engines, self.slabs = engines, slabs

    def after_h(self):
        for r in range(1, len(self.slabs)):
            a, b = self.engines[r - 1], self.engines[r]
            src = self.slabs[r].x0 - 1 - self.slabs[r - 1].lo
            for c in ("Hy", "Hz"):
                _t(b.plane(c, 0, nxt=True)).copy_(_t(a.plane(c, src, nxt=True)))

    def after_e(self):
        for r in range(len(self.slabs) - 1):
            a, b = self.engines[r], self.engines[r + 1]
            dst = self.slabs[r].nx_local - 1
            src = self.slabs[r].x1 - self.slabs[r + 1].lo
            for c in ("Ey", "Ez"):
                _t(a.plane(c, dst)).copy_(_t(b.plane(c, src)))


class DistHalo:
    """One slab per rank: torch.distributed point-to-point with the neighbours."""

    def __init__(self, engine, slab: Slab, group=None):
        import torch.distributed as dist
        self.dist = dist
        self.e, self.sl, self.group = engine, slab, group

    def _peer(self, r):
        g = self.group
        return r if g is None else self.dist.get_global_rank(g, r)

    def _swap(self, sends, recvs):
        d = self.dist
        ops = [d.P2POp(d.isend, _t(x), self._peer(p), self.group) for p, x in sends]
        ops += [d.P2POp(d.irecv, _t(x), self._peer(p), self.group) for p, x in recvs]
        if ops:
            for w in d.batch_isend_irecv(ops):
                w.wait()

    def after_h(self):
        sl, e = self.sl, self.e
        sends = [(sl.r + 1, e.plane(c, sl.x1 - 1 - sl.lo, nxt=True)) for c in ("Hy", "Hz")] \
            if sl.r + 1 < sl.n else []
        recvs = [(sl.r - 1, e.plane(c, 0, nxt=True)) for c in ("Hy", "Hz")] if sl.r > 0 else []
        self._swap(sends, recvs)

    def after_e(self):
        sl, e = self.sl, self.e
        sends = [(sl.r - 1, e.plane(c, sl.x0 - sl.lo)) for c in ("Ey", "Ez")] if sl.r > 0 else []
        recvs = [(sl.r + 1, e.plane(c, sl.nx_local - 1)) for c in ("Ey", "Ez")] \
            if sl.r + 1 < sl.n else []
        self._swap(sends, recvs)


class SlabDriver:
    """Steps a set of slab engines (``begin``/``half``/``plane``) with a halo transport."""

    def __init__(self, engines, halo):
        self.engines, self.halo = engines, halo

    def run(self, t0: int, k: int):
        if k <= 0:
            return
        for e in self.engines:
            e.begin(t0, k)
        for _ in range(k):
            for e in self.engines:
                e.half(0)
            self.halo.after_h()
            for e in self.engines:
                e.half(1)
            self.halo.after_e()


def assemble_accs(monitors, parts_per_slab, accs_per_slab, nx, ny, nz, like):
    """Global accumulators from the slabs' parts (a sum of disjoint row blocks)."""
    out = []
    for m, mon in enumerate(monitors):
        shp = global_acc_shape(mon, nx, ny, nz)
        g = torch.zeros(shp, dtype=like.dtype, device=like.device)
        for parts, accs in zip(parts_per_slab, accs_per_slab):
            p = parts[m]
            if p is not None:
                g[:, :, p.row0: p.row0 + p.rows] += accs[m]
        out.append(g)
    return out


def owned_rows(state, sl: Slab):
    """{name: (global row0, rows)} of the owned planes of a slab-local state."""
    g = state if isinstance(state, dict) else state._asdict()
    out = {}
    for k, v in g.items():
        pole = k.startswith("P") and v is not None and v.ndim == 4
        if v is None or (k not in X_OFF and not pole):
            continue
        c = sl.nx_local - v.shape[1 if pole else 0]         # x extent nx - c
        o = 0 if pole else X_OFF[k]
        r0 = max(sl.x0 - o, 0)
        r1 = min(sl.x1 - o, sl.nx - c)
        out[k] = (r0, max(0, r1 - r0))
    return out


def assemble_state(state_like, slabs, local_states):
    """The global state from the owned rows of every slab."""
    g = state_like if isinstance(state_like, dict) else state_like._asdict()
    l0 = local_states[0] if isinstance(local_states[0], dict) else local_states[0]._asdict()
    out = {k: (None if v is None or l0.get(k) is None else
               torch.empty(tuple(v.shape), dtype=l0[k].dtype, device=l0[k].device))
           for k, v in g.items()}
    for sl, ls in zip(slabs, local_states):
        lg = ls if isinstance(ls, dict) else ls._asdict()
        for k, (r0, n) in owned_rows(ls, sl).items():
            if n > 0 and k.startswith("P") and lg[k].ndim == 4:
                out[k][:, r0: r0 + n] = lg[k][:, r0 - sl.lo: r0 - sl.lo + n]
            elif n > 0:
                out[k][r0: r0 + n] = lg[k][r0 - sl.lo: r0 - sl.lo + n]
    return out if isinstance(state_like, dict) else type(state_like)(**out)


def _engine(state, coeffs, source, parts, sl, **kw):
    """The library plan of one slab (Engine3D restricted to the owned planes)."""
    from .engine3d import Engine3D
    mons = [p.monitor for p in parts if p is not None]
    return Engine3D(state, coeffs, source, mons, own=sl.own_local, **kw)


def _expand_accs(parts, accs):
    """Per-monitor list (None where the slab holds no part) from the engine's list."""
    it = iter(accs)
    return [None if p is None else next(it) for p in parts]


def _dims(state):
    Ex = state["Ex"] if isinstance(state, dict) else state.Ex
    return Ex.shape[0] + 1, Ex.shape[1], Ex.shape[2]


def run_3d_slabs(state, coeffs, n_steps: int, *, source=None, monitors=(), n_slabs: int = 2,
                 point_sign: int = 1, phase_mode: str = "exact", ring_slots: int = 0,
                 make_engine=None):
    """``run_3d`` (core/monitors_3d.py:192-210) with the grid split into ``n_slabs`` x
    slabs held by this process on one device: the single-process form of
    ``run_3d_distributed``, with the same per-slab plans and halo planes.
    ``make_engine(state, coeffs, source, parts, slab, **kw)`` builds a slab's stepper
    (default: the library plan)."""
    monitors = list(monitors)
    nx, ny, nz = _dims(state)
    slabs = slab_bounds(nx, n_slabs)
    make = make_engine or _engine
    engines, parts_all = [], []
    try:
        for sl in slabs:
            parts = slice_monitors(monitors, sl, ny, nz)
            parts_all.append(parts)
            engines.append(make(slice_state(state, sl), slice_coeffs(coeffs, sl),
                                slice_source(source, sl), parts, sl, point_sign=point_sign,
                                phase_mode=phase_mode, ring_slots=ring_slots))
        SlabDriver(engines, LocalHalo(engines, slabs)).run(0, n_steps)
        like = engines[0].accs[0] if engines[0].accs else torch.zeros(())
        accs = assemble_accs(monitors, parts_all,
                             [_expand_accs(p, e.accs) for p, e in zip(parts_all, engines)],
                             nx, ny, nz, like)
        st = assemble_state(state, slabs, [e.state() for e in engines])
        return st, accs
    finally:
        for e in engines:
            e.close()


def run_3d_distributed(state, coeffs, n_steps: int, *, source=None, monitors=(), rank: int,
                       world: int, group=None, point_sign: int = 1, phase_mode: str = "exact",
                       ring_slots: int = 0, dst: int = 0, keep_engine: bool = False,
                       make_engine=None):
    """``run_3d`` with rank ``rank`` of ``world`` advancing slab ``rank`` of the grid
    (``state``/``coeffs`` are the global problem, identical on every rank). Returns
    (slab-local state, accs): the global accumulators on ``dst``, None elsewhere. With
    ``keep_engine`` the engine is returned third (for timing) and not closed."""
    import torch.distributed as dist
    monitors = list(monitors)
    nx, ny, nz = _dims(state)
    sl = slab_bounds(nx, world)[rank]
    parts = slice_monitors(monitors, sl, ny, nz)
    make = make_engine or _engine
    eng = make(slice_state(state, sl), slice_coeffs(coeffs, sl), slice_source(source, sl),
               parts, sl, point_sign=point_sign, phase_mode=phase_mode, ring_slots=ring_slots)
    try:
        SlabDriver([eng], DistHalo(eng, sl, group)).run(0, n_steps)
        mine = _expand_accs(parts, eng.accs)
        accs = []
        for m, mon in enumerate(monitors):
            g = torch.zeros(global_acc_shape(mon, nx, ny, nz),
                            dtype=getattr(eng, "acc_dtype", torch.float32), device=eng.device)
            if parts[m] is not None:
                g[:, :, parts[m].row0: parts[m].row0 + parts[m].rows] = mine[m]
            dist.reduce(g, dst=dst if group is None else dist.get_global_rank(group, dst),
                        op=dist.ReduceOp.SUM, group=group)
            accs.append(g if rank == dst else None)
        out = (eng.state(), accs if rank == dst else None)
        return out + (eng,) if keep_engine else out
    finally:
        if not keep_engine:
            eng.close()
