"""Checkpointed 3D adjoint on the B200 kernels (reference: core/adjoint3d.py:56-115).

``run_3d_adjoint(c, n_steps, chunk, source, monitors, loss_fn, state0)`` keeps the
reference's signature and result, ``(loss_value, accs)``, with d loss / d eps accumulated
into whatever graph produced ``c.eps``. Instead of re-running each chunk under torch
autograd, the reverse sweep runs the library's discrete-adjoint kernels
(``mtb_yee3d_adjoint_*``): the exact transpose of the forward split step and of the plane
sampling. Per chunk (last first) the chunk's start state is restored on a recording plan,
which re-runs the chunk step by step keeping E after every step (d/d eps of
E' = E + (dt curl + s) / eps_c needs the increment); the adjoint plan then sweeps the
chunk's steps in reverse. ``chunk`` bounds that record (at most 32 steps are kept at a
time); the gradient does not depend on it. Conductive damping and dispersive poles are
transposed with the step (the pole recurrence is linear, so its adjoint needs no record
of P), and so are PMC walls.
"""
from __future__ import annotations

import ctypes as C

import torch

from .. import _lib as L
from ..engine3d import Engine3D

__all__ = ["run_3d_adjoint"]


def run_3d_adjoint(c, n_steps: int, chunk: int, source, monitors, loss_fn, state0):
    """Returns (loss_value, accs); gradients accumulate on the graph of ``c.eps``.
    ``loss_fn(accs)`` must return a real scalar built from the monitor accumulators."""
    monitors = list(monitors)
    n = int(n_steps)
    K = max(1, min(int(chunk), 32))
    eps_src = c.eps
    cd = c._replace(eps=eps_src.detach())
    eng = Engine3D(state0, cd, source, monitors, point_sign=+1, ring_slots=K)
    rec = adj = None
    try:
        chunks = [(s0, min(K, n - s0)) for s0 in range(0, n, K)]
        snaps = []
        for s0, k in chunks:
            snaps.append(eng.snapshot())
            eng.run(s0, k)
        accs = [a.clone() for a in eng.accs]
        accs_leaf = [a.detach().clone().requires_grad_(True) for a in accs]
        with torch.enable_grad():
            loss = loss_fn(accs_leaf)
        g_accs = torch.autograd.grad(loss, accs_leaf, allow_unused=True)
        g_accs = [torch.zeros_like(a) if g is None else g.detach().to(torch.float32).contiguous()
                  for a, g in zip(accs, g_accs)]
        lib = L.load()
        nx, ny, nz, zp = eng.nx, eng.ny, eng.nz, eng.zp
        dev = eng.device
        box = lambda: torch.zeros((nx, ny, zp), dtype=torch.float32, device=dev)  # noqa: E731
        gf, gpsi, tmp, geps = [box() for _ in range(6)], [box() for _ in range(12)], \
            [box() for _ in range(15)], box()
        bufs = L.Adj3DBuffers()
        for q in range(6):
            bufs.g[q] = L.ptr(gf[q])
        for q in range(12):
            bufs.g_psi[q] = L.ptr(gpsi[q])
        for q in range(15):
            bufs.tmp[q] = L.ptr(tmp[q])
        bufs.g_eps = L.ptr(geps)
        # with poles: d J / d P(n) and d J / d P(n-1) per E component, n_poles boxes each
        gpol = [[torch.zeros((eng.n_poles * nx, ny, zp), dtype=torch.float32, device=dev)
                 for _ in range(2)] for _ in range(3)] if eng.n_poles else []
        for c, pair in enumerate(gpol):
            for h in range(2):
                bufs.g_pol[c][h] = L.ptr(pair[h])
        by_ptr = {L.ptr(a): q for q, a in enumerate(eng.accs)}
        nreg = eng.n_regions
        regs = (L.DftRegion * max(1, nreg))()
        for r in range(nreg):
            C.memmove(C.addressof(regs[r]), C.addressof(eng.regions[r]), C.sizeof(L.DftRegion))
            regs[r].acc = L.ptr(g_accs[by_ptr[int(eng.regions[r].acc)]])
        adj = C.c_void_p()
        L.check(lib.mtb_yee3d_adjoint_create(C.byref(eng.S), C.byref(bufs),
                                             regs if nreg else None, nreg, eng.groups,
                                             eng.n_groups, eng.ring_elems, K, C.byref(adj)),
                "mtb_yee3d_adjoint_create")
        keep = [gf, gpsi, tmp, geps, g_accs, gpol]
        N = nx * ny * zp
        record = torch.empty((K + 1, 3, nx, ny, zp), dtype=torch.float32, device=dev)
        rec = Engine3D(state0, cd, source, [], point_sign=+1, ring_slots=K)
        stream = eng._sptr()
        for ci in range(len(chunks) - 1, -1, -1):
            s0, k = chunks[ci]
            rec.restore(snaps[ci])
            for cc, t in enumerate(rec.live_e()):
                record[0, cc].copy_(t)
            for q in range(k):
                rec.run(s0 + q, 1)
                for cc, t in enumerate(rec.live_e()):
                    record[q + 1, cc].copy_(t)
            L.check(lib.mtb_yee3d_adjoint_run(adj, s0, k, L.ptr(record), N, 3 * N, stream),
                    "mtb_yee3d_adjoint_run")
        g_eps = eng._unpack(geps, (nx, ny, nz))
        del keep
    finally:
        if adj is not None:
            L.load().mtb_yee3d_adjoint_destroy(adj)
        if rec is not None:
            rec.close()
        eng.close()
    if eps_src.requires_grad:
        torch.autograd.backward(eps_src, g_eps.to(eps_src.dtype))
    return float(loss.detach()), accs
