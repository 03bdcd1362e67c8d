"""Reverse-mode gradients of the 2D TM and TE runs through the B200 kernels.

The reference gets dJ/d eps from torch autograd through ``run_tm`` (core/run.py:43-120),
optionally checkpointed (``checkpoint_every``). Here the same derivative comes from the
library's discrete-adjoint kernels (``mtb_yee2d_adjoint_*``): the exact transpose of the
forward TM step with CPML and of the DFT / flux sampling, run backwards in time.

Forward: the run goes in chunks of ``chunk`` steps (the checkpoint interval); the live
state at each chunk start is kept (box layout). Backward, chunk by chunk from the last: the
chunk is re-run from its snapshot on a recording plan whose ring keeps the full-grid E of
every step (Ez for TM, Ex and Ey for TE: needed for d/d eps of E = D / eps), then the
adjoint plan sweeps the chunk's steps in reverse. The ring holds at most 64 steps, so a
longer chunk is walked forward once keeping the state at the start of each 64-step
sub-chunk, and the sub-chunks are then recorded and reversed from the last. Gradients reach ``coeffs.eps_inf`` (TM) or
``coeffs.eps_x`` / ``coeffs.eps_y`` (TE, and through them ``eps_inf``); other coefficient
tensors and the initial state receive none (a gradient request for them raises
NotImplementedError).
"""
from __future__ import annotations

import ctypes as C

import torch

from . import _lib as L
from .engine2d import Engine2D, _cuts

STATE_TM = ("Ez", "Hx", "Hy", "Dz", "psi_Ezy", "psi_Ezx", "psi_Hyx", "psi_Hxy")
STATE_TE = ("Hz", "Ex", "Ey", "Dx", "Dy", "psi_Hzy", "psi_Hzx", "psi_Eyx", "psi_Exy")


class _Grid:
    """The attributes a DFTFieldsMonitor takes from a Grid."""

    def __init__(self, dt, device):
        self.dt, self.dtype, self.device = dt, torch.float32, device


def _record_monitors(dt, device, te):
    from .core.monitors import DFTFieldsMonitor
    comps = ("Ex", "Ey") if te else ("Ez",)
    return [DFTFieldsMonitor(_Grid(dt, device), [1.0], c) for c in comps]


class GradRun2D:
    """One differentiable TM or TE run: forward() keeps chunk snapshots, backward()
    turns output gradients into d J / d eps (TM eps_inf; TE eps_x, eps_y)."""

    def __init__(self, state, coeffs, n_steps, source, monitors, chunk=32,
                 phase_mode="exact"):
        self.te = hasattr(state, "Hz")
        # symmetry cuts: TM mirrors and rotations (a live on-plane H line for the odd ones,
        # whose adjoint lines the backward pass allocates) and TE mirrors
        self.cuts = _cuts(coeffs, self.te)
        lines = tuple(n for c, n in zip(self.cuts, ("Hx0", "Hy0")) if c[0] == 2)
        self.names = (STATE_TE if self.te else STATE_TM) + lines
        self.state0, self.coeffs, self.n = state, coeffs, int(n_steps)
        self.source, self.monitors = source, list(monitors)
        self.chunk = max(1, int(chunk))
        self.sub = min(self.chunk, 64)                    # recording ring depth
        self.phase_mode = phase_mode
        self.chunks = [(s0, min(self.chunk, self.n - s0)) for s0 in range(0, self.n, self.chunk)]

    def forward(self):
        eng = Engine2D([(self.state0, self.coeffs, self.source, self.monitors)],
                       phase_mode=self.phase_mode, ring_slots=self.sub, graph=False)
        self.snaps = []
        for s0, k in self.chunks:
            self.snaps.append(eng.snapshot(0))
            eng.run(s0, k)
        st = eng.state(0)
        self.out_state = st
        self.accs = [a.clone() for a in eng.accumulators(0)]
        self.eng = eng
        return [getattr(st, f) for f in self.names] + self.accs

    def backward(self, grads):
        eng, lib = self.eng, L.load()
        it = eng.items[0]
        nx, ny = it.nx, it.ny
        P = int(eng.structs[0].pitch)
        dev = eng.device
        box = lambda: torch.zeros((nx, P), dtype=torch.float32, device=dev)  # noqa: E731
        nfld = 5 if self.te else 4
        g, gpsi, tmp = [box() for _ in range(nfld)], [box() for _ in range(4)], \
            [box() for _ in range(4)]
        geps = [box() for _ in range(2 if self.te else 1)]
        # poles: d J / d P(n), d J / d P(n-1) (zero at the end: P is not an output); TE
        # has a second set for its Ey stack
        n_p = int(eng.structs[0].n_poles)
        n_py = int(eng.structs[0].n_poles_y) if self.te else 0
        gpol = [torch.zeros((n_p * nx, P), dtype=torch.float32, device=dev) for _ in range(2)] \
            if n_p else []
        gpol_y = [torch.zeros((n_py * nx, P), dtype=torch.float32, device=dev)
                  for _ in range(2)] if n_py else []
        # live on-plane H lines (cut 2): d J / d Hx0 (nx) and d J / d Hy0 (ny), two buffers
        gcut = [[torch.zeros(n, dtype=torch.float32, device=dev) for _ in range(2)]
                if c[0] == 2 else None for c, n in zip(self.cuts, (nx, ny))]
        # magnetic poles: d J / d B (Bx, By) and d J / d M(n), M(n-1) per component
        n_m = int(eng.structs[0].n_mpoles)
        gb = [box() for _ in range(2)] if n_m else []
        gmp = [[torch.zeros((n_m * nx, P), dtype=torch.float32, device=dev) for _ in range(2)]
               for _ in range(2)] if n_m else []
        for a, name in enumerate(("Hx0", "Hy0")):     # d J / d (the final line) -> buffer 0
            if gcut[a] is not None and grads[self.names.index(name)] is not None:
                gcut[a][0].copy_(grads[self.names.index(name)].reshape(-1))
        targets = g + gpsi
        if self.te:
            offs = [(0, 0)] * 5 + [(0, 1), (1, 0), (0, 0), (0, 0)]
        else:
            yoff = 0 if self.out_state.psi_Hyx.shape[1] == ny else 1
            offs = [(0, 0)] * 6 + [(1, yoff), (1, yoff)]
        ns = len(self.names)
        for q, name in enumerate(self.names):
            gr = grads[q]
            if q >= len(targets) or gr is None or gr.numel() == 0:   # lines: seeded above
                continue
            targets[q].copy_(eng._pack(gr, nx, P, offs[q]))
        # d J / d acc in the forward regions' layout
        gaccs = []
        for q, a in enumerate(self.accs):
            gr = grads[ns + q]
            gaccs.append(torch.zeros_like(a) if gr is None
                         else gr.detach().to(torch.float32).contiguous())
        by_ptr = {L.ptr(a): q for q, a in enumerate(it.accs)}
        nreg = eng.n_regions
        regs = (L.DftRegion * max(1, nreg))()
        for r in range(nreg):
            C.memmove(C.addressof(regs[r]), C.addressof(eng.regions[r]), C.sizeof(L.DftRegion))
            regs[r].acc = L.ptr(gaccs[by_ptr[int(eng.regions[r].acc)]])
        bufs = L.Adj2DBuffers()
        for q in range(nfld):
            bufs.g[q] = L.ptr(g[q])
        for q in range(4):
            bufs.g_psi[q], bufs.tmp[q] = L.ptr(gpsi[q]), L.ptr(tmp[q])
        for q in range(len(geps)):
            bufs.g_eps[q] = L.ptr(geps[q])
        for q in range(len(gpol)):
            bufs.g_pol[q] = L.ptr(gpol[q])
        for q in range(len(gpol_y)):
            bufs.g_pol_y[q] = L.ptr(gpol_y[q])
        for a, pair in enumerate(gcut):
            for h in range(2 if pair else 0):
                bufs.g_cut[a][h] = L.ptr(pair[h])
        for c in range(len(gb)):
            bufs.g_b[c] = L.ptr(gb[c])
            for h in range(2):
                bufs.g_mpol[c][h] = L.ptr(gmp[c][h])
        adj = C.c_void_p()
        L.check(lib.mtb_yee2d_adjoint_create(C.byref(eng.structs[0]), C.byref(bufs),
                                             regs if nreg else None, nreg, eng.groups,
                                             eng.n_groups, eng.ring_elems, self.sub,
                                             C.byref(adj)), "mtb_yee2d_adjoint_create")
        keep = [gaccs, g, gpsi, tmp, geps, gpol, gpol_y, gcut, gb, gmp]
        stream = eng._sptr()
        try:
            rec_mons = _record_monitors(float(self.coeffs.dt), dev, self.te)
            zero = type(self.state0)(*[torch.zeros_like(t) if torch.is_tensor(t) else t
                                       for t in self.state0])
            rec = None

            def from_state0():      # the initial state as imported (explicit Ez honoured)
                nonlocal rec
                if rec is not None:
                    rec.close()
                rec = Engine2D([(self.state0, self.coeffs, self.source, rec_mons)],
                               phase_mode=self.phase_mode, ring_slots=self.sub, graph=False)

            def restored(snap):
                nonlocal rec
                if rec is None:
                    rec = Engine2D([(zero, self.coeffs, self.source, rec_mons)],
                                   phase_mode=self.phase_mode, ring_slots=self.sub,
                                   graph=False)
                rec.restore(0, snap)

            for c in range(len(self.chunks) - 1, -1, -1):
                s0, k = self.chunks[c]
                subs = [(s0 + o, min(self.sub, k - o)) for o in range(0, k, self.sub)]
                starts = [self.snaps[c]] + [None] * (len(subs) - 1)
                if len(subs) > 1:         # keep each sub-chunk's starting state
                    if c == 0:
                        from_state0()
                    else:
                        restored(self.snaps[c])
                    for q, (u0, uk) in enumerate(subs[:-1]):
                        rec.run(u0, uk)
                        starts[q + 1] = rec.snapshot(0)
                for q in range(len(subs) - 1, -1, -1):
                    u0, uk = subs[q]
                    if c == 0 and q == 0:
                        from_state0()
                    else:
                        restored(starts[q])
                    rec.run(u0, uk)
                    ring, selems, nslots = C.c_void_p(), C.c_int64(), C.c_int32()
                    L.check(lib.mtb_yee2d_ring(rec.plan, C.byref(ring), C.byref(selems),
                                               C.byref(nslots)), "mtb_yee2d_ring")
                    rf = rec.structs[0].ring_full
                    offs2 = (C.c_int64 * 2)(*((int(rf[1]), int(rf[2])) if self.te
                                              else (int(rf[0]), int(rf[0]))))
                    L.check(lib.mtb_yee2d_adjoint_run(adj, u0, uk, ring, selems.value, offs2,
                                                      stream), "mtb_yee2d_adjoint_run")
            if rec is not None:
                rec.close()
        finally:
            lib.mtb_yee2d_adjoint_destroy(adj)
        del keep
        if self.te:
            return (eng._unpack(geps[0], (nx - 1, ny)), eng._unpack(geps[1], (nx, ny - 1)))
        return (eng._unpack(geps[0], (nx, ny)),)

    def release(self):
        if getattr(self, "eng", None) is not None:
            self.eng.close()
            self.eng = None
        self.snaps = []


class _RunFn2D(torch.autograd.Function):
    """Inputs: the eps tensors the kernels read (TM eps_inf; TE eps_x, eps_y) and
    the runner; outputs: the final state's tensors and the accumulators."""

    @staticmethod
    def forward(ctx, runner, *eps):
        outs = runner.forward()
        ctx.runner = runner
        ctx.dtypes = [e.dtype for e in eps]
        return tuple(outs)

    @staticmethod
    def backward(ctx, *grads):
        runner = ctx.runner
        try:
            g_eps = runner.backward(grads)
        finally:
            runner.release()
        return (None,) + tuple(gr.to(dtype=dt) for gr, dt in zip(g_eps, ctx.dtypes))


def run_grad(state, coeffs, n_steps, *, source=None, monitors=(), checkpoint_every=0,
             phase_mode="exact"):
    """Differentiable run_tm / run_te: returns (state, accs) connected to the
    coefficients' eps tensors (TM eps_inf; TE eps_x, eps_y)."""
    te = hasattr(state, "Hz")
    eps_names = ("eps_x", "eps_y") if te else ("eps_inf",)
    for f in getattr(coeffs, "_fields", ()):
        t = getattr(coeffs, f)
        if torch.is_tensor(t) and t.requires_grad and f not in eps_names and f != "eps_inf":
            raise L.MtbUnsupported(f"gradients with respect to coeffs.{f} on the B200 path")
    for t in state:
        if torch.is_tensor(t) and t.requires_grad:
            raise L.MtbUnsupported("gradients with respect to the initial state on the B200 path")
    for mon in monitors:
        if getattr(mon, "reduce", "sum") != "sum":
            raise L.MtbUnsupported(f"gradients through {type(mon).__name__} (stack-reduced)")
    chunk = checkpoint_every if checkpoint_every > 0 else 32
    runner = GradRun2D(state, coeffs, n_steps, source, monitors, chunk, phase_mode)
    outs = _RunFn2D.apply(runner, *[getattr(coeffs, f) for f in eps_names])
    ns = len(runner.names)
    st = runner.out_state._replace(**dict(zip(runner.names, outs[:ns])))
    return st, list(outs[ns:])


run_tm_grad = run_grad
