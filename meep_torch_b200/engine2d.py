"""2D engine: turns the reference's state / coeffs / source / monitor objects
into one C plan (include/meep_b200.h, mtb_yee2d_*) and back.

The objects are duck-typed on the reference's interfaces so both this
package's mirror classes and the reference's own (meep_torch.core) work:

* state  -- ``TMState`` (core/stepper_tm.py:12-34) or ``TEState``
  (core/stepper_te.py:11-24): torch tensors on one CUDA device, float32.
* coeffs -- ``TMCoeffs`` / ``TECoeffs`` (core/coeffs.py:21-74, :294-344).
* source -- ``.amplitude(t)``, ``.mask``, optional ``.h_masks`` /
  ``.h_amplitude(t)`` (core/run.py:17-24, core/sources.py:49-91).
* monitors -- ``DFTFieldsMonitor`` / ``FluxMonitorTM`` / ``FluxMonitorTE`` /
  ``FluxMonitorTEY`` (core/monitors.py:24-155), reduce == "sum".

Anything outside that set raises ``MtbUnsupported`` (a NotImplementedError)
before any device work; there is no CPU or torch fallback in this module.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib as L
from ._lib import MtbUnsupported

PHASE_MODES = {"exact": 0, "reference_fp32": 1}


def _round4(n: int) -> int:
    return (n + 3) // 4 * 4


def _is_te(state) -> bool:
    return hasattr(state, "Hz") and not hasattr(state, "Ez")


def _need(cond, msg):
    if not cond:
        raise MtbUnsupported(msg)


def _opt_none(obj, names):
    for n in names:
        v = getattr(obj, n, None)
        _need(v is None or (isinstance(v, (int, bool)) and not v),
              f"{type(obj).__name__}.{n} is set: not supported by the B200 path")


def _cuts(c, te):
    """The symmetry cuts of a coefficient tuple as the struct's (cut, map, phase) per
    axis (y, x): core/coeffs.py y_mirror / x_mirror / y_rot2 / rot4 (TM) and y_mirror /
    x_mirror (TE). TM: 1 = even mirror (zero H ghost), 2 = a live on-plane H line whose
    ghost Ez is phase * Ez(partner), map 0 the cut cell, 1 reversed (Rotate2), 2 the
    other cut's transposed cell (Rotate4). TE: only the even mirror touches the step."""
    ym = int(getattr(c, "y_mirror_lo", 0) or 0)
    xm = int(getattr(c, "x_mirror_lo", 0) or 0)
    if te:
        return (1 if ym == 1 else 0, 0, 1.0), (1 if xm == 1 else 0, 0, 1.0)
    r2 = int(getattr(c, "y_rot2_lo", 0) or 0)
    r4 = int(getattr(c, "rot4_lo", 0) or 0)
    if ym == 1:
        cy = (1, 0, 1.0)
    elif ym == -1:
        cy = (2, 0, -1.0)
    elif r2:
        cy = (2, 1, float(r2))
    elif r4:
        cy = (2, 2, float(r4))
    else:
        cy = (0, 0, 1.0)
    if xm == 1:
        cx = (1, 0, 1.0)
    elif xm == -1:
        cx = (2, 0, -1.0)
    elif r4:
        cx = (2, 2, float(r4))
    else:
        cx = (0, 0, 1.0)
    return cy, cx


def _magnetic_pairs(c, pairs):
    """The magnetic pairs (h1, h2) of core/coeffs.py:161-175, :401-415, one entry per H
    component named in ``pairs``: None where they are absent or inert (h1 = 1 and h2 =
    dt, where H' = h1 H - h2 curl is the plain step), else the two tensors."""
    dt = torch.tensor(float(c.dt), dtype=torch.float32)
    out = []
    for n1, n2 in pairs:
        h1, h2 = getattr(c, n1, None), getattr(c, n2, None)
        if h1 is None and h2 is None:
            out.append(None)
            continue
        _need(h1 is not None and h2 is not None, f"magnetic pair ({n1}, {n2}) incomplete")
        inert = bool(torch.all(h1 == 1)) and \
            bool(torch.all(h2.to(torch.float32) == dt.to(h2.device)))
        out.append(None if inert else (h1, h2))
    return out


def coef_table(source, attr: str, t0: int, k: int, dt: float) -> np.ndarray:
    """FP64 per-step mask coefficients dt * amplitude(t), t = t0 .. t0+k-1.

    Known profiles of core/sources.py are evaluated vectorised in FP64 with the
    same formula; anything else calls the source's own method per step."""
    t_idx = np.arange(t0, t0 + k, dtype=np.float64)
    fn = getattr(source, attr)
    prof = getattr(source, "profile", None)
    src_dt = getattr(source, "dt", None)
    if attr == "amplitude" and prof is not None and src_dt is not None and \
            type(fn).__name__ == "method" and fn.__func__.__name__ == "amplitude" and \
            _plain_half_step(source):
        t = (t_idx + 0.5) * src_dt
        amp = _profile_vec(prof, t)
        if amp is not None:
            return dt * amp
    return np.array([dt * float(fn(int(t))) for t in range(t0, t0 + k)], dtype=np.float64)


def _plain_half_step(source) -> bool:
    # LineSource / SoftSource / PlaneSource / PointSource3D sample their profile
    # at (t_idx + 1/2) dt (core/sources.py:90-91, :116-117, monitors_3d.py:48, :66)
    return type(source).__name__ in ("LineSource", "SoftSource", "PlaneSource", "PointSource3D")


def _profile_vec(prof, t: np.ndarray):
    name = type(prof).__name__
    if name == "GaussianPulse" and hasattr(prof, "t0") and hasattr(prof, "w"):
        # core/sources.py:33-36
        d = t - prof.t0
        return np.cos(2 * math.pi * prof.fcen * d) * np.exp(-(d ** 2) / (2 * prof.w ** 2))
    if name == "CWRamp":
        # core/sources.py:44-46
        return np.sin(2 * math.pi * prof.fcen * t) * np.minimum(1.0, t / prof.t_ramp)
    if name == "ContinuousSource" and hasattr(prof, "t_ramp"):
        # core/sources.py:105-111
        ramp = (0.5 - 0.5 * np.cos(math.pi * np.minimum(1.0, t / prof.t_ramp))
                if prof.t_ramp > 0 else 1.0)
        return np.sin(2 * math.pi * prof.fcen * t) * ramp
    return None


def _cells(mask: torch.Tensor, n_rows: int, device) -> tuple:
    """CSR-by-row list of the nonzero cells of a 2D mask (rows = box rows)."""
    m = mask.detach().to(device=device, dtype=torch.float32)
    idx = torch.nonzero(m, as_tuple=False)
    if idx.numel() == 0:
        return None
    rows = idx[:, 0]
    counts = torch.bincount(rows, minlength=n_rows)
    row_ptr = torch.zeros(n_rows + 1, dtype=torch.int32, device=device)
    row_ptr[1:] = torch.cumsum(counts, 0).to(torch.int32)
    col = idx[:, 1].to(torch.int32).contiguous()
    w = m[idx[:, 0], idx[:, 1]].contiguous()
    return row_ptr, col, w


@dataclass
class _Item:
    state: object
    coeffs: object
    source: object
    monitors: list
    te: bool = False
    nx: int = 0
    ny: int = 0
    pitch: int = 0
    box: dict = field(default_factory=dict)      # name -> [buf0, buf1] or tensor
    keep: list = field(default_factory=list)     # tensors the plan points at
    accs: list = field(default_factory=list)
    stacks: list = field(default_factory=list)   # point probes: (acc index, ring offset)
    amp_col: int = -1
    hamp_col: int = -1
    src_scale: object = None     # conductivity: d2 / dt on the electric source cells


class Engine2D:
    """A batch of independent 2D structures advanced by one mtb_yee2d plan.

    ``items``: iterable of (state, coeffs, source, monitors). States are
    imported into box-layout ping-pong buffers at construction; ``run``
    advances every structure; ``state(b)`` / ``accumulators(b)`` export in
    the reference's types and shapes."""

    def __init__(self, items, *, phase_mode: str = "exact", rows_per_warp: int = 0,
                 ring_slots: int = 0, variant: int = 0, graph: bool = True, stream=None,
                 arena: bool = False):
        self.lib = L.load()
        self.use_arena = bool(arena)
        self.items = [_Item(*it) for it in items]
        _need(len(self.items) > 0, "empty batch")
        self.device = None
        self.phase_mode = PHASE_MODES[phase_mode]
        self.stream = stream
        self.t = None
        for it in self.items:
            self._validate(it)
        self._build(rows_per_warp, ring_slots, variant, graph)

    # ---------------------------------------------------------------- import
    def _validate(self, it: _Item):
        s, c = it.state, it.coeffs
        it.te = _is_te(s)
        main = s.Hz if it.te else s.Ez
        _need(isinstance(main, torch.Tensor) and main.is_cuda,
              "state tensors must be CUDA tensors (the B200 path has no CPU mode)")
        _need(main.dtype == torch.float32, f"state dtype {main.dtype}: the B200 path computes "
              "in float32 (convert the grid to float32)")
        if self.device is None:
            self.device = main.device
        _need(main.device == self.device, "all structures of a batch must share one device")
        if it.te:
            it.nx, it.ny = main.shape[0] + 1, main.shape[1] + 1
            for n_, cn in ((s.Px_cur.shape[0], "c1x"), (s.Py_cur.shape[0], "c1y")):
                _need(n_ <= L.MTB_MAX_POLES, f"{n_} dispersive poles (at most {L.MTB_MAX_POLES})")
                _need(getattr(c, cn).shape[0] == n_, f"pole coefficients {cn} count")
            # in-plane tensor eps / oriented poles: the three-pass TE kernels
            it.te3 = (getattr(c, "inv_xx_x", None) is not None or
                      getattr(c, "c3xy", None) is not None)
            it.mag = _magnetic_pairs(c, [("hz1", "hz2")])
        else:
            it.nx, it.ny = main.shape
            np_ = s.P_cur.shape[0]
            _need(np_ <= L.MTB_MAX_POLES, f"{np_} dispersive poles (at most {L.MTB_MAX_POLES})")
            _need(tuple(c.c1.shape) == (np_, it.nx, it.ny), "pole coefficients c1 shape")
            it.n_mp = 0 if getattr(c, "mc1x", None) is None else int(c.mc1x.shape[0])
            _need((getattr(s, "Bx", None) is None) == (it.n_mp == 0),
                  "TMState.Bx and the coefficients' magnetic poles must come together")
            _need(it.n_mp <= L.MTB_MAX_POLES,
                  f"{it.n_mp} magnetic poles (at most {L.MTB_MAX_POLES})")
            if it.n_mp:
                _need(tuple(s.Mx_cur.shape[:1]) == (it.n_mp,), "TMState.Mx_cur pole count")
            it.mag = _magnetic_pairs(c, [("h1x", "h2x"), ("h1y", "h2y")])
        it.cuts = _cuts(c, it.te)
        if not it.te:
            # the live on-plane H lines of the cuts (init_tm_state Hx0 / Hy0)
            for (cut, _, _), name, n in ((it.cuts[0], "Hx0", it.nx), (it.cuts[1], "Hy0", it.ny)):
                h0 = getattr(s, name, None)
                _need((cut == 2) == (h0 is not None),
                      f"TMState.{name} does not match the coefficients' symmetry cut")
                _need(h0 is None or tuple(h0.shape) == (n,), f"TMState.{name} shape")
        # instantaneous chi2 / chi3: TM on the tile kernels (core/stepper_tm.py:222-230)
        it.nl = bool(getattr(c, "has_kerr", False) or getattr(c, "has_chi2", False))
        if it.nl and it.te:
            # TE chi2 / chi3: Jacobi sweeps on the three-pass kernels (scalar eps only)
            _need(getattr(c, "inv_xx_x", None) is None, "TE chi2 / chi3 with the tensor eps")
            it.te3 = True
        for k in ("k_hx", "k_hy", "k_ex", "k_ey"):
            kv = getattr(c, k)
            _need(bool(torch.all(kv == 1)), f"CPML kappa != 1 ({k})")
        for mon in it.monitors:
            red = getattr(mon, "reduce", "sum")
            _need(red == "sum" or (red == "stack" and hasattr(mon, "ix") and hasattr(mon, "iy")),
                  f"{type(mon).__name__}: only sum-reduced monitors and point probes run on "
                  "the B200 path")
        it.pitch = _round4(it.ny)

    def _pack(self, src: torch.Tensor, nx, pitch, off=(0, 0)) -> torch.Tensor:
        box = torch.empty((nx, pitch), dtype=torch.float32, device=self.device)
        src = src.detach().to(dtype=torch.float32).contiguous()
        n0, n1 = (src.shape[0], src.shape[1]) if src.dim() == 2 else (0, 0)
        L.check(self.lib.mtb_pack(L.ptr(src) if src.numel() else 0, n0, n1, 1, n1, 1,
                                  L.ptr(box), nx, pitch, 1, pitch, 1, off[0], off[1], 0,
                                  self._sptr()), "pack")
        return box

    def _pack_stack(self, t3, nx, pitch):
        """A (n, r, c) stack of planes -> (n * nx, pitch) box planes, plane k at rows
        k * nx (each plane in the box layout of an nx-row array)."""
        n = t3.shape[0]
        box = torch.zeros((n * nx, pitch), dtype=torch.float32, device=self.device)
        for k in range(n):
            box[k * nx:(k + 1) * nx].copy_(self._pack(t3[k], nx, pitch))
        return box

    def _unpack_stack(self, box, n, nx, shape):
        return torch.stack([self._unpack(box[k * nx:(k + 1) * nx], shape) for k in range(n)]) \
            if n else torch.zeros((0, *shape), dtype=torch.float32, device=self.device)

    def _pair(self, src, nx, pitch, off=(0, 0)):
        a = self._pack(src, nx, pitch, off)
        return [a, a.clone()]

    def _sptr(self):
        st = self.stream if self.stream is not None else torch.cuda.current_stream(self.device)
        return st.cuda_stream

    def _profiles(self, it: _Item):
        c, nx, ny = it.coeffs, it.nx, it.ny
        dev = self.device

        def flat(t):
            return t.detach().reshape(-1).to(device=dev, dtype=torch.float32).contiguous()

        def node(b, a, n):
            # interior-sliced node profile -> full n nodes; walls inert (b=1, a=0)
            b, a = flat(b), flat(a)
            fb = torch.ones(n, dtype=torch.float32, device=dev)
            fa = torch.zeros(n, dtype=torch.float32, device=dev)
            if b.numel() == n:
                fb.copy_(b); fa.copy_(a)
            elif b.numel() == n - 2:
                fb[1:-1] = b; fa[1:-1] = a
            elif b.numel() == n - 1 and not it.te:
                fb[:-1] = b; fa[:-1] = a                  # from the cut row (TM cuts)
            else:
                raise MtbUnsupported(f"unexpected CPML profile length {b.numel()} for n={n}")
            return fb, fa

        hx = (flat(c.b_hx), flat(c.a_hx))
        hy = (flat(c.b_hy), flat(c.a_hy))
        _need(hx[0].numel() == nx - 1 and hy[0].numel() == ny - 1, "CPML half-node profile length")
        ex = node(c.b_ex, c.a_ex, nx)
        ey = node(c.b_ey, c.a_ey, ny)
        it.keep += [*hx, *hy, *ex, *ey]
        return hx, hy, ex, ey

    def _build(self, rows_per_warp, ring_slots, variant=0, graph=True):
        lib = self.lib
        dev = self.device
        structs = (L.Yee2DStruct * len(self.items))()
        regions, groups, group_key = [], [], {}
        ring = 0
        amp_cols = 0
        self._amp_sources = []      # (column, source, attr, dt)
        col_of = {}

        def group(freqs, dt):
            f = tuple(float(x) for x in torch.as_tensor(freqs).detach().reshape(-1).cpu()
                      .to(torch.float64).tolist())
            key = (f, float(dt))
            if key not in group_key:
                arr = (C.c_double * len(f))(*f)
                group_key[key] = len(groups)
                groups.append((arr, len(f), float(dt)))
            return group_key[key], len(f)

        def alloc_ring(n):
            nonlocal ring
            off = ring
            ring += _round4(n)
            return off

        for b, it in enumerate(self.items):
            s, c, te = it.state, it.coeffs, it.te
            nx, ny, P = it.nx, it.ny, it.pitch
            S = structs[b]
            S.pol = L.MTB_TE if te else L.MTB_TM
            S.nx, S.ny, S.pitch = nx, ny, P
            S.y_pmc = 1 if (not te and getattr(c, "y_pmc", False)) else 0
            S.dt, S.dx = float(c.dt), float(c.dx)
            eps_b = None
            pol_bufs = None
            if te:
                f_main, f_x, f_y = self._pair(s.Hz, nx, P), self._pair(s.Dx, nx, P), \
                    self._pair(s.Dy, nx, P)
                eps_a = self._pack(c.eps_x, nx, P)
                eps_b = self._pack(c.eps_y, nx, P)
                inv_a = self._pack(torch.reciprocal(c.eps_x.to(torch.float32)), nx, P)
                inv_b = self._pack(torch.reciprocal(c.eps_y.to(torch.float32)), nx, P)
                psis = [self._pair(s.psi_Hzy, nx, P, (0, 1)), self._pair(s.psi_Hzx, nx, P, (1, 0)),
                        self._pair(s.psi_Eyx, nx, P), self._pair(s.psi_Exy, nx, P)]
                S.inv_eps_b = L.ptr(inv_b)
                it.keep += [eps_b, inv_b]
                # dispersive poles on Ex and Ey (core/stepper_te.py:136-175)
                pol_bufs = {}
                for ax, (pcur, pprev, cs) in enumerate(
                        ((s.Px_cur, s.Px_prev, ("c1x", "c2x", "c3x")),
                         (s.Py_cur, s.Py_prev, ("c1y", "c2y", "c3y")))):
                    n_p = pcur.shape[0]
                    if not n_p:
                        continue
                    # three rotating buffers: P(n) in slot 0, P(n-1) in slot 2
                    pp = [self._pack_stack(pcur, nx, P), None, self._pack_stack(pprev, nx, P)]
                    pp[1] = torch.zeros_like(pp[0])
                    pc = [self._pack_stack(getattr(c, k), nx, P) for k in cs]
                    for k in range(3):
                        if ax == 0:
                            S.pol_p[k], S.pol_c[k] = L.ptr(pp[k]), L.ptr(pc[k])
                        else:
                            S.pol_py[k], S.pol_cy[k] = L.ptr(pp[k]), L.ptr(pc[k])
                    if ax == 0:
                        S.n_poles = n_p
                    else:
                        S.n_poles_y = n_p
                    pol_bufs["x" if ax == 0 else "y"] = pp
                    it.keep += pp + pc
                pol_bufs = pol_bufs or None
                if it.te3:
                    # E is kept between steps (core/stepper_te.py:150-175)
                    ebx, eby = self._pack(s.Ex, nx, P), self._pack(s.Ey, nx, P)
                    S.te3, S.e_x, S.e_y = 1, L.ptr(ebx), L.ptr(eby)
                    it.keep += [ebx, eby]
                    if getattr(c, "inv_xx_x", None) is not None:
                        tv = [self._pack(getattr(c, k), nx, P)
                              for k in ("inv_xx_x", "inv_xy_x", "inv_yy_y", "inv_xy_y")]
                        for k in range(4):
                            S.tinv[k] = L.ptr(tv[k])
                        it.keep += tv
                    for name, attr in (("c3xy", "c3xy"), ("c3yx", "c3yx")):
                        v = getattr(c, name, None)
                        if v is not None:
                            st_ = self._pack_stack(v, nx, P)
                            setattr(S, attr, L.ptr(st_))
                            it.keep.append(st_)
                    it.te3_box = (ebx, eby)
                    if it.nl:
                        z2 = torch.zeros_like(c.eps_x)
                        nlb = [self._pack(v, nx, P) for v in
                               (c.chi2_x if c.chi2_x is not None else z2, c.chi3_x, c.eps_x,
                                c.chi2_y if c.chi2_y is not None else torch.zeros_like(c.eps_y),
                                c.chi3_y, c.eps_y)]
                        et = [torch.zeros((nx, P), dtype=torch.float32, device=dev)
                              for _ in range(2)]
                        for k in range(3):
                            S.nlx[k], S.nly[k] = L.ptr(nlb[k]), L.ptr(nlb[3 + k])
                        S.e_t[0], S.e_t[1] = L.ptr(et[0]), L.ptr(et[1])
                        it.keep += nlb + et
            else:
                f_main, f_x, f_y = self._pair(s.Dz, nx, P), self._pair(s.Hx, nx, P), \
                    self._pair(s.Hy, nx, P)
                eps_a = self._pack(c.eps_inf, nx, P)
                inv_a = self._pack(torch.reciprocal(c.eps_inf.to(torch.float32)), nx, P)
                # the E-side CPML memory covers the interior, or from the cut row /
                # column (symmetry cuts), or every column (y PMC)
                xoff = 1 if s.psi_Hyx.shape[0] == nx - 2 else 0
                yoff = 1 if s.psi_Hyx.shape[1] == ny - 2 else 0
                psis = [self._pair(s.psi_Ezy, nx, P), self._pair(s.psi_Ezx, nx, P),
                        self._pair(s.psi_Hyx, nx, P, (xoff, yoff)),
                        self._pair(s.psi_Hxy, nx, P, (xoff, yoff))]
                # dispersive poles: P planes (ping-pong) and c1, c2, c3
                # (core/stepper_tm.py:203-231)
                n_p = s.P_cur.shape[0]
                S.n_poles = n_p
                psum = 0.0
                if n_p:
                    # three rotating buffers: P(n) in slot 0, P(n-1) in slot 2
                    pp = [self._pack(s.P_cur.reshape(n_p * nx, ny), n_p * nx, P), None,
                          self._pack(s.P_prev.reshape(n_p * nx, ny), n_p * nx, P)]
                    pp[1] = torch.zeros_like(pp[0])
                    pc = [self._pack(getattr(c, k).reshape(n_p * nx, ny), n_p * nx, P)
                          for k in ("c1", "c2", "c3")]
                    for k in range(3):
                        S.pol_p[k], S.pol_c[k] = L.ptr(pp[k]), L.ptr(pc[k])
                    pol_bufs = pp
                    it.keep += pp + pc
                    psum = s.P_cur.sum(0)
                # Ez is normally (Dz - sum P)/eps exactly (update_eh); an imported
                # state where it is not is honoured on the first step
                ez_ref = (s.Dz - psum) / c.eps_inf.to(s.Dz.dtype)
                if not torch.equal(ez_ref, s.Ez):
                    eex = self._pack(s.Ez, nx, P)
                    S.explicit_e = 1
                    S.e_explicit = L.ptr(eex)
                    it.keep.append(eex)
            it.box = dict(main=f_main, x=f_x, y=f_y, psi=psis, eps_a=eps_a, eps_b=eps_b,
                          inv_a=inv_a)
            (S.cut_y, S.cut_map_y, S.cut_ph_y), (S.cut_x, S.cut_map_x, S.cut_ph_x) = it.cuts
            for name, attr in (("Hx0", "f_x0"), ("Hy0", "f_y0")):
                h0 = None if te else getattr(s, name, None)
                if h0 is None:
                    continue
                buf = torch.zeros((2, _round4(h0.shape[0])), dtype=torch.float32, device=dev)
                buf[:, :h0.shape[0]] = h0.detach().to(device=dev, dtype=torch.float32)
                getattr(S, attr)[0], getattr(S, attr)[1] = L.ptr(buf[0]), L.ptr(buf[1])
                it.box[name] = buf
                it.keep.append(buf)
            if pol_bufs is not None:
                if te:
                    for ax, bufs in pol_bufs.items():
                        it.box["pol_" + ax] = bufs
                else:
                    it.box["pol"] = pol_bufs
            it.keep += [*f_main, *f_x, *f_y, eps_a] + [t for p in psis for t in p]
            S.f_main[0], S.f_main[1] = L.ptr(f_main[0]), L.ptr(f_main[1])
            S.f_x[0], S.f_x[1] = L.ptr(f_x[0]), L.ptr(f_x[1])
            S.f_y[0], S.f_y[1] = L.ptr(f_y[0]), L.ptr(f_y[1])
            S.inv_eps_a = L.ptr(inv_a)
            it.keep.append(inv_a)
            for k in range(4):
                S.psi[k][0], S.psi[k][1] = L.ptr(psis[k][0]), L.ptr(psis[k][1])
            # electric conductivity (sigma_d): D' = d1 D + d2 curl H, and the soft
            # current on D scaled by d2 (core/stepper_tm.py:158-163, :197-200;
            # core/stepper_te.py D update and step_source)
            it.src_scale = None
            it.plain = (not te and not S.n_poles and not S.explicit_e and not (S.cut_y or S.cut_x)
                        and not it.nl)
            if not te and it.n_mp:
                # magnetic Lorentz poles: B pairs, M stacks (M(n) in slot 0, M(n-1) in
                # slot 2, as the electric poles) and mc1..mc3
                nm = it.n_mp
                S.n_mpoles = nm
                fb = [self._pair(s.Bx, nx, P), self._pair(s.By, nx, P)]
                mstk = []
                for c_, (cur, prev, cs) in enumerate(
                        ((s.Mx_cur, s.Mx_prev, ("mc1x", "mc2x", "mc3x")),
                         (s.My_cur, s.My_prev, ("mc1y", "mc2y", "mc3y")))):
                    mm = [self._pack_stack(cur, nx, P), None, self._pack_stack(prev, nx, P)]
                    mm[1] = torch.zeros_like(mm[0])
                    mc = [self._pack_stack(getattr(c, k), nx, P) for k in cs]
                    for b in range(2):
                        S.f_b[c_][b] = L.ptr(fb[c_][b])
                    for k in range(3):
                        S.mpol[c_][k], S.mpc[c_][k] = L.ptr(mm[k]), L.ptr(mc[k])
                    mstk.append(mm)
                    it.keep += fb[c_] + mm + mc
                it.box["B"], it.box["M"] = fb, mstk
                it.plain = False
            if it.nl and not te:
                x2 = self._pack(c.chi2 if c.chi2 is not None else torch.zeros_like(c.eps_inf),
                                nx, P)
                x3 = self._pack(c.chi3, nx, P)
                S.chi2, S.chi3, S.eps_nl = L.ptr(x2), L.ptr(x3), L.ptr(eps_a)
                it.keep += [x2, x3]
            cond = ([("d1x", "d2x"), ("d1y", "d2y")] if te else [("d1", "d2")])
            if getattr(c, cond[0][0], None) is not None:
                for k, (n1, n2) in enumerate(cond):
                    b1 = self._pack(getattr(c, n1), nx, P)
                    b2 = self._pack(getattr(c, n2), nx, P)
                    S.cond_d1[k], S.cond_d2[k] = L.ptr(b1), L.ptr(b2)
                    it.keep += [b1, b2]
                it.plain = False
                d2e = getattr(c, cond[-1][1])
                it.src_scale = d2e.to(device=dev, dtype=torch.float32) / float(c.dt)
            # magnetic conductivity / permeability: H' = h1 H -/+ h2 curl
            # (core/stepper_tm.py:121-125, core/stepper_te.py:112-114)
            for k, pr in enumerate(it.mag):
                if pr is None:
                    continue
                b1, b2 = self._pack(pr[0], nx, P), self._pack(pr[1], nx, P)
                S.mag_h1[k], S.mag_h2[k] = L.ptr(b1), L.ptr(b2)
                it.keep += [b1, b2]
                it.plain = False
            self._check_psi_outside(it)
            hx, hy, ex, ey = self._profiles(it)
            S.hx_b, S.hx_a = L.ptr(hx[0]), L.ptr(hx[1])
            S.hy_b, S.hy_a = L.ptr(hy[0]), L.ptr(hy[1])
            S.ex_b, S.ex_a = L.ptr(ex[0]), L.ptr(ex[1])
            S.ey_b, S.ey_a = L.ptr(ey[0]), L.ptr(ey[1])

            # ---- sources
            src = it.source
            if src is not None:
                mask = getattr(src, "mask", None)
                if mask is not None:
                    want = (nx, ny - 1) if te else (nx, ny)
                    _need(tuple(mask.shape) == want,
                          f"source mask shape {tuple(mask.shape)} != {want}")
                    if it.src_scale is not None:
                        # the plan subtracts (dt amp) w; under conductivity the
                        # reference subtracts d2 amp mask
                        mask = mask.to(device=dev, dtype=torch.float32) * it.src_scale
                    cl = _cells(mask, nx, dev)
                    if cl is not None:
                        it.amp_col = col_of.setdefault((id(src), "amplitude"), amp_cols)
                        if it.amp_col == amp_cols:
                            amp_cols += 1
                            self._amp_sources.append((it.amp_col, src, "amplitude", float(c.dt), "e"))
                        self._set_cells(S.src_e, cl, it.amp_col, it)
                h_masks = getattr(src, "h_masks", None) or {}
                if h_masks:
                    key = (id(src), "h_amplitude")
                    hcol = col_of.setdefault(key, amp_cols)
                    if hcol == amp_cols:
                        amp_cols += 1
                        self._amp_sources.append((hcol, src, "h_amplitude", float(c.dt), "h"))
                    for name, m in h_masks.items():
                        if m is None:
                            continue
                        if te:
                            _need(name == "src_hz_mask", f"TE magnetic source {name}")
                            _need(tuple(m.shape) == (nx - 1, ny - 1), "src_hz_mask shape")
                            target = S.src_h1
                        elif name == "src_hy_mask":
                            _need(tuple(m.shape) == (nx - 1, ny), "src_hy_mask shape")
                            target = S.src_h1
                        elif name == "src_hx_mask":
                            _need(tuple(m.shape) == (nx, ny - 1), "src_hx_mask shape")
                            target = S.src_h2
                        else:
                            raise MtbUnsupported(f"magnetic source {name}")
                        cl = _cells(m, nx, dev)
                        if cl is not None:
                            self._set_cells(target, cl, hcol, it)

            # ---- monitors
            lines = []
            ring_full = [-1, -1, -1]
            it.accs = []
            it.stacks = []                   # (monitor index, ring offset) of point probes
            for mon in it.monitors:
                kind = type(mon).__name__
                if getattr(mon, "reduce", "sum") == "stack":
                    # a point probe (core/monitors.py:11-21): Ez of one node, one value
                    # per step (stack-reduced, core/run.py:28-38)
                    _need(not te, f"{kind} samples Ez: a TM state")
                    ix, iy = int(mon.ix), int(mon.iy)
                    _need(0 <= ix < nx and 0 <= iy < ny, f"{kind} at ({ix}, {iy}) outside the grid")
                    o = alloc_ring(1)
                    lines.append((L.C2_MAIN, 0, ix, iy, iy + 1, o))
                    it.stacks.append((len(it.accs), o))
                    it.accs.append(torch.zeros(0, dtype=torch.float32, device=dev))
                    continue
                g, nf = group(mon.freqs, mon.dt)
                if kind == "DFTFieldsMonitor":
                    comp = mon.component
                    names = ("Hz", "Ex", "Ey") if te else ("Ez", "Hx", "Hy")
                    _need(comp in names, f"DFTFieldsMonitor on {comp}")
                    ci = names.index(comp)
                    shp = {"Ez": (nx, ny), "Hx": (nx, ny - 1), "Hy": (nx - 1, ny),
                           "Hz": (nx - 1, ny - 1), "Ex": (nx - 1, ny), "Ey": (nx, ny - 1)}[comp]
                    if ring_full[ci] < 0:
                        ring_full[ci] = alloc_ring(nx * P)
                    acc = torch.zeros((nf, 2) + shp, dtype=torch.float32, device=dev)
                    n = shp[0] * shp[1]
                    regions.append(self._region(acc, 0, n, 2 * n, ring_full[ci], -1, shp[0],
                                                shp[1], P, shp[1], g,
                                                2 if comp.startswith("E") else 1))
                elif kind in ("FluxMonitorTM", "FluxMonitorTE", "FluxMonitorTEY"):
                    lo, hi = int(mon.lo), int(mon.hi)
                    Ln = hi - lo
                    _need(Ln > 0, "empty flux line")
                    if kind == "FluxMonitorTM":
                        _need(not te, "FluxMonitorTM on a TE state")
                        idx = int(mon.idx)
                        if mon.x_normal:      # Ez row idx; Hy rows idx-1, idx
                            e_line = (L.C2_MAIN, 0, idx)
                            h_lines = [(L.C2_Y, 0, idx - 1), (L.C2_Y, 0, idx)]
                        else:                 # Ez column idx; Hx columns idx-1, idx
                            e_line = (L.C2_MAIN, 1, idx)
                            h_lines = [(L.C2_X, 1, idx - 1), (L.C2_X, 1, idx)]
                        toff_e, toff_h = 2, 1
                    elif kind == "FluxMonitorTE":
                        _need(te, "FluxMonitorTE on a TM state")
                        idx = int(mon.ix)     # Ey row ix; Hz rows ix-1, ix
                        e_line = (L.C2_Y, 0, idx)
                        h_lines = [(L.C2_MAIN, 0, idx - 1), (L.C2_MAIN, 0, idx)]
                        toff_e, toff_h = 1, 2
                    else:
                        _need(te, "FluxMonitorTEY on a TM state")
                        idx = int(mon.iy)     # Ex column iy; Hz columns iy-1, iy
                        e_line = (L.C2_X, 1, idx)
                        h_lines = [(L.C2_MAIN, 1, idx - 1), (L.C2_MAIN, 1, idx)]
                        toff_e, toff_h = 1, 2
                    offs = []
                    for comp, kd, index in [e_line] + h_lines:
                        o = alloc_ring(Ln)
                        lines.append((comp, kd, index, lo, hi, o))
                        offs.append(o)
                    acc = torch.zeros((nf, 4, Ln), dtype=torch.float32, device=dev)
                    regions.append(self._region(acc, 0, Ln, 4 * Ln, offs[0], -1, 1, Ln, Ln, Ln,
                                                g, toff_e))
                    regions.append(self._region(acc, 2 * Ln, 3 * Ln, 4 * Ln, offs[1], offs[2], 1,
                                                Ln, Ln, Ln, g, toff_h))
                else:
                    raise MtbUnsupported(f"monitor {kind}")
                it.accs.append(acc)
                it.keep.append(acc)
            _need(len(lines) <= 16, "more than 16 monitor lines on one structure")
            if lines:
                arr = (L.LineSample * len(lines))()
                for q, (comp, kd, index, lo, hi, o) in enumerate(lines):
                    arr[q].comp, arr[q].kind, arr[q].index = comp, kd, index
                    arr[q].lo, arr[q].hi, arr[q].ring_off = lo, hi, o
                raw = torch.frombuffer(bytearray(bytes(arr)), dtype=torch.uint8).to(dev)
                it.keep.append(raw)
                S.lines = L.ptr(raw)
                S.n_lines = len(lines)
            for ci in range(3):
                S.ring_full[ci] = ring_full[ci]

        self.n_amp_cols = amp_cols
        self.ring_elems = ring
        reg_arr = (L.DftRegion * max(1, len(regions)))(*regions) if regions else None
        grp_arr = (L.PhaseGroup * max(1, len(groups)))()
        for q, (arr, nf, dt) in enumerate(groups):
            grp_arr[q].freqs = C.cast(arr, C.POINTER(C.c_double))
            grp_arr[q].nf, grp_arr[q].mode, grp_arr[q].dt = nf, self.phase_mode, dt
        self._groups = groups
        self.regions = reg_arr           # host descriptors the plan was built from
        self.n_regions = len(regions)
        self.groups = grp_arr
        self.n_groups = len(groups)
        if self.use_arena:
            self._make_arena(structs)
        tun = L.Tuning(rows_per_warp, ring_slots, 0 if graph else -1, variant)
        plan = C.c_void_p()
        L.check(lib.mtb_yee2d_plan_create(structs, len(self.items), reg_arr, len(regions),
                                          grp_arr, len(groups), ring, amp_cols, C.byref(tun),
                                          C.byref(plan)), "mtb_yee2d_plan_create")
        self.plan = plan
        self.structs = structs

    def _make_arena(self, structs):
        """Move every structure's stepped fields (main, x, y, the four CPML memories and
        the on-plane cut lines) into one flat buffer per parity, ``self.arena`` (2, n):
        structure b owns ``arena[p, it.arena_off : it.arena_off + it.arena_len]``, its
        arrays back to back in that order (``it.arena_segs``: name, offset, shape). A
        caller can then read or write a whole state with one copy (the CW operator's
        Krylov vectors live in this layout). Pole stacks stay outside (they rotate
        through three buffers)."""
        segs, total = [], 0
        for b, it in enumerate(self.items):
            bx = it.box
            lst = [("main", bx["main"]), ("x", bx["x"]), ("y", bx["y"])]
            lst += [(f"psi{k}", bx["psi"][k]) for k in range(4)]
            lst += [(n, [bx[n][0], bx[n][1]]) for n in ("Hx0", "Hy0") if n in bx]
            it.arena_off, it.arena_segs = total, []
            for name, pair in lst:
                segs.append((it, name, pair, total))
                it.arena_segs.append((name, total, tuple(pair[0].shape)))
                total += pair[0].numel()
            it.arena_len = total - it.arena_off
        arena = torch.zeros((2, total), dtype=torch.float32, device=self.device)
        remap = {}
        for it, name, pair, off in segs:
            views = []
            for p in range(2):
                v = arena[p, off:off + pair[p].numel()].view(pair[p].shape)
                v.copy_(pair[p])
                remap[L.ptr(pair[p])] = L.ptr(v)
                views.append(v)
            if name.startswith("psi"):
                it.box["psi"][int(name[3])] = views
            else:
                it.box[name] = views
        for S in structs:
            for arr in (S.f_main, S.f_x, S.f_y, S.f_x0, S.f_y0, *S.psi):
                for p in range(2):
                    if arr[p]:
                        arr[p] = remap.get(arr[p], arr[p])
        self.arena = arena

    def _set_cells(self, target, cl, col, it):
        row_ptr, colv, w = cl
        it.keep += [row_ptr, colv, w]
        target.row_ptr, target.col, target.w = L.ptr(row_ptr), L.ptr(colv), L.ptr(w)
        target.n, target.amp_col = int(colv.numel()), col

    @staticmethod
    def _region(acc, re_off, im_off, f_stride, ring_a, ring_b, rows, cols, ring_pitch,
                acc_pitch, grp, toff):
        r = L.DftRegion()
        r.acc = L.ptr(acc)
        r.re_off, r.im_off, r.f_stride = re_off, im_off, f_stride
        r.ring_a, r.ring_b = ring_a, ring_b
        r.rows, r.cols, r.ring_pitch, r.acc_pitch = rows, cols, ring_pitch, acc_pitch
        r.group, r.toff = grp, toff
        return r

    def _check_psi_outside(self, it: _Item):
        """CPML memory must vanish where its profile is inert (b == 1, a == 0):
        the kernels never touch it there (the reference keeps it at zero)."""
        c = it.coeffs

        def inert(b, a):
            return (b.detach().reshape(-1) == 1) & (a.detach().reshape(-1) == 0)

        s = it.state
        if it.te:
            checks = [(s.psi_Hzy, None, inert(c.b_ey, c.a_ey)), (s.psi_Hzx, inert(c.b_ex, c.a_ex), None),
                      (s.psi_Eyx, inert(c.b_hx, c.a_hx), None), (s.psi_Exy, None, inert(c.b_hy, c.a_hy))]
        else:
            checks = [(s.psi_Ezy, None, inert(c.b_hy, c.a_hy)), (s.psi_Ezx, inert(c.b_hx, c.a_hx), None),
                      (s.psi_Hyx, inert(c.b_ex, c.a_ex), None), (s.psi_Hxy, None, inert(c.b_ey, c.a_ey))]
        for psi, rows, cols in checks:
            if psi.numel() == 0:
                continue
            m = psi != 0
            if rows is not None:
                m = m & rows.to(psi.device)[:, None]
            if cols is not None:
                m = m & cols.to(psi.device)[None, :]
            _need(not bool(m.any()), "CPML memory is nonzero outside its absorbing layer")

    # ------------------------------------------------------------------ run
    def run(self, t0: int, k: int):
        """Advance every structure k steps starting at step index t0. Point probes
        (stack-reduced) hold the k values of this call afterwards."""
        self._checked = False
        if k <= 0:
            return
        if any(it.stacks for it in self.items):
            self._run_stacked(t0, k)
            return
        self._run(t0, k)

    def _run_stacked(self, t0: int, k: int):
        """Run in pieces of one ring flush and copy the probes' samples out after each:
        the ring holds the samples of the last flush only."""
        lib = self.lib
        ring, selems, nslots = C.c_void_p(), C.c_int64(), C.c_int32()
        L.check(lib.mtb_yee2d_ring(self.plan, C.byref(ring), C.byref(selems), C.byref(nslots)),
                "mtb_yee2d_ring")
        G = int(nslots.value)
        offs, where = [], []
        for b, it in enumerate(self.items):
            for q, o in it.stacks:
                where.append((b, q))
                offs.append(o)
        off_d = torch.tensor(offs, dtype=torch.int64, device=self.device)
        out = torch.empty((k, len(offs)), dtype=torch.float32, device=self.device)
        s = 0
        while s < k:
            n = min(G, k - s)
            self._run(t0 + s, n)
            L.check(lib.mtb_yee2d_ring_gather(self.plan, L.ptr(off_d), len(offs), n,
                                              L.ptr(out[s:]), self._sptr()),
                    "mtb_yee2d_ring_gather")
            s += n
        for j, (b, q) in enumerate(where):
            self.items[b].accs[q] = out[:, j].clone()

    def _run(self, t0: int, k: int):
        nc = max(self.n_amp_cols, 1)
        ce = np.zeros((k, nc), dtype=np.float64)
        ch = np.zeros((k, nc), dtype=np.float64)
        have_e = have_h = False
        for col, src, attr, dt, kind in self._amp_sources:
            v = coef_table(src, attr, t0, k, dt)
            if kind == "e":
                ce[:, col] = v
                have_e = True
            else:
                ch[:, col] = v
                have_h = True
        pe = ce.ctypes.data_as(C.POINTER(C.c_double)) if have_e else None
        ph = ch.ctypes.data_as(C.POINTER(C.c_double)) if have_h else None
        L.check(self.lib.mtb_yee2d_run(self.plan, t0, k, pe, ph, self._sptr()), "mtb_yee2d_run")
        self.last_launches = self.lib.mtb_yee2d_last_launches(self.plan)

    def reset(self):
        """Zero every field, CPML and accumulator buffer (both ping-pong halves)
        with the library's own fill kernel -- a fresh t = 0 run of the same batch."""
        for it in self.items:
            bufs = [*it.box["main"], *it.box["x"], *it.box["y"]] + \
                [t for p in it.box["psi"] for t in p] + list(it.accs) + \
                list(it.box.get("pol", [])) + list(it.box.get("pol_x", [])) + \
                list(it.box.get("pol_y", []))
            for t in bufs:
                n = t.numel()
                if n == 0:
                    continue
                L.check(self.lib.mtb_pack(0, 0, 0, 0, 0, 0, L.ptr(t), 1, 1, n, n, n, 0, 0, 0,
                                          self._sptr()), "reset")

    def set_eps(self, b: int, eps: torch.Tensor):
        """Replace structure b's permittivity in place (a TM structure without
        conductivity, poles or an explicit first-step Ez): eps and 1/eps are packed
        into the plan's own buffers, so a batch of new designs of the same shapes
        reuses the plan (and its graphs); call reset() before the next run."""
        it = self.items[b]
        _need(getattr(it, "plain", False), "set_eps: TM structures without conductivity, "
              "poles or an explicit first-step Ez only")
        _need(tuple(eps.shape) == (it.nx, it.ny), f"set_eps: eps shape {tuple(eps.shape)} "
              f"!= {(it.nx, it.ny)}")
        e = eps.to(device=self.device, dtype=torch.float32)
        it.box["eps_a"].copy_(self._pack(e, it.nx, it.pitch))
        it.box["inv_a"].copy_(self._pack(torch.reciprocal(e), it.nx, it.pitch))

    def _live_buffers(self, b: int):
        """The buffers of structure b the next step reads: fields, CPML memory, pole
        stacks, the live on-plane H lines of symmetry cuts, and B with the magnetic pole
        stacks."""
        it, cur = self.items[b], self.current
        pols = [it.box[k] for k in ("pol", "pol_x", "pol_y") if k in it.box]
        ps = self.pole_slot
        return [it.box["main"][cur], it.box["x"][cur], it.box["y"][cur]] + \
            [p[cur] for p in it.box["psi"]] + \
            [b for pol in pols for b in (pol[ps], pol[(ps + 2) % 3])] + \
            [it.box[n][cur] for n in ("Hx0", "Hy0") if n in it.box] + \
            [fb[cur] for fb in it.box.get("B", ())] + \
            [b for m in it.box.get("M", ()) for b in (m[ps], m[(ps + 2) % 3])]

    def snapshot(self, b: int = 0):
        """Copy of structure b's live state (box layout) for restore()."""
        return [t.clone() for t in self._live_buffers(b)]

    def restore(self, b: int, snap):
        """Make a snapshot() structure b's live state again (t_idx is the caller's)."""
        for dst, src in zip(self._live_buffers(b), snap):
            dst.copy_(src)

    def set_timing(self, on: bool = True):
        L.check(self.lib.mtb_yee2d_set_timing(self.plan, 1 if on else 0), "set_timing")

    def timing(self):
        """(step_ms, step_launches, dft_ms, dft_launches) since set_timing(True)."""
        a, b, c, d = C.c_double(), C.c_int64(), C.c_double(), C.c_int64()
        L.check(self.lib.mtb_yee2d_timing(self.plan, C.byref(a), C.byref(b), C.byref(c),
                                          C.byref(d)), "timing")
        return a.value, b.value, c.value, d.value

    @property
    def current(self) -> int:
        return self.lib.mtb_yee2d_current(self.plan)

    @property
    def pole_slot(self) -> int:
        """The pole buffer holding P(n) (three rotate; P(n-1) is two slots on)."""
        return self.lib.mtb_yee2d_pole_slot(self.plan)

    # ---------------------------------------------------------------- export
    def _unpack(self, box, shape, off=(0, 0), den=None, den_off=None):
        out = torch.empty(shape, dtype=torch.float32, device=self.device)
        if out.numel() == 0:
            return out
        P = box.shape[1]
        if den is None:
            L.check(self.lib.mtb_unpack(L.ptr(box), shape[0], shape[1], 1, P, 1, off[0], off[1],
                                        0, L.ptr(out), shape[1], 1, self._sptr()), "unpack")
        else:
            L.check(self.lib.mtb_unpack_ratio(L.ptr(box), L.ptr(den), shape[0], shape[1], 1, P,
                                              1, off[0], off[1], 0, L.ptr(out), shape[1], 1,
                                              self._sptr()), "unpack")
        return out

    def check(self):
        """Raise if a bounded wait of a staging kernel (row march, temporally blocked
        tiles) expired; synchronises the plan's stream (once per run)."""
        if not getattr(self, "_checked", False):
            L.check(self.lib.mtb_yee2d_check(self.plan, self._sptr()), "mtb_yee2d_check")
            self._checked = True

    def state(self, b: int = 0):
        """Current state of structure b, as the input state's own type."""
        self.check()
        it = self.items[b]
        cur = self.current
        s, nx, ny, bx = it.state, it.nx, it.ny, it.box
        if it.te:
            Hz = self._unpack(bx["main"][cur], (nx - 1, ny - 1))
            Dx = self._unpack(bx["x"][cur], (nx - 1, ny))
            Dy = self._unpack(bx["y"][cur], (nx, ny - 1))
            pol = {}
            te3 = getattr(it, "te3_box", None)
            if "pol_x" in bx:
                n_p = s.Px_cur.shape[0]
                ps_ = self.pole_slot
                pc = self._unpack_stack(bx["pol_x"][ps_], n_p, nx, (nx - 1, ny))
                pol.update(Px_cur=pc, Px_prev=self._unpack_stack(bx["pol_x"][(ps_ + 2) % 3], n_p,
                                                                 nx, (nx - 1, ny)))
                Ex = (Dx - pc.sum(0)) / it.coeffs.eps_x.to(Dx)
            else:
                Ex = self._unpack(bx["x"][cur], (nx - 1, ny), den=bx["eps_a"])
            if "pol_y" in bx:
                n_p = s.Py_cur.shape[0]
                ps_ = self.pole_slot
                pc = self._unpack_stack(bx["pol_y"][ps_], n_p, nx, (nx, ny - 1))
                pol.update(Py_cur=pc, Py_prev=self._unpack_stack(bx["pol_y"][(ps_ + 2) % 3], n_p,
                                                                 nx, (nx, ny - 1)))
                Ey = (Dy - pc.sum(0)) / it.coeffs.eps_y.to(Dy)
            else:
                Ey = self._unpack(bx["y"][cur], (nx, ny - 1), den=bx["eps_b"])
            if te3 is not None:                 # the stored E of the three-pass kernels
                Ex = self._unpack(te3[0], (nx - 1, ny))
                Ey = self._unpack(te3[1], (nx, ny - 1))
            ps = bx["psi"]
            return s._replace(
                Hz=Hz, Ex=Ex, Ey=Ey, Dx=Dx, Dy=Dy, **pol,
                psi_Hzy=self._unpack(ps[0][cur], (nx - 1, ny - 2), (0, 1)),
                psi_Hzx=self._unpack(ps[1][cur], (nx - 2, ny - 1), (1, 0)),
                psi_Eyx=self._unpack(ps[2][cur], (nx - 1, ny - 1)),
                psi_Exy=self._unpack(ps[3][cur], (nx - 1, ny - 1)))
        Dz = self._unpack(bx["main"][cur], (nx, ny))
        pol = {}
        if "pol" in bx:
            n_p = s.P_cur.shape[0]
            ps_ = self.pole_slot
            pc = self._unpack(bx["pol"][ps_], (n_p * nx, ny)).reshape(n_p, nx, ny)
            pp = self._unpack(bx["pol"][(ps_ + 2) % 3], (n_p * nx, ny)).reshape(n_p, nx, ny)
            pol = dict(P_cur=pc, P_prev=pp)
            Ez = (Dz - pc.sum(0)) / it.coeffs.eps_inf.to(Dz)
        else:
            Ez = self._unpack(bx["main"][cur], (nx, ny), den=bx["eps_a"])
        if it.nl:
            # the fixed point the kernels use (core/stepper_tm.py:222-230)
            c = it.coeffs
            rhs = Dz - (pol["P_cur"].sum(0) if "P_cur" in pol else 0.0)
            eps = c.eps_inf.to(Dz)
            x2 = c.chi2.to(Dz) if c.chi2 is not None else torch.zeros_like(Dz)
            x3 = c.chi3.to(Dz)
            Ez = rhs / eps
            for _ in range(3):
                Ez = rhs / (eps + x2 * Ez + x3 * Ez * Ez)
        ps = bx["psi"]
        nx_e, ny_e = s.psi_Hyx.shape
        xoff, yoff = int(nx_e == nx - 2), int(ny_e == ny - 2)
        for name, n in (("Hx0", nx), ("Hy0", ny)):
            if name in bx:
                pol[name] = bx[name][cur][:n].clone()
        if "B" in bx:
            nm, ps_ = it.n_mp, self.pole_slot
            shp = ((nx, ny - 1), (nx - 1, ny))
            pol.update(Bx=self._unpack(bx["B"][0][cur], shp[0]),
                       By=self._unpack(bx["B"][1][cur], shp[1]))
            for c_, sfx in enumerate(("x", "y")):
                mm = bx["M"][c_]
                pol[f"M{sfx}_cur"] = self._unpack_stack(mm[ps_], nm, nx, shp[c_])
                pol[f"M{sfx}_prev"] = self._unpack_stack(mm[(ps_ + 2) % 3], nm, nx, shp[c_])
        return s._replace(
            Ez=Ez, Dz=Dz, **pol,
            Hx=self._unpack(bx["x"][cur], (nx, ny - 1)),
            Hy=self._unpack(bx["y"][cur], (nx - 1, ny)),
            psi_Ezy=self._unpack(ps[0][cur], (nx, ny - 1)),
            psi_Ezx=self._unpack(ps[1][cur], (nx - 1, ny)),
            psi_Hyx=self._unpack(ps[2][cur], (nx_e, ny_e), (xoff, yoff)),
            psi_Hxy=self._unpack(ps[3][cur], (nx_e, ny_e), (xoff, yoff)))

    def accumulators(self, b: int = 0):
        return list(self.items[b].accs)

    def close(self):
        if getattr(self, "plan", None):
            self.lib.mtb_yee2d_plan_destroy(self.plan)
            self.plan = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
