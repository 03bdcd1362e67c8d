"""3D engine: the reference's State3D / Coeffs3D / source / monitors
(core/stepper_3d.py:28-67, core/monitors_3d.py:18-189) -> one mtb_yee3d plan.

Supported: the CPML boundary (12 psi arrays) or the matched-sigma absorber, scalar
eps, conductive damping (sigma_d, sigma_b), dispersive poles, PMC walls; point / mask /
plane-indexed soft currents on Ex, Ey or Ez; FluxMonitor3D and plane
DFTFieldsMonitor3D (sum-reduced).
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib as L
from ._lib import MtbUnsupported
from .engine2d import PHASE_MODES, _need, _round4, coef_table

FIELDS = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")
PSI = ("psi_Ez_y", "psi_Ey_z", "psi_Ex_z", "psi_Ez_x", "psi_Ey_x", "psi_Ex_y",
       "psi_Hz_y", "psi_Hy_z", "psi_Hx_z", "psi_Hz_x", "psi_Hy_x", "psi_Hx_y")
POLES = ("Px_cur", "Px_prev", "Py_cur", "Py_prev", "Pz_cur", "Pz_prev")
# box offset of each psi array: the E-side ones cover the interior of
# their derivative axis (core/stepper_3d.py:52-57)
PSI_OFF = ((0, 0, 0),) * 6 + ((0, 1, 0), (0, 0, 1), (0, 0, 1), (1, 0, 0), (1, 0, 0), (0, 1, 0))


def _plain_profiles(cpml, dims):
    """The CPML profiles the kernels read: inert (b = 1, a = 0, kappa = 1) on every axis
    when there is no CPML (the absorber-only boundary, cpml None), and inert where the
    reference writes its plain-derivative profile (b = 0, a = 0: the memory is reset to
    zero every step, so b = 1 with memory left at zero is the same update)."""
    out = {}
    for ax, (kh, ke) in enumerate((("hx", "ex"), ("hy", "ey"), ("hz", "ez"))):
        for key, n in ((kh, dims[ax] - 1), (ke, dims[ax] - 2)):
            if cpml is None:
                b, a, k = (torch.ones(n), torch.zeros(n), torch.ones(n))
            else:
                b, a, k = cpml[key]
                plain = (a == 0) & (b == 0)
                b = torch.where(plain, torch.ones_like(b), b)
            out[key] = (b, a, k)
    return out


def field_shapes(nx, ny, nz):
    return {"Ex": (nx - 1, ny, nz), "Ey": (nx, ny - 1, nz), "Ez": (nx, ny, nz - 1),
            "Hx": (nx, ny - 1, nz - 1), "Hy": (nx - 1, ny, nz - 1), "Hz": (nx - 1, ny - 1, nz)}


def flux_window(normal, idx, nx, ny, nz, win=None, ap=0):
    """The common cropped window of FluxMonitor3D._plane (core/monitors_3d.py:124-162):
    returns (pairs, (l0, h0, l1, h1)) with pairs = [(E comp, H comp)] * 2 for the
    a/b tangential pairs."""
    if normal == "z":
        pairs, m0, m1 = [("Ex", "Hy"), ("Ey", "Hx")], nx - 1, ny - 1
    elif normal == "x":
        pairs, m0, m1 = [("Ey", "Hz"), ("Ez", "Hy")], ny - 1, nz - 1
    else:
        pairs, m0, m1 = [("Ez", "Hx"), ("Ex", "Hz")], nx - 1, nz - 1
    if win is not None:
        l0, h0, l1, h1 = win
    else:
        l0, h0, l1, h1 = ap, m0 - ap, ap, m1 - ap
    l0 = max(0, l0); l1 = max(0, l1)
    h0 = min(m0, h0); h1 = min(m1, h1)
    return pairs, (l0, h0, l1, h1)


class Engine3D:
    """One 3D structure advanced by an mtb_yee3d plan.

    ``state`` is a State3D-like object with the 6 fields and 12 CPML arrays
    (or a dict of them); ``coeffs`` a Coeffs3D-like object (dt, dx, eps,
    damp, cpml, pols, pmc)."""

    def __init__(self, state, coeffs, source=None, monitors=(), *, point_sign: int = 1,
                 phase_mode: str = "exact", rows_per_seg: int = 0, ring_slots: int = 0,
                 variant: int = 0, stream=None, own=None, geometry: int = 0):
        self.lib = L.load()
        self.stream = stream
        self.keep = []
        self.state_in = state
        g = state if isinstance(state, dict) else {k: getattr(state, k, None)
                                                    for k in FIELDS + PSI + POLES}
        Ex = g["Ex"]
        _need(isinstance(Ex, torch.Tensor) and Ex.is_cuda, "3D state must be CUDA tensors")
        _need(Ex.dtype == torch.float32, f"3D state dtype {Ex.dtype}: float32 only")
        self.device = Ex.device
        nx, ny, nz = Ex.shape[0] + 1, Ex.shape[1], Ex.shape[2]
        self.nx, self.ny, self.nz = nx, ny, nz
        self.zp = zp = _round4(nz)
        shapes = field_shapes(nx, ny, nz)
        for k in FIELDS:
            _need(tuple(g[k].shape) == shapes[k], f"{k} shape {tuple(g[k].shape)}")
        # without CPML memory in the state (the absorber-only boundary) the engine keeps
        # zero memory of its own, which inert profiles leave untouched
        self.own_psi = all(g.get(k) is None for k in PSI)
        _need(self.own_psi or all(g.get(k) is not None for k in PSI),
              "3D CPML memory: all twelve arrays or none")
        pols = getattr(coeffs, "pols", None)
        n_p = 0 if pols is None else int(pols["x"][2].shape[0])
        _need(n_p <= L.MTB_MAX_POLES, f"{n_p} dispersive poles (at most {L.MTB_MAX_POLES})")
        # conductive damping (core/stepper_3d.py:217-235): the plain step when every pair
        # is (1, dt), else the split kernels' damped form with the 12 arrays
        dtf = torch.tensor(float(coeffs.dt), dtype=torch.float32)
        self._damp = None
        if any(not (bool(torch.all(d1 == 1)) and
                    bool(torch.all(d2.to(torch.float32) == dtf.to(d2.device))))
               for d1, d2 in coeffs.damp.values()):
            self._damp = {k: coeffs.damp[k] for k in ("ex", "ey", "ez", "hx", "hy", "hz")}
        self.phase_mode = PHASE_MODES[phase_mode]
        S = L.Yee3DStruct()
        S.nx, S.ny, S.nz, S.zpitch = nx, ny, nz, zp
        S.dt, S.dx = float(coeffs.dt), float(coeffs.dx)
        self._dt = float(coeffs.dt)
        S.point_sign = int(point_sign)
        # PMC walls (core/stepper_3d.py _term_pmc): bit a set for a PMC wall on axis a
        S.pmc_axes = sum(1 << int(a) for a in set(getattr(coeffs, "pmc", ()) or ()))
        self.box = {}
        for q, k in enumerate(FIELDS):
            pair = self._pair(g[k])
            self.box[k] = pair
            S.f[q][0], S.f[q][1] = L.ptr(pair[0]), L.ptr(pair[1])
        zero_box = (torch.zeros((nx, ny, zp), dtype=torch.float32, device=self.device)
                    if self.own_psi else None)
        for q, k in enumerate(PSI):
            if self.own_psi:
                # inert profiles everywhere: the kernels never read or write this memory,
                # so one zero box serves all twelve arrays and both buffers
                pair = [zero_box, zero_box]
            else:
                pair = self._pair(g[k], PSI_OFF[q])
            self.box[k] = pair
            S.psi[q][0], S.psi[q][1] = L.ptr(pair[0]), L.ptr(pair[1])
        eps = coeffs.eps
        _need(tuple(eps.shape) == (nx, ny, nz), "eps must be cell-centred (nx, ny, nz)")
        self.eps_box = self._pack(eps.to(self.device))
        S.eps = L.ptr(self.eps_box)
        cp = _plain_profiles(coeffs.cpml, (nx, ny, nz))
        dims = (nx, ny, nz)
        for ax, (kh, ke) in enumerate((("hx", "ex"), ("hy", "ey"), ("hz", "ez"))):
            bH, aH, kH = cp[kh]
            bE, aE, kE = cp[ke]
            _need(bool(torch.all(kH == 1)) and bool(torch.all(kE == 1)), "CPML kappa != 1")
            hb, ha = self._flat(bH), self._flat(aH)
            _need(hb.numel() == dims[ax] - 1, "CPML half-node profile length")
            eb, ea = self._node(bE, aE, dims[ax])
            S.prof_b[ax][0], S.prof_a[ax][0] = L.ptr(hb), L.ptr(ha)
            S.prof_b[ax][1], S.prof_a[ax][1] = L.ptr(eb), L.ptr(ea)
            self.keep += [hb, ha, eb, ea]
        if not self.own_psi:
            self._check_psi(g, cp)
        # dispersive poles (core/stepper_3d.py:236-300): P stacks ping-pong with the fields
        self.n_poles = n_p
        if n_p:
            shapes_ = field_shapes(nx, ny, nz)
            S.n_poles = n_p
            self.pol_box = {}
            for ci, key in enumerate("xyz"):
                comp = "E" + key
                cur = g.get(f"P{key}_cur")
                prev = g.get(f"P{key}_prev")
                _need(cur is not None and tuple(cur.shape) == (n_p,) + shapes_[comp],
                      f"P{key}_cur shape")
                bufs = [self._pack_stack(cur), self._pack_stack(prev)]
                c3 = self._pack_stack(pols[key][2])
                self.pol_box[key] = bufs
                self.keep += bufs + [c3]
                S.pol_p[ci][0], S.pol_p[ci][1] = L.ptr(bufs[0]), L.ptr(bufs[1])
                S.pol_c3[ci] = L.ptr(c3)
            c1 = pols["x"][0].reshape(-1).tolist()
            c2 = pols["x"][1].reshape(-1).tolist()
            for k in range(n_p):
                S.pol_c1[k], S.pol_c2[k] = float(c1[k]), float(c2[k])
        if self._damp is not None:
            shapes_ = field_shapes(nx, ny, nz)
            for q, comp in enumerate(FIELDS):
                for h, v in enumerate(self._damp[comp.lower()]):
                    v = torch.as_tensor(v, dtype=torch.float32, device=self.device)
                    box = self._pack(v.expand(shapes_[comp]).contiguous())
                    self.keep.append(box)
                    S.damp[q][h] = L.ptr(box)
        # ---- source
        self.source = source
        if source is not None:
            self._set_source(S, source, shapes)
        # ---- monitors
        self.monitors = list(monitors)
        regions, groups, gkey = [], [], {}
        planes, offs = [], []
        ring = 0

        def add_plane(comp, axis, index, w):
            nonlocal ring
            l0, h0, l1, h1 = w
            planes.append((FIELDS.index(comp), axis, index, l0, h0, l1, h1, 0))
            offs.append(ring)
            o = ring
            ring += _round4((h0 - l0) * (h1 - l1))
            return o

        def group(freqs, dt):
            f = tuple(float(x) for x in torch.as_tensor(freqs).detach().reshape(-1).cpu()
                      .to(torch.float32).to(torch.float64).tolist())
            key = (f, float(dt))
            if key not in gkey:
                gkey[key] = len(groups)
                groups.append(((C.c_double * len(f))(*f), len(f), float(dt)))
            return gkey[key], len(f)

        self.accs = []
        for mon in self.monitors:
            kind = type(mon).__name__
            _need(getattr(mon, "reduce", "sum") == "sum", f"{kind} reduce")
            gi, nf = group(mon.freqs, mon.dt)
            if kind == "FluxMonitor3D":
                axis = "xyz".index(mon.normal)
                idx = int(mon.idx)
                pairs, w = flux_window(mon.normal, idx, nx, ny, nz, getattr(mon, "win", None),
                                       int(getattr(mon, "ap", 0)))
                rows, cols = max(0, w[1] - w[0]), max(0, w[3] - w[2])
                M = rows * cols
                acc = torch.zeros((nf, 8, rows, cols), dtype=torch.float32, device=self.device)
                if M > 0:
                    for p, (ec, hc) in enumerate(pairs):
                        oe = add_plane(ec, axis, idx, w)
                        oh0 = add_plane(hc, axis, idx - 1, w)
                        oh1 = add_plane(hc, axis, idx, w)
                        regions.append(self._region(acc, (4 * p) * M, (4 * p + 1) * M, 8 * M, oe,
                                                    -1, rows, cols, gi, 2))
                        regions.append(self._region(acc, (4 * p + 2) * M, (4 * p + 3) * M, 8 * M,
                                                    oh0, oh1, rows, cols, gi, 1))
            elif kind == "DFTFieldsMonitor3D":
                _need(mon.plane is not None, "full-grid 3D DFT monitor")
                axis, idx = mon.plane
                comp = mon.component
                shp = shapes[comp]
                a0, a1 = [a for a in range(3) if a != axis]
                w = getattr(mon, "win", None) or (0, shp[a0], 0, shp[a1])
                _need(0 <= w[0] <= w[1] <= shp[a0] and 0 <= w[2] <= w[3] <= shp[a1],
                      "DFT plane window")
                rows, cols = w[1] - w[0], w[3] - w[2]
                M = rows * cols
                acc = torch.zeros((nf, 2, rows, cols), dtype=torch.float32, device=self.device)
                o = add_plane(comp, axis, int(idx), w)
                regions.append(self._region(acc, 0, M, 2 * M, o, -1, rows, cols, gi,
                                            2 if comp.startswith("E") else 1))
            else:
                raise MtbUnsupported(f"3D monitor {kind}")
            self.accs.append(acc)
        if planes:
            pl = torch.tensor(planes, dtype=torch.int32, device=self.device)
            po = torch.tensor(offs, dtype=torch.int64, device=self.device)
            self.keep += [pl, po]
            S.planes, S.plane_ring_off, S.n_planes = L.ptr(pl), L.ptr(po), len(planes)
        reg_arr = (L.DftRegion * len(regions))(*regions) if regions else None
        grp_arr = (L.PhaseGroup * max(1, len(groups)))()
        for q, (arr, nf, dt) in enumerate(groups):
            grp_arr[q].freqs = C.cast(arr, C.POINTER(C.c_double))
            grp_arr[q].nf, grp_arr[q].mode, grp_arr[q].dt = nf, self.phase_mode, dt
        self._groups = groups
        tun = L.Tuning(rows_per_seg, ring_slots, 0, variant, geometry)
        plan = C.c_void_p()
        L.check(self.lib.mtb_yee3d_plan_create(C.byref(S), reg_arr, len(regions), grp_arr,
                                               len(groups), ring, C.byref(tun), C.byref(plan)),
                "mtb_yee3d_plan_create")
        self.plan = plan
        self.S = S
        if own is not None:
            L.check(self.lib.mtb_yee3d_set_slab(plan, int(own[0]), int(own[1])),
                    "mtb_yee3d_set_slab")
        self.own = (0, nx) if own is None else (int(own[0]), int(own[1]))
        self.regions, self.n_regions = reg_arr, len(regions)
        self.groups, self.n_groups = grp_arr, len(groups)
        self.ring_elems = ring

    # ------------------------------------------------------------ helpers
    def _sptr(self):
        st = self.stream if self.stream is not None else torch.cuda.current_stream(self.device)
        return st.cuda_stream

    def _pack(self, src, off=(0, 0, 0)):
        nx, ny, zp = self.nx, self.ny, self.zp
        box = torch.empty((nx, ny, zp), dtype=torch.float32, device=self.device)
        src = src.detach().to(dtype=torch.float32).contiguous()
        n0, n1, n2 = src.shape
        L.check(self.lib.mtb_pack(L.ptr(src) if src.numel() else 0, n0, n1, n2, n1 * n2, n2,
                                  L.ptr(box), nx, ny, zp, ny * zp, zp, off[0], off[1], off[2],
                                  self._sptr()), "pack")
        return box

    def _pack_stack(self, t4):
        """(n, ...) component stack -> (n * nx, ny, zpitch) box planes."""
        n = t4.shape[0]
        out = torch.zeros((n * self.nx, self.ny, self.zp), dtype=torch.float32,
                          device=self.device)
        for k in range(n):
            out[k * self.nx:(k + 1) * self.nx].copy_(self._pack(t4[k]))
        return out

    def _pair(self, src, off=(0, 0, 0)):
        a = self._pack(src, off)
        return [a, a.clone()]

    def _flat(self, t):
        v = t.detach().reshape(-1).to(device=self.device, dtype=torch.float32).contiguous()
        self.keep.append(v)
        return v

    def _node(self, b, a, n):
        b, a = self._flat(b), self._flat(a)
        fb = torch.ones(n, dtype=torch.float32, device=self.device)
        fa = torch.zeros(n, dtype=torch.float32, device=self.device)
        _need(b.numel() == n - 2, "CPML node profile length")
        fb[1:-1] = b
        fa[1:-1] = a
        return fb, fa

    def _check_psi(self, g, cp):
        """psi must be zero where its derivative-axis profile is inert."""
        axes = (1, 2, 2, 0, 0, 1, 1, 2, 2, 0, 0, 1)
        for q, k in enumerate(PSI):
            ax = axes[q]
            key = ("h" if q < 6 else "e") + "xyz"[ax]
            b, a, _ = cp[key]
            inert = (b.reshape(-1) == 1) & (a.reshape(-1) == 0)
            sh = [1, 1, 1]
            sh[ax] = -1
            m = (g[k] != 0) & inert.to(g[k].device).reshape(sh)
            _need(not bool(m.any()), f"{k} is nonzero outside its absorbing layer")

    def _set_source(self, S, source, shapes):
        src = source.src
        comp = src[0]
        _need(comp in ("Ex", "Ey", "Ez"), f"source component {comp}")
        nx, ny = self.nx, self.ny
        S.src_comp = ("Ex", "Ey", "Ez").index(comp)
        if isinstance(src[1], torch.Tensor):              # (comp, mask): subtracted
            mask = src[1].to(self.device, torch.float32)
            _need(tuple(mask.shape) == shapes[comp], "source mask shape")
            idx = torch.nonzero(mask)
            w = mask[idx[:, 0], idx[:, 1], idx[:, 2]]
            S.src_is_point = 0
        elif len(src) == 3:                               # (comp, ix, plane): point-like sign
            ix, plane = int(src[1]), src[2].to(self.device, torch.float32)
            nz_ = torch.nonzero(plane)
            idx = torch.cat([torch.full((nz_.shape[0], 1), ix, device=self.device,
                                        dtype=nz_.dtype), nz_], 1)
            w = plane[nz_[:, 0], nz_[:, 1]]
            S.src_is_point = 1
        else:                                             # (comp, i, j, k)
            i, j, k = (int(v) for v in src[1:4])
            idx = torch.tensor([[i, j, k]], device=self.device)
            w = torch.ones(1, dtype=torch.float32, device=self.device)
            S.src_is_point = 1
        if idx.numel() == 0:
            return
        rows = idx[:, 0] * ny + idx[:, 1]
        order = torch.argsort(rows * (self.zp + 1) + idx[:, 2])
        rows, idx, w = rows[order], idx[order], w[order]
        counts = torch.bincount(rows, minlength=nx * ny)
        row_ptr = torch.zeros(nx * ny + 1, dtype=torch.int32, device=self.device)
        row_ptr[1:] = torch.cumsum(counts, 0).to(torch.int32)
        col = idx[:, 2].to(torch.int32).contiguous()
        w = w.to(torch.float32).contiguous()
        self.keep += [row_ptr, col, w]
        S.src.row_ptr, S.src.col, S.src.w = L.ptr(row_ptr), L.ptr(col), L.ptr(w)
        S.src.n, S.src.amp_col = int(col.numel()), 0

    @staticmethod
    def _region(acc, re_off, im_off, f_stride, ring_a, ring_b, rows, cols, grp, toff):
        r = L.DftRegion()
        r.acc = L.ptr(acc)
        r.re_off, r.im_off, r.f_stride = re_off, im_off, f_stride
        r.ring_a, r.ring_b = ring_a, ring_b
        r.rows, r.cols, r.ring_pitch, r.acc_pitch = rows, cols, cols, cols
        r.group, r.toff = grp, toff
        return r

    # ---------------------------------------------------------------- run
    def run(self, t0: int, k: int):
        if k <= 0:
            return
        coef = None
        if self.source is not None:
            # the reference's point / plane coefficient is coeffs.dt * amplitude(t)
            v = coef_table(self.source, "amplitude", t0, k, self._dt)
            self._coef = np.ascontiguousarray(v, dtype=np.float64)
            coef = self._coef.ctypes.data_as(C.POINTER(C.c_double))
        L.check(self.lib.mtb_yee3d_run(self.plan, t0, k, coef, self._sptr()), "mtb_yee3d_run")
        self.last_launches = self.lib.mtb_yee3d_last_launches(self.plan)

    def begin(self, t0: int, k: int):
        """Stage steps t0 .. t0+k-1 for half(); the amplitudes as in run()."""
        coef = None
        if self.source is not None:
            v = coef_table(self.source, "amplitude", t0, k, self._dt)
            self._coef = np.ascontiguousarray(v, dtype=np.float64)
            coef = self._coef.ctypes.data_as(C.POINTER(C.c_double))
        L.check(self.lib.mtb_yee3d_begin(self.plan, t0, k, coef, self._sptr()), "mtb_yee3d_begin")

    def half(self, part: int):
        """H (part 0) or E (part 1) update of the next staged step."""
        L.check(self.lib.mtb_yee3d_half(self.plan, int(part), self._sptr()), "mtb_yee3d_half")

    def plane(self, comp: str, i: int, nxt: bool = False):
        """Box plane i (ny x zpitch, contiguous) of a field: the live buffer, or the
        other one (where a half(0) put H(n+1/2)) when ``nxt``."""
        cur = self.current
        return self.box[comp][cur ^ 1 if nxt else cur][i]

    def reset(self):
        """Zero every field, CPML and accumulator buffer (t = 0 again)."""
        bufs = [t for p in self.box.values() for t in p] + list(self.accs) + \
            [t for p in getattr(self, "pol_box", {}).values() for t in p]
        for t in bufs:
            n = t.numel()
            L.check(self.lib.mtb_pack(0, 0, 0, 0, 0, 0, L.ptr(t), 1, 1, n, n, n, 0, 0, 0,
                                      self._sptr()), "reset")

    def set_timing(self, on: bool = True):
        L.check(self.lib.mtb_yee3d_set_timing(self.plan, 1 if on else 0), "set_timing")

    def timing(self):
        a, b, c, d = C.c_double(), C.c_int64(), C.c_double(), C.c_int64()
        L.check(self.lib.mtb_yee3d_timing(self.plan, C.byref(a), C.byref(b), C.byref(c),
                                          C.byref(d)), "timing")
        return a.value, b.value, c.value, d.value

    @property
    def current(self):
        return self.lib.mtb_yee3d_current(self.plan)

    def _live_buffers(self):
        cur = self.current
        out = [self.box[k][cur] for k in FIELDS + PSI]
        for key in ("xyz" if self.n_poles else ""):
            out += [self.pol_box[key][cur], self.pol_box[key][cur ^ 1]]   # P(n), P(n-1)
        return out

    def snapshot(self):
        """Copy of the live state (box layout: six fields, twelve psi, then with poles
        P(n) and P(n-1) of Ex, Ey, Ez) for restore()."""
        return [t.clone() for t in self._live_buffers()]

    def restore(self, snap):
        """Make a snapshot() the live state again (t_idx is the caller's)."""
        for dst, src in zip(self._live_buffers(), snap):
            dst.copy_(src)

    def live_e(self):
        """The live Ex, Ey, Ez boxes (views; the next step overwrites the other buffer)."""
        cur = self.current
        return [self.box[k][cur] for k in FIELDS[:3]]

    def check(self):
        """Raise if a bounded wait of the one-pass kernel expired (synchronises)."""
        L.check(self.lib.mtb_yee3d_check(self.plan, self._sptr()), "mtb_yee3d_check")

    def fields(self):
        """Current fields and CPML memory as reference-shaped tensors."""
        self.check()
        cur = self.current
        nx, ny, nz, zp = self.nx, self.ny, self.nz, self.zp
        shapes = field_shapes(nx, ny, nz)
        out = {}
        for k in FIELDS:
            out[k] = self._unpack(self.box[k][cur], shapes[k])
        psi_shapes = [shapes["Hx"], shapes["Hx"], shapes["Hy"], shapes["Hy"], shapes["Hz"],
                      shapes["Hz"], (nx - 1, ny - 2, nz), (nx - 1, ny, nz - 2),
                      (nx, ny - 1, nz - 2), (nx - 2, ny - 1, nz), (nx - 2, ny, nz - 1),
                      (nx, ny - 2, nz - 1)]
        for q, k in enumerate(PSI):
            out[k] = (None if self.own_psi else
                      self._unpack(self.box[k][cur], psi_shapes[q], PSI_OFF[q]))
        if self.n_poles:
            nxb = self.nx
            for key in "xyz":
                shp = shapes["E" + key]
                for name, b in (("cur", cur), ("prev", cur ^ 1)):
                    box = self.pol_box[key][b]
                    out[f"P{key}_{name}"] = torch.stack(
                        [self._unpack(box[k * nxb:(k + 1) * nxb], shp)
                         for k in range(self.n_poles)])
        return out

    def _unpack(self, box, shape, off=(0, 0, 0)):
        out = torch.empty(shape, dtype=torch.float32, device=self.device)
        if out.numel() == 0:
            return out
        ny, zp = self.ny, self.zp
        L.check(self.lib.mtb_unpack(L.ptr(box), shape[0], shape[1], shape[2], ny * zp, zp,
                                    off[0], off[1], off[2], L.ptr(out), shape[1] * shape[2],
                                    shape[2], self._sptr()), "unpack")
        return out

    def state(self):
        f = self.fields()
        s = self.state_in
        if isinstance(s, dict):
            return f
        return s._replace(**f)

    def close(self):
        if getattr(self, "plan", None):
            self.lib.mtb_yee3d_plan_destroy(self.plan)
            self.plan = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
