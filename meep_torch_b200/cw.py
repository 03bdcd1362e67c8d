"""Frequency-domain (CW) solve on the step kernels.

Reference: ``fields.solve_cw`` and its helpers ``_cw_unknowns``, ``_cw_pack``,
``_cw_unpack`` and ``_cw_rhs`` (mp/cpp/core.py:666-778), after meep's
src/cw_fields.cpp. The steady state at one frequency f solves

    A x = b,   A x = (step(x) - x) / dt + iW x,   iW = (1 - exp(-2 pi i f dt)) / dt,

where step is one source-free FDTD step and b one source injection scaled by -1/dt.
The unknowns are what the step carries forward (Dz, Hx, Hy, the four CPML memories,
the on-plane H lines of a symmetry cut, the pole histories); Ez is re-derived from
them after every unpack.

Here the real and imaginary parts of x are the two structures of one kernel plan,
so one matrix-vector product is one launch of the TM step over both. The Krylov
vectors stay on the device in the plan's own box layout (``Engine2D(arena=True)``):
loading a vector into the plan and reading the stepped one back are one copy each,
and the padding cells of the layout are identically zero in every Krylov vector, so
inner products and norms equal those of the reference's packed vectors. The solver
is BiCGSTAB(l) (Sleijpen and Fokkema, ETNA 1, 1993), written here in torch vector
operations on complex64 tensors.
"""
from __future__ import annotations

import cmath
import math

import torch

from .engine2d import Engine2D, MtbUnsupported

__all__ = ["CWOperator", "bicgstab_l", "solve_cw", "solve_cw_fields", "cw_amplitude"]


def cw_amplitude(src, t_idx: int) -> complex:
    """The complex current amplitude of a source at step ``t_idx``: a profile with a
    ``camplitude(t)`` (its analytic continuation, real part = the amplitude) is
    evaluated at (t_idx + 1/2) dt, anything else gives its real amplitude
    (core/sources.py:11-24)."""
    prof = getattr(src, "profile", None)
    dt = getattr(src, "dt", None)
    if prof is None or dt is None or not hasattr(prof, "camplitude"):
        return complex(src.amplitude(t_idx))
    return complex(prof.camplitude((t_idx + 0.5) * dt))


def _zero_state(state):
    """A zero state of the same type and shapes (Ez = Dz / eps = 0 is consistent)."""
    return state._replace(**{k: torch.zeros_like(v) for k, v in state._asdict().items()
                             if torch.is_tensor(v)})


class CWOperator:
    """A x = (step(x) - x) / dt + iW x over the TM unknowns, on the kernels.

    ``x`` is a complex64 device vector in the plan layout: the real part is structure
    0's arena segment, the imaginary part structure 1's, followed (with dispersive
    poles) by the P(n) and P(n-1) stacks in the box layout. ``from_states`` /
    ``to_states`` convert to and from a pair of the caller's TM states."""

    def __init__(self, state, coeffs, frequency: float, *, variant: int = 0):
        if hasattr(state, "Hz"):
            raise MtbUnsupported("solve_cw: 2D TM only (Ez/Hx/Hy)")
        if getattr(state, "Bx", None) is not None:
            raise MtbUnsupported("solve_cw with magnetic Lorentz poles")
        self.coeffs = coeffs
        self.template = _zero_state(state)
        self.eng = Engine2D([(self.template, coeffs, None, []),
                             (_zero_state(state), coeffs, None, [])],
                            arena=True, variant=variant)
        it0, it1 = self.eng.items
        self.n_ar = it0.arena_len
        self.off = (it0.arena_off, it1.arena_off)
        self.n_p = int(state.P_cur.shape[0])
        self.pl = 0 if not self.n_p else it0.box["pol"][0].numel()
        self.N = self.n_ar + 2 * self.pl
        self.dt = float(coeffs.dt)
        self.frequency = float(frequency)
        self.iomega = complex((1.0 - cmath.exp(-2j * math.pi * self.frequency * self.dt))
                              / self.dt)
        self.t = 0
        self.matvecs = 0
        seg = {name: (o - it0.arena_off, shape) for name, o, shape in it0.arena_segs}
        self._main = seg["main"]

    # ------------------------------------------------------------ layout
    def _load(self, eng, x):
        """Write x into the plan's current buffers (real -> structure 0, imaginary ->
        structure 1)."""
        a = eng.arena[eng.current]
        n = self.n_ar
        for part, off in zip((x.real, x.imag), self.off):
            a[off:off + n].copy_(part[:n])
        if self.n_p:
            s = eng.pole_slot
            for b, part in enumerate((x.real, x.imag)):
                pp = eng.items[b].box["pol"]
                pp[s].view(-1).copy_(part[n:n + self.pl])
                pp[(s + 2) % 3].view(-1).copy_(part[n + self.pl:])

    def _read(self, eng):
        a = eng.arena[eng.current]
        n = self.n_ar
        parts = []
        for b, off in enumerate(self.off):
            p = [a[off:off + n]]
            if self.n_p:
                s = eng.pole_slot
                pp = eng.items[b].box["pol"]
                p += [pp[s].view(-1), pp[(s + 2) % 3].view(-1)]
            parts.append(torch.cat(p) if len(p) > 1 else p[0])
        return torch.complex(parts[0], parts[1])

    def from_states(self, re, im):
        """The vector of a (real, imaginary) pair of TM states."""
        tmp = Engine2D([(re, self.coeffs, None, []), (im, self.coeffs, None, [])],
                       arena=True)
        try:
            return self._read(tmp).clone()
        finally:
            tmp.close()

    def to_states(self, x):
        """The (real, imaginary) TM states of a vector, Ez = (Dz - sum P) / eps."""
        self._load(self.eng, x)
        return self.eng.state(0), self.eng.state(1)

    def zeros(self):
        return torch.zeros(self.N, dtype=torch.complex64, device=self.eng.device)

    # ------------------------------------------------------------ operator
    def step(self, x):
        """One source-free step of both parts."""
        self._load(self.eng, x)
        self.eng.run(self.t, 1)
        self.matvecs += 1
        return self._read(self.eng)

    def __call__(self, x):
        y = self.step(x)
        return (y - x) / self.dt + self.iomega * x

    def rhs(self, sources, t_idx: int = 0):
        """b: one injection of each source's complex CW current into Dz, scaled by
        -1/dt (mp/cpp/core.py:705-719): Dz = +scale a mask / dt, scale = d2 under
        conductivity else dt. Magnetic sheets are not injected, as there."""
        b = self.zeros()
        o, _ = self._main
        nx, ny = self.eng.items[0].nx, self.eng.items[0].ny
        P = self.eng.items[0].pitch
        dz = b[o:o + nx * P].view(nx, P)
        c = self.coeffs
        d2 = getattr(c, "d2", None)
        for src in sources:
            mask = getattr(src, "mask", None)
            if mask is None:
                continue
            a = cw_amplitude(src, t_idx)
            m = mask.to(device=b.device, dtype=torch.float32)
            scale = (d2.to(device=b.device, dtype=torch.float32) if d2 is not None
                     else torch.full_like(m, self.dt))
            dz[:, :ny] += torch.complex(scale * m * a.real, scale * m * a.imag) / self.dt
        return b

    def close(self):
        self.eng.close()


def bicgstab_l(A, b, x, L: int = 2, tol: float = 1e-8, maxiters: int = 10000):
    """BiCGSTAB(l) for A x = b (Sleijpen and Fokkema 1993: l BiCG steps, then a minimal
    residual polynomial of degree l over the l + 1 residuals, orthogonalised by modified
    Gram-Schmidt). ``x`` is updated in place. Returns (ierr, iterations): ierr 0 when
    |r| <= tol |b|, 1 when maxiters outer iterations ran out, 2 on a breakdown (a
    vanishing or non-finite inner product). Scalars stay on the device; the one host
    synchronisation per iteration is the convergence test."""
    if L < 1:
        raise ValueError("bicgstab_l: L >= 1")
    bnorm = float(torch.linalg.vector_norm(b))
    if bnorm == 0.0:
        x.zero_()
        return 0, 0
    r = [None] * (L + 1)
    u = [None] * (L + 1)
    r[0] = b - A(x)
    rt = r[0].clone()
    u[0] = torch.zeros_like(b)
    one = torch.ones((), dtype=b.dtype, device=b.device)
    rho0, alpha, omega = one.clone(), torch.zeros_like(one), one.clone()
    it = 0
    while True:
        rn = float(torch.linalg.vector_norm(r[0]))
        if not math.isfinite(rn):
            return 2, it
        if rn <= tol * bnorm:
            return 0, it
        if it >= maxiters:
            return 1, it
        rho0 = -omega * rho0
        for j in range(L):
            rho1 = torch.vdot(rt, r[j])
            beta = alpha * rho1 / rho0
            rho0 = rho1
            for i in range(j + 1):
                u[i] = r[i] - beta * u[i]
            u[j + 1] = A(u[j])
            alpha = rho0 / torch.vdot(rt, u[j + 1])
            for i in range(j + 1):
                r[i] = r[i] - alpha * u[i + 1]
            r[j + 1] = A(r[j])
            x.add_(alpha * u[0])
        tau = [[None] * (L + 1) for _ in range(L + 1)]
        sigma = [None] * (L + 1)
        gp = [None] * (L + 1)
        for j in range(1, L + 1):
            for i in range(1, j):
                tau[i][j] = torch.vdot(r[i], r[j]) / sigma[i]
                r[j] = r[j] - tau[i][j] * r[i]
            sigma[j] = torch.vdot(r[j], r[j])
            gp[j] = torch.vdot(r[j], r[0]) / sigma[j]
        g = [None] * (L + 1)
        g[L] = gp[L]
        omega = g[L]
        for j in range(L - 1, 0, -1):
            acc = gp[j]
            for i in range(j + 1, L + 1):
                acc = acc - tau[j][i] * g[i]
            g[j] = acc
        gpp = [None] * (L + 1)
        for j in range(1, L):
            acc = g[j + 1]
            for i in range(j + 1, L):
                acc = acc + tau[j][i] * g[i + 1]
            gpp[j] = acc
        x.add_(g[1] * r[0])
        r[0] = r[0] - gp[L] * r[L]
        u[0] = u[0] - g[L] * u[L]
        for j in range(1, L):
            u[0] = u[0] - g[j] * u[j]
            x.add_(gpp[j] * r[j])
            r[0] = r[0] - gp[j] * r[j]
        it += 1


def solve_cw(state_re, state_im, coeffs, sources, frequency: float, *, t_idx: int = 0,
             tol: float = 1e-8, maxiters: int = 10000, L: int = 2, variant: int = 0):
    """Steady-state TM fields at ``frequency`` on the kernels, starting from the
    (real, imaginary) states. Returns (state_re, state_im, converged, iterations)."""
    op = CWOperator(state_re, coeffs, frequency, variant=variant)
    try:
        b = op.rhs(sources, t_idx)
        if not bool(b.abs().gt(0).any()):
            raise ValueError("zero current amplitudes in solve_cw")
        x = op.from_states(state_re, state_im)
        ierr, iters = bicgstab_l(op, b, x, L=L, tol=tol, maxiters=maxiters)
        re, im = op.to_states(x)
    finally:
        op.close()
    return re, im, ierr == 0, iters


def solve_cw_fields(fields, tol: float = 1e-8, maxiters: int = 10000, L: int = 2,
                    frequency=None):
    """``fields.solve_cw`` (mp/cpp/core.py:721-778) of the reference's fields object on
    the kernels: the same checks and frequency inference, the same operator and
    right-hand side, its state pair replaced by the solution, the step counter kept."""
    if getattr(fields, "_state_im", None) is None:
        raise RuntimeError("solve_cw needs complex fields: build the Simulation with "
                           "force_complex_fields=True")
    if fields._has("Hz"):
        raise NotImplementedError("solve_cw: 2D TM only (Ez/Hx/Hy)")
    m = fields._mcoeffs
    if getattr(fields, "_n_mpoles", 0):
        raise NotImplementedError("solve_cw with magnetic Lorentz poles")
    if getattr(m, "has_kerr", False) or getattr(m, "has_chi2", False):
        raise NotImplementedError("solve_cw with chi2/chi3: the step operator is nonlinear")
    if frequency is None:
        fs = {getattr(getattr(s, "profile", None), "fcen", None) for s in fields._sources}
        fs.discard(None)
        if len(fs) != 1:
            raise ValueError(f"solve_cw cannot infer one frequency from the sources "
                             f"(found {sorted(fs)}); pass frequency=")
        frequency = fs.pop()
    re, im, ok, iters = solve_cw(fields._state, fields._state_im, m, fields._sources,
                                 float(frequency), t_idx=fields._t, tol=tol,
                                 maxiters=maxiters, L=L)
    fields._cw_iters = iters
    fields._state, fields._state_im = re, im
    return ok
