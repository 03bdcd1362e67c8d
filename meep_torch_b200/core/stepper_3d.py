"""3D coefficients and state (reference: core/stepper_3d.py:28-67, :150-292).

Boundaries: CPML, the matched-sigma absorber, or CPML on some axes and the absorber on
others; conductivity and ADE poles. PMC walls are not on the B200 path. dt = 0.5 dx /
sqrt(3).
"""
import math
from typing import NamedTuple

import torch

from .pml import absorber_sigma, cpml_profiles, side_counts


class Coeffs3D(NamedTuple):
    dt: float
    dx: float
    eps: torch.Tensor        # (nx, ny, nz) cell-centred
    damp: dict               # comp -> (d1, d2); sigma = 0 gives (1, dt)
    cpml: dict | None        # "hx".."ez" -> (b, a, kappa) broadcast along their axis
    pols: dict | None = None
    pmc: tuple = ()


class State3D(NamedTuple):
    Ex: torch.Tensor         # (nx-1, ny, nz)
    Ey: torch.Tensor         # (nx, ny-1, nz)
    Ez: torch.Tensor         # (nx, ny, nz-1)
    Hx: torch.Tensor         # (nx, ny-1, nz-1)
    Hy: torch.Tensor         # (nx-1, ny, nz-1)
    Hz: torch.Tensor         # (nx-1, ny-1, nz)
    psi_Ez_y: torch.Tensor | None = None
    psi_Ey_z: torch.Tensor | None = None
    psi_Ex_z: torch.Tensor | None = None
    psi_Ez_x: torch.Tensor | None = None
    psi_Ey_x: torch.Tensor | None = None
    psi_Ex_y: torch.Tensor | None = None
    psi_Hz_y: torch.Tensor | None = None
    psi_Hy_z: torch.Tensor | None = None
    psi_Hx_z: torch.Tensor | None = None
    psi_Hz_x: torch.Tensor | None = None
    psi_Hy_x: torch.Tensor | None = None
    psi_Hx_y: torch.Tensor | None = None
    Px_cur: torch.Tensor | None = None
    Px_prev: torch.Tensor | None = None
    Py_cur: torch.Tensor | None = None
    Py_prev: torch.Tensor | None = None
    Pz_cur: torch.Tensor | None = None
    Pz_prev: torch.Tensor | None = None


def _bc(v, ax):
    sh = [1, 1, 1]
    sh[ax] = v.shape[0]
    return v.reshape(sh)


def _axis_sides3(v):
    if isinstance(v, (tuple, list)):
        return tuple(side_counts(p) for p in v)
    return (side_counts(v),) * 3


def _avg3(v, axis):
    a = [slice(None)] * 3
    b = [slice(None)] * 3
    a[axis] = slice(None, -1)
    b[axis] = slice(1, None)
    return 0.5 * (v[tuple(a)] + v[tuple(b)])


def _inert(n, ax, dtype, device):
    """A profile that leaves the derivative plain and the CPML memory at zero (b = 1,
    a = 0, kappa = 1): the kernels never touch the memory of such a node."""
    sh = [1, 1, 1]
    sh[ax] = n
    return (torch.ones(sh, dtype=dtype, device=device), torch.zeros(sh, dtype=dtype,
                                                                     device=device),
            torch.ones(sh, dtype=dtype, device=device))


def build_3d_coeffs(nx: int, ny: int, nz: int, dx: float, eps=None, npml=0,
                    dtype=torch.float32, device="cuda", sigma_d=None, sigma_b=None,
                    poles=(), pole_masks=None, n_abs=0, absorber_axes=(), absorber_m: int = 2,
                    absorber_R0: float = 1e-15, pmc_axes=(), **kw) -> Coeffs3D:
    """Coefficients of the 3D step (core/stepper_3d.py:150-266). Boundaries as the
    reference offers them: CPML (``npml``), the matched-sigma absorber (``n_abs`` with
    ``npml = 0``: no CPML, the absorber's conductivity damps D and B), or both (CPML on
    the axes not in ``absorber_axes``, plain derivatives plus the absorber on those).
    CPML profiles: H side on the n-1 half nodes, E side on the interior [1:-1] of each
    axis (:192-206). With ``sigma_d`` / ``sigma_b`` ((nx, ny, nz) cell-centred, added to
    the absorber's), the damping pairs of :217-235 Yee-averaged onto each component;
    with ``poles`` / ``pole_masks`` the ADE stacks of :236-266. ``pmc_axes``: PMC walls
    instead of PEC on those axes, whose CPML profile is the plain derivative (:186-189)."""
    for k, v in kw.items():
        if v not in (None, 0, (), []):
            raise NotImplementedError(f"{k}: not implemented on the B200 path")
    dt = 0.5 * dx / math.sqrt(3.0)
    e = (eps.to(dtype=dtype, device=device) if isinstance(eps, torch.Tensor)
         else torch.ones(nx, ny, nz, dtype=dtype, device=device))
    dims = (nx, ny, nz)
    npml_ax, nabs_ax = _axis_sides3(npml), _axis_sides3(n_abs)
    has_pml = any(l or h for l, h in npml_ax)
    has_abs = any(l or h for l, h in nabs_ax)
    if not has_pml and not has_abs:
        raise NotImplementedError("a PEC box without CPML or absorber is not on the B200 path")
    abs_axes = set(absorber_axes) if (has_pml and has_abs) else {0, 1, 2} if has_abs else set()
    cpml = None
    if has_pml:
        cpml = {}
        for ax, kh, ke in ((0, "hx", "ex"), (1, "hy", "ey"), (2, "hz", "ez")):
            if ax in abs_axes or ax in pmc_axes:
                cpml[kh] = _inert(dims[ax] - 1, ax, dtype, device)
                cpml[ke] = _inert(dims[ax] - 2, ax, dtype, device)
                continue
            b, a, k = cpml_profiles(dims[ax] - 1, npml_ax[ax], 0.5, dt, dx, dtype=dtype,
                                    device=device)
            cpml[kh] = (_bc(b, ax), _bc(a, ax), _bc(k, ax))
            b, a, k = cpml_profiles(dims[ax], npml_ax[ax], 0.0, dt, dx, dtype=dtype, device=device)
            cpml[ke] = (_bc(b[1:-1], ax), _bc(a[1:-1], ax), _bc(k[1:-1], ax))
    sig_abs = None
    if abs_axes:
        # the boundary conductivity is the largest of the absorbing axes' ramps
        sig_abs = torch.zeros(nx, ny, nz, dtype=dtype, device=device)
        for ax in sorted(abs_axes):
            ramp = absorber_sigma(dims[ax], nabs_ax[ax], dx, R0=absorber_R0, m=absorber_m,
                                  dtype=dtype, device=device)
            sig_abs = torch.maximum(sig_abs, _bc(ramp, ax).expand(nx, ny, nz))
        sigma_d = sig_abs + (sigma_d.to(dtype=dtype, device=device) if sigma_d is not None
                             else 0.0)
        sigma_b = sig_abs + (sigma_b.to(dtype=dtype, device=device) if sigma_b is not None
                             else 0.0)
    if sigma_d is None and sigma_b is None:
        one = torch.ones((), dtype=dtype, device=device)
        d2 = torch.full((), dt, dtype=dtype, device=device)
        damp = {c: (one, d2) for c in ("ex", "ey", "ez", "hx", "hy", "hz")}
    else:
        zero = torch.zeros(nx, ny, nz, dtype=dtype, device=device)
        sd = sigma_d.to(dtype=dtype, device=device) if sigma_d is not None else zero
        sb = sigma_b.to(dtype=dtype, device=device) if sigma_b is not None else zero

        def dpair(sg):
            return (1 - sg * dt / 2) / (1 + sg * dt / 2), dt / (1 + sg * dt / 2)
        damp = {"ex": dpair(_avg3(sd, 0)), "ey": dpair(_avg3(sd, 1)), "ez": dpair(_avg3(sd, 2)),
                "hx": dpair(_avg3(_avg3(sb, 1), 2)), "hy": dpair(_avg3(_avg3(sb, 0), 2)),
                "hz": dpair(_avg3(_avg3(sb, 0), 1))}
    pols = None
    if len(poles):
        from .coeffs import _pole_recurrence
        pols = {}
        for key, shape, ax in (("x", (nx - 1, ny, nz), 0), ("y", (nx, ny - 1, nz), 1),
                               ("z", (nx, ny, nz - 1), 2)):
            npl = len(poles)
            c3 = torch.zeros(npl, *shape, dtype=dtype, device=device)
            vs = []
            for q, pole in enumerate(poles):
                v1, v2, v3 = _pole_recurrence(pole, dt)
                m = (pole_masks[q] if pole_masks is not None else
                     torch.ones(nx, ny, nz, dtype=dtype, device=device))
                c3[q] = v3 * _avg3(m.to(dtype=dtype, device=device), ax)
                vs.append((v1, v2))
            c1 = torch.tensor([v[0] for v in vs], dtype=dtype, device=device).reshape(npl, 1, 1, 1)
            c2 = torch.tensor([v[1] for v in vs], dtype=dtype, device=device).reshape(npl, 1, 1, 1)
            pols[key] = (c1, c2, c3)
    return Coeffs3D(dt=dt, dx=dx, eps=e, damp=damp, cpml=cpml, pols=pols,
                    pmc=tuple(int(a) for a in pmc_axes))


def init_3d_state(nx: int, ny: int, nz: int, npml: int = 0, n_poles: int = 0,
                  dtype=torch.float32, device="cuda") -> State3D:
    z = lambda *s: torch.zeros(*s, dtype=dtype, device=device)
    psi = {}
    if npml > 0:
        psi = dict(
            psi_Ez_y=z(nx, ny - 1, nz - 1), psi_Ey_z=z(nx, ny - 1, nz - 1),
            psi_Ex_z=z(nx - 1, ny, nz - 1), psi_Ez_x=z(nx - 1, ny, nz - 1),
            psi_Ey_x=z(nx - 1, ny - 1, nz), psi_Ex_y=z(nx - 1, ny - 1, nz),
            psi_Hz_y=z(nx - 1, ny - 2, nz), psi_Hy_z=z(nx - 1, ny, nz - 2),
            psi_Hx_z=z(nx, ny - 1, nz - 2), psi_Hz_x=z(nx - 2, ny - 1, nz),
            psi_Hy_x=z(nx - 2, ny, nz - 1), psi_Hx_y=z(nx, ny - 2, nz - 1))
    if n_poles:
        psi.update(
            Px_cur=z(n_poles, nx - 1, ny, nz), Px_prev=z(n_poles, nx - 1, ny, nz),
            Py_cur=z(n_poles, nx, ny - 1, nz), Py_prev=z(n_poles, nx, ny - 1, nz),
            Pz_cur=z(n_poles, nx, ny, nz - 1), Pz_prev=z(n_poles, nx, ny, nz - 1))
    return State3D(z(nx - 1, ny, nz), z(nx, ny - 1, nz), z(nx, ny, nz - 1),
                   z(nx, ny - 1, nz - 1), z(nx - 1, ny, nz - 1), z(nx - 1, ny - 1, nz), **psi)


def step_3d(state, c, src_amp: float = 0.0, src=None):
    """One 3D step on the GPU (core/stepper_3d.py:303-445); prefer run_3d."""
    from ..engine3d import Engine3D

    class _Src:
        def __init__(self):
            self.src = src

        def amplitude(self, t):
            return src_amp
    eng = Engine3D(state, c, _Src() if src is not None else None, ())
    eng.run(0, 1)
    out = eng.state()
    eng.close()
    return out
