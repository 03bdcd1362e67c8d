"""3D coefficients and state (reference: core/stepper_3d.py:28-67, :150-292).

CPML boundary only (the reference's matched-sigma absorber, conductivity,
poles and PMC walls are not on the B200 path). dt = 0.5 dx / sqrt(3).
"""
import math
from typing import NamedTuple

import torch

from .pml import cpml_profiles, side_counts


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


def build_3d_coeffs(nx: int, ny: int, nz: int, dx: float, eps=None, npml=0,
                    dtype=torch.float32, device="cuda", sigma_d=None, sigma_b=None,
                    poles=(), pole_masks=None, **kw) -> Coeffs3D:
    """CPML coefficients: H-side profiles on the n-1 half nodes, E-side on the
    interior [1:-1] of each axis (core/stepper_3d.py:192-206); with ``sigma_d`` /
    ``sigma_b`` ((nx, ny, nz) cell-centred), the damping pairs of :217-235 Yee-averaged
    onto each component; with ``poles`` / ``pole_masks`` the ADE stacks of :236-266."""
    for k, v in kw.items():
        if v not in (None, 0, (), []):
            raise NotImplementedError(f"{k}: not implemented on the B200 path")
    dt = 0.5 * dx / math.sqrt(3.0)
    e = (eps.to(dtype=dtype, device=device) if isinstance(eps, torch.Tensor)
         else torch.ones(nx, ny, nz, dtype=dtype, device=device))
    dims = (nx, ny, nz)
    npml_ax = _axis_sides3(npml)
    if not any(l or h for l, h in npml_ax):
        raise NotImplementedError("npml = 0 (absorber / PEC box): the B200 path runs the CPML form")
    cpml = {}
    for ax, kh, ke in ((0, "hx", "ex"), (1, "hy", "ey"), (2, "hz", "ez")):
        b, a, k = cpml_profiles(dims[ax] - 1, npml_ax[ax], 0.5, dt, dx, dtype=dtype, device=device)
        cpml[kh] = (_bc(b, ax), _bc(a, ax), _bc(k, ax))
        b, a, k = cpml_profiles(dims[ax], npml_ax[ax], 0.0, dt, dx, dtype=dtype, device=device)
        cpml[ke] = (_bc(b[1:-1], ax), _bc(a[1:-1], ax), _bc(k[1:-1], ax))
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
    return Coeffs3D(dt=dt, dx=dx, eps=e, damp=damp, cpml=cpml, pols=pols)


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
