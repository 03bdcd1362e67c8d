"""TM / TE coefficient sets (reference: core/coeffs.py:21-74, :134-291,
:294-344, :357-503).

The NamedTuple field names are the reference's, so either side's objects can
be handed to either side's run drivers. The builders cover the B200 path's
feature set -- scalar eps, CPML (kappa = 1), PEC walls or TM PMC-in-y walls;
the reference's dispersive / conductive / nonlinear / symmetry options raise
NotImplementedError here (the reference itself still runs them).
"""
from typing import NamedTuple

import torch

from .grid import Grid
from .pml import cpml_profiles, side_counts


def _axis_sides(npml):
    """((x_lo, x_hi), (y_lo, y_hi)) from an int or a pair of ints/pairs."""
    if isinstance(npml, (tuple, list)):
        px, py = npml
        return side_counts(px), side_counts(py)
    return (int(npml), int(npml)), (int(npml), int(npml))


class TMCoeffs(NamedTuple):
    dt: float
    dx: float
    eps_inf: torch.Tensor
    chi3: torch.Tensor
    has_kerr: bool
    c1: torch.Tensor
    c2: torch.Tensor
    c3: torch.Tensor
    y_pmc: bool
    b_hy: torch.Tensor
    a_hy: torch.Tensor
    k_hy: torch.Tensor
    b_hx: torch.Tensor
    a_hx: torch.Tensor
    k_hx: torch.Tensor
    b_ex: torch.Tensor
    a_ex: torch.Tensor
    k_ex: torch.Tensor
    b_ey: torch.Tensor
    a_ey: torch.Tensor
    k_ey: torch.Tensor
    d1: torch.Tensor | None = None
    d2: torch.Tensor | None = None
    h1x: torch.Tensor | None = None
    h2x: torch.Tensor | None = None
    h1y: torch.Tensor | None = None
    h2y: torch.Tensor | None = None
    mc1x: torch.Tensor | None = None
    mc2x: torch.Tensor | None = None
    mc3x: torch.Tensor | None = None
    mc1y: torch.Tensor | None = None
    mc2y: torch.Tensor | None = None
    mc3y: torch.Tensor | None = None
    chi2: torch.Tensor | None = None
    has_chi2: bool = False
    y_mirror_lo: int = 0
    x_mirror_lo: int = 0
    y_rot2_lo: int = 0
    rot4_lo: int = 0


class TECoeffs(NamedTuple):
    dt: float
    dx: float
    eps_x: torch.Tensor
    eps_y: torch.Tensor
    chi3_x: torch.Tensor
    chi3_y: torch.Tensor
    has_kerr: bool
    c1x: torch.Tensor
    c2x: torch.Tensor
    c3x: torch.Tensor
    c1y: torch.Tensor
    c2y: torch.Tensor
    c3y: torch.Tensor
    b_hx: torch.Tensor
    a_hx: torch.Tensor
    k_hx: torch.Tensor
    b_hy: torch.Tensor
    a_hy: torch.Tensor
    k_hy: torch.Tensor
    b_ey: torch.Tensor
    a_ey: torch.Tensor
    k_ey: torch.Tensor
    b_ex: torch.Tensor
    a_ex: torch.Tensor
    k_ex: torch.Tensor
    d1x: torch.Tensor | None = None
    d2x: torch.Tensor | None = None
    d1y: torch.Tensor | None = None
    d2y: torch.Tensor | None = None
    hz1: torch.Tensor | None = None
    hz2: torch.Tensor | None = None
    inv_xx_x: torch.Tensor | None = None
    inv_xy_x: torch.Tensor | None = None
    inv_yy_y: torch.Tensor | None = None
    inv_xy_y: torch.Tensor | None = None
    chi2_x: torch.Tensor | None = None
    chi2_y: torch.Tensor | None = None
    has_chi2: bool = False
    c3xy: torch.Tensor | None = None
    c3yx: torch.Tensor | None = None
    y_mirror_lo: int = 0
    x_mirror_lo: int = 0


def _as_field(val, grid: Grid, default: float) -> torch.Tensor:
    if val is None:
        val = default
    if isinstance(val, torch.Tensor):
        if val.shape != (grid.nx, grid.ny):
            raise ValueError(f"expected shape {(grid.nx, grid.ny)}, got {tuple(val.shape)}")
        return val.to(dtype=grid.dtype, device=grid.device)
    return torch.full((grid.nx, grid.ny), float(val), dtype=grid.dtype, device=grid.device)


_UNSUPPORTED = ("poles", "pole_masks", "chi3", "chi2", "sigma_d", "sigma_b", "mu", "m_poles",
                "m_pole_masks", "y_mirror", "x_mirror", "y_rot2", "rot4", "eps_tensor",
                "poles_x", "poles_y", "pole_masks_x", "pole_masks_y", "poles_tensor",
                "pole_masks_tensor")


def _reject(kw):
    for k, v in kw.items():
        if k not in _UNSUPPORTED:
            raise TypeError(f"unexpected keyword argument {k!r}")
        if v is None or (isinstance(v, (int, float)) and v == 0) or (
                isinstance(v, (tuple, list)) and len(v) == 0):
            continue
        raise NotImplementedError(
            f"{k}: not implemented on the B200 path (use the reference stepper)")


def build_tm_coeffs(grid: Grid, eps_inf=None, npml=0, y_pmc: bool = False, **kw) -> TMCoeffs:
    """TM coefficients: eps map, CPML profiles sliced to the live nodes --
    H side on the n-1 half nodes, E side on the interior [1:-1] (the full
    axis under y_pmc, where the y layer is off) -- as core/coeffs.py:246-291."""
    _reject(kw)
    dt, dx = grid.dt, grid.dx
    eps = _as_field(eps_inf, grid, 1.0)
    zero = _as_field(None, grid, 0.0)
    px, py = _axis_sides(npml)
    if sum(px) >= grid.nx or (sum(py) >= grid.ny and not y_pmc):
        raise ValueError(f"npml={npml} too large for grid {grid.nx}x{grid.ny}")

    def prof(n, offset, pair, use=True):
        return cpml_profiles(n, pair if use else 0, offset, dt, dx, dtype=grid.dtype,
                             device=grid.device)

    b_hy, a_hy, k_hy = prof(grid.ny - 1, 0.5, py, use=not y_pmc)
    b_hx, a_hx, k_hx = prof(grid.nx - 1, 0.5, px)
    b_ex, a_ex, k_ex = (v[1:-1] for v in prof(grid.nx, 0.0, px))
    b_ey, a_ey, k_ey = prof(grid.ny, 0.0, py, use=not y_pmc)
    if not y_pmc:
        b_ey, a_ey, k_ey = b_ey[1:-1], a_ey[1:-1], k_ey[1:-1]
    empty = grid.zeros(0, grid.nx, grid.ny)
    return TMCoeffs(
        dt=dt, dx=dx, eps_inf=eps, chi3=zero, has_kerr=False, c1=empty, c2=empty.clone(),
        c3=empty.clone(), y_pmc=y_pmc,
        b_hy=b_hy[None, :], a_hy=a_hy[None, :], k_hy=k_hy[None, :],
        b_hx=b_hx[:, None], a_hx=a_hx[:, None], k_hx=k_hx[:, None],
        b_ex=b_ex[:, None], a_ex=a_ex[:, None], k_ex=k_ex[:, None],
        b_ey=b_ey[None, :], a_ey=a_ey[None, :], k_ey=k_ey[None, :],
        chi2=zero.clone(), has_chi2=False)


def _avg_to_ex(v):
    return 0.5 * (v[:-1, :] + v[1:, :])


def _avg_to_ey(v):
    return 0.5 * (v[:, :-1] + v[:, 1:])


def build_te_coeffs(grid: Grid, eps_inf=None, npml=0, **kw) -> TECoeffs:
    """TE coefficients: eps Yee-averaged to Ex (nx-1, ny) and Ey (nx, ny-1)
    (core/coeffs.py:347-354, :387-388) and the CPML slices of :480-491."""
    _reject(kw)
    dt, dx = grid.dt, grid.dx
    eps = _as_field(eps_inf, grid, 1.0)
    zero = _as_field(None, grid, 0.0)
    px, py = _axis_sides(npml)
    if sum(px) >= grid.nx or sum(py) >= grid.ny:
        raise ValueError(f"npml={npml} too large for grid {grid.nx}x{grid.ny}")

    def prof(n, offset, pair):
        return cpml_profiles(n, pair, offset, dt, dx, dtype=grid.dtype, device=grid.device)

    b_hx, a_hx, k_hx = prof(grid.nx - 1, 0.5, px)
    b_hy, a_hy, k_hy = prof(grid.ny - 1, 0.5, py)
    b_ey, a_ey, k_ey = (v[1:-1] for v in prof(grid.ny, 0.0, py))
    b_ex, a_ex, k_ex = (v[1:-1] for v in prof(grid.nx, 0.0, px))
    ex0 = grid.zeros(0, grid.nx - 1, grid.ny)
    ey0 = grid.zeros(0, grid.nx, grid.ny - 1)
    return TECoeffs(
        dt=dt, dx=dx, eps_x=_avg_to_ex(eps), eps_y=_avg_to_ey(eps),
        chi3_x=_avg_to_ex(zero), chi3_y=_avg_to_ey(zero), has_kerr=False,
        c1x=ex0, c2x=ex0.clone(), c3x=ex0.clone(), c1y=ey0, c2y=ey0.clone(), c3y=ey0.clone(),
        b_hx=b_hx[:, None], a_hx=a_hx[:, None], k_hx=k_hx[:, None],
        b_hy=b_hy[None, :], a_hy=a_hy[None, :], k_hy=k_hy[None, :],
        b_ey=b_ey[None, :], a_ey=a_ey[None, :], k_ey=k_ey[None, :],
        b_ex=b_ex[:, None], a_ex=a_ex[:, None], k_ex=k_ex[:, None],
        chi2_x=_avg_to_ex(zero), chi2_y=_avg_to_ey(zero), has_chi2=False)
