"""TM / TE coefficient sets (reference: core/coeffs.py:21-74, :134-291,
:294-344, :357-503).

The NamedTuple field names are the reference's, so either side's objects can
be handed to either side's run drivers. The builders cover the B200 path's
feature set -- scalar eps, CPML (kappa = 1), PEC walls, TM PMC-in-y walls and the
low-edge symmetry cuts (mirrors; TM Rotate2 / Rotate4), conductivity, permeability and
dispersive and magnetic poles, chi2 / chi3, the TE tensor eps and oriented poles.
"""
import math
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


_UNSUPPORTED = ()


def _check_parity(**kw):
    for k, v in kw.items():
        if v not in (0, 1, -1):
            raise ValueError(f"symmetry parity {k}={v}: must be 0, +1 or -1")


def _cut_axes(grid, px, py, y_cut, x_cut, y_pmc=False):
    """A low-edge symmetry cut takes the place of that side's absorber: the kept half
    spans the cut plane to the far edge, so the low layer count drops to zero before the
    fit check (core/coeffs.py:209-220, :459-469)."""
    if y_cut:
        py = (0, py[1])
    if x_cut:
        px = (0, px[1])
    if sum(px) >= grid.nx or (sum(py) >= grid.ny and not y_pmc):
        raise ValueError(f"npml too large for grid {grid.nx}x{grid.ny}")
    return px, py


def _reject(kw):
    for k, v in kw.items():
        if k not in _UNSUPPORTED:
            raise TypeError(f"unexpected keyword argument {k!r}")
        if v is None or (isinstance(v, (int, float)) and v == 0) or (
                isinstance(v, (tuple, list)) and len(v) == 0):
            continue
        raise NotImplementedError(
            f"{k}: not implemented on the B200 path (use the reference stepper)")


def _cond_tm(grid: Grid, sigma_d, sigma_b=None, mu=None):
    """Conductivity / permeability pairs of core/coeffs.py:161-175, built when any of
    sigma_d, sigma_b, mu is given: d1 = (1 - sd dt/2) / (1 + sd dt/2), d2 = dt / (1 +
    sd dt/2) on Dz; h1 = (1 - sb dt/2) / (1 + sb dt/2), h2 = dt / (mu (1 + sb dt/2)) with
    sigma_b and mu averaged onto Hx (along y) and Hy (along x)."""
    if sigma_d is None and sigma_b is None and mu is None:
        return {}
    dt = grid.dt
    sd = _as_field(sigma_d, grid, 0.0)
    sb = _as_field(sigma_b, grid, 0.0)
    mu_ = _as_field(mu, grid, 1.0)
    sbx, mux = 0.5 * (sb[:, :-1] + sb[:, 1:]), 0.5 * (mu_[:, :-1] + mu_[:, 1:])
    sby, muy = 0.5 * (sb[:-1, :] + sb[1:, :]), 0.5 * (mu_[:-1, :] + mu_[1:, :])
    return dict(d1=(1 - sd * dt / 2) / (1 + sd * dt / 2), d2=dt / (1 + sd * dt / 2),
                h1x=(1 - sbx * dt / 2) / (1 + sbx * dt / 2), h2x=dt / (mux * (1 + sbx * dt / 2)),
                h1y=(1 - sby * dt / 2) / (1 + sby * dt / 2), h2y=dt / (muy * (1 + sby * dt / 2)))


def _cond_te(grid: Grid, sigma_d, sigma_b=None, mu=None):
    """TE pairs of core/coeffs.py:401-415: sigma_d averaged to Ex / Ey, sigma_b and mu
    averaged over the four nodes around Hz."""
    if sigma_d is None and sigma_b is None and mu is None:
        return {}
    dt = grid.dt
    sd = _as_field(sigma_d, grid, 0.0)
    sb = _as_field(sigma_b, grid, 0.0)
    mu_ = _as_field(mu, grid, 1.0)
    sdx, sdy = _avg_to_ex(sd), _avg_to_ey(sd)
    sbz = 0.25 * (sb[:-1, :-1] + sb[1:, :-1] + sb[:-1, 1:] + sb[1:, 1:])
    muz = 0.25 * (mu_[:-1, :-1] + mu_[1:, :-1] + mu_[:-1, 1:] + mu_[1:, 1:])
    return dict(d1x=(1 - sdx * dt / 2) / (1 + sdx * dt / 2), d2x=dt / (1 + sdx * dt / 2),
                d1y=(1 - sdy * dt / 2) / (1 + sdy * dt / 2), d2y=dt / (1 + sdy * dt / 2),
                hz1=(1 - sbz * dt / 2) / (1 + sbz * dt / 2), hz2=dt / (muz * (1 + sbz * dt / 2)))


def _pole_recurrence(pole, dt):
    """ADE recurrence scalars (c1, c2, c3) of one pole, as core/coeffs.py:87-106:
    pole = (fn, gamma, sigma[, fc]); w0 = 2 pi fn drives c1 / c2, wc = 2 pi fc (fc = fn
    by default: Lorentz; fn = 0, fc = plasma frequency: Drude) drives c3."""
    fn, gamma, sigma = pole[0], pole[1], pole[2]
    fc = pole[3] if len(pole) > 3 else fn
    w0, wc, G = 2 * math.pi * fn, 2 * math.pi * fc, 2 * math.pi * gamma
    den = 1.0 + G * dt / 2.0
    return ((2.0 - w0 * w0 * dt * dt) / den, -(1.0 - G * dt / 2.0) / den,
            sigma * wc * wc * dt * dt / den)


def _poles_tm(grid: Grid, eps, poles, pole_masks):
    """(c1, c2, c3), each (n_poles, nx, ny), as core/coeffs.py:195-203."""
    n = len(poles)
    c1, c2, c3 = (grid.zeros(n, grid.nx, grid.ny) for _ in range(3))
    for k, pole in enumerate(poles):
        cv1, cv2, cv3 = _pole_recurrence(pole, grid.dt)
        mask = pole_masks[k] if pole_masks is not None else torch.ones_like(eps)
        c1[k] = cv1 * torch.ones_like(eps)
        c2[k] = cv2 * torch.ones_like(eps)
        c3[k] = cv3 * mask.to(eps)
    return c1, c2, c3


def _mpoles_tm(grid: Grid, m_poles, m_pole_masks):
    """Magnetic Lorentz recurrences (core/coeffs.py:177-193): per pole (fn, gamma,
    sigma), c1 = (2 - w0^2 dt^2) / den, c2 = -(1 - G dt / 2) / den, c3 = sigma w0^2 dt^2 /
    den with w0 = 2 pi fn, G = 2 pi gamma, den = 1 + G dt / 2, c3 scaled by the pole's
    mask averaged onto Hx (along y) and Hy (along x)."""
    dt, nm = grid.dt, len(m_poles)
    out = {}
    for suf, shape, avg in (("x", (grid.nx, grid.ny - 1), lambda v: 0.5 * (v[:, :-1] + v[:, 1:])),
                            ("y", (grid.nx - 1, grid.ny), lambda v: 0.5 * (v[:-1, :] + v[1:, :]))):
        c1, c2, c3 = (grid.zeros(nm, *shape) for _ in range(3))
        for k, (fn, gamma, sigma, *_) in enumerate(m_poles):
            w0, G = 2 * math.pi * fn, 2 * math.pi * gamma
            den = 1.0 + G * dt / 2.0
            m = (m_pole_masks[k] if m_pole_masks is not None
                 else torch.ones(grid.nx, grid.ny, dtype=grid.dtype, device=grid.device))
            c1[k] = (2.0 - w0 * w0 * dt * dt) / den
            c2[k] = -(1.0 - G * dt / 2.0) / den
            c3[k] = (sigma * w0 * w0 * dt * dt / den) * avg(m.to(device=grid.device,
                                                                 dtype=grid.dtype))
        out[f"mc1{suf}"], out[f"mc2{suf}"], out[f"mc3{suf}"] = c1, c2, c3
    return out


def build_tm_coeffs(grid: Grid, eps_inf=None, poles=(), pole_masks=None, npml=0,
                    y_pmc: bool = False, sigma_d=None, sigma_b=None, mu=None,
                    y_mirror: int = 0, x_mirror: int = 0, y_rot2: int = 0, rot4: int = 0,
                    chi2=None, chi3=None, m_poles=(), m_pole_masks=None, **kw) -> TMCoeffs:
    """TM coefficients: eps map, CPML profiles sliced to the live nodes --
    H side on the n-1 half nodes, E side on the interior [1:-1] (the full
    axis under y_pmc, where the y layer is off) -- as core/coeffs.py:246-291;
    ``sigma_d``, ``sigma_b``, ``mu`` (scalars or (nx, ny)) give the conductivity and
    permeability pairs of :161-175, ``poles`` / ``pole_masks`` the ADE recurrences of
    :87-106, :195-203. ``y_mirror`` / ``x_mirror`` (+1 even, -1 odd), ``y_rot2`` and
    ``rot4`` (phase +-1) cut the low-y / low-x edge (:209-285): no absorber on the cut
    side, and the E-side profiles run from the cut node to the node before the far wall.
    ``chi2`` / ``chi3`` (scalars or (nx, ny)): instantaneous nonlinearity (:155-158),
    flagged by ``has_chi2`` / ``has_kerr`` when any value is nonzero. ``m_poles`` /
    ``m_pole_masks``: magnetic Lorentz poles (:177-193), not combined with sigma_d,
    sigma_b or mu."""
    _reject(kw)
    _check_parity(y_mirror=y_mirror, x_mirror=x_mirror, y_rot2=y_rot2, rot4=rot4)
    if y_mirror and y_rot2:
        raise ValueError("y_mirror and y_rot2 both cut the low-y edge")
    if rot4 and (y_mirror or x_mirror or y_rot2):
        raise ValueError("rot4 cuts both low edges by itself")
    if rot4 and grid.nx != grid.ny:
        raise ValueError(f"rot4 needs a square grid, got {grid.nx}x{grid.ny}")
    y_cut, x_cut = bool(y_mirror or y_rot2 or rot4), bool(x_mirror or rot4)
    if y_pmc and (y_cut or x_cut):
        raise ValueError("symmetry cuts and y_pmc exclude each other")
    live_line = y_mirror == -1 or x_mirror == -1 or y_rot2 or rot4
    if live_line and (sigma_b is not None or mu is not None or m_poles):
        raise NotImplementedError("odd mirror / Rotate2 / Rotate4 with sigma_b, mu or m_poles: "
                                  "the on-plane H line has no magnetic coefficients")
    if m_poles and (sigma_d is not None or sigma_b is not None or mu is not None):
        raise NotImplementedError("m_poles with sigma_b/mu not combined")
    dt, dx = grid.dt, grid.dx
    eps = _as_field(eps_inf, grid, 1.0)
    x2, x3 = _as_field(chi2, grid, 0.0), _as_field(chi3, grid, 0.0)
    px, py = _cut_axes(grid, *_axis_sides(npml), y_cut, x_cut, y_pmc)

    def prof(n, offset, pair, use=True):
        return cpml_profiles(n, pair if use else 0, offset, dt, dx, dtype=grid.dtype,
                             device=grid.device)

    def e_side(n, pair, cut, full=False):
        # the E-side (integer node) profile over the nodes whose D is updated
        v = prof(n, 0.0, pair, use=not full)
        if full:
            return v
        return tuple(t[:-1] for t in v) if cut else tuple(t[1:-1] for t in v)

    b_hy, a_hy, k_hy = prof(grid.ny - 1, 0.5, py, use=not y_pmc)
    b_hx, a_hx, k_hx = prof(grid.nx - 1, 0.5, px)
    b_ex, a_ex, k_ex = e_side(grid.nx, px, x_cut)
    b_ey, a_ey, k_ey = e_side(grid.ny, py, y_cut, full=y_pmc)
    c1, c2, c3 = _poles_tm(grid, eps, list(poles), pole_masks)
    return TMCoeffs(
        dt=dt, dx=dx, eps_inf=eps, chi3=x3, has_kerr=bool((x3 != 0).any()), c1=c1, c2=c2,
        c3=c3, y_pmc=y_pmc, y_mirror_lo=y_mirror, x_mirror_lo=x_mirror, y_rot2_lo=y_rot2,
        rot4_lo=rot4,
        b_hy=b_hy[None, :], a_hy=a_hy[None, :], k_hy=k_hy[None, :],
        b_hx=b_hx[:, None], a_hx=a_hx[:, None], k_hx=k_hx[:, None],
        b_ex=b_ex[:, None], a_ex=a_ex[:, None], k_ex=k_ex[:, None],
        b_ey=b_ey[None, :], a_ey=a_ey[None, :], k_ey=k_ey[None, :],
        chi2=x2, has_chi2=bool((x2 != 0).any()), **_cond_tm(grid, sigma_d, sigma_b, mu),
        **(_mpoles_tm(grid, list(m_poles), m_pole_masks) if m_poles else {}))


def _avg_to_ex(v):
    return 0.5 * (v[:-1, :] + v[1:, :])


def _avg_to_ey(v):
    return 0.5 * (v[:, :-1] + v[:, 1:])


def _axis_poles(grid: Grid, eps, shared, axis_poles, shared_masks, axis_masks, shape, avg):
    """(c1, c2, c3) of one TE E axis (core/coeffs.py:109-131): the shared poles, then the
    axis-only ones; masks are Yee-averaged from cell centres onto the E nodes."""
    allp = list(shared) + list(axis_poles)
    c1, c2, c3 = (grid.zeros(len(allp), *shape) for _ in range(3))
    ns = len(shared)
    for k, pole in enumerate(allp):
        cv1, cv2, cv3 = _pole_recurrence(pole, grid.dt)
        if k < ns:
            m = shared_masks[k] if shared_masks is not None else None
        else:
            m = axis_masks[k - ns] if axis_masks is not None else None
        mask = (m if m is not None else torch.ones_like(eps)).to(eps)
        c1[k] = cv1
        c2[k] = cv2
        c3[k] = cv3 * avg(mask)
    return c1, c2, c3


def build_te_coeffs(grid: Grid, eps_inf=None, poles=(), pole_masks=None, npml=0,
                    sigma_d=None, poles_x=(), poles_y=(), pole_masks_x=None,
                    pole_masks_y=None, sigma_b=None, mu=None, y_mirror: int = 0,
                    x_mirror: int = 0, chi2=None, chi3=None, eps_tensor=None,
                    poles_tensor=(), pole_masks_tensor=None, **kw) -> TECoeffs:
    """TE coefficients: eps Yee-averaged to Ex (nx-1, ny) and Ey (nx, ny-1)
    (core/coeffs.py:347-354, :387-388), the CPML slices of :480-491, with
    ``sigma_d``, ``sigma_b``, ``mu`` the conductivity and permeability pairs of
    :401-415, and the per-axis ADE pole stacks of :416-425 (shared ``poles`` on both
    axes, ``poles_x`` / ``poles_y`` on one). ``y_mirror`` / ``x_mirror`` (+-1) cut the
    low edge (:457-469): no absorber there; the profiles keep their interior slices.
    ``chi2`` / ``chi3`` are averaged onto Ex / Ey (:380-387); the kernels run them for TM
    only. ``eps_tensor`` = (exx, exy, eyy) at cell centres gives the inverse tensor
    Yee-averaged onto the E nodes (:389-399); ``poles_tensor`` = [(fn, gamma, (sxx, sxy,
    syy)[, fc]), ...] appends one oriented pole to each axis stack with the off-diagonal
    drives c3xy / c3yx (:428-456)."""
    _reject(kw)
    _check_parity(y_mirror=y_mirror, x_mirror=x_mirror)
    dt, dx = grid.dt, grid.dx
    eps = _as_field(eps_inf, grid, 1.0)
    x2, x3 = _as_field(chi2, grid, 0.0), _as_field(chi3, grid, 0.0)
    px, py = _cut_axes(grid, *_axis_sides(npml), bool(y_mirror), bool(x_mirror))

    def prof(n, offset, pair):
        return cpml_profiles(n, pair, offset, dt, dx, dtype=grid.dtype, device=grid.device)

    b_hx, a_hx, k_hx = prof(grid.nx - 1, 0.5, px)
    b_hy, a_hy, k_hy = prof(grid.ny - 1, 0.5, py)
    b_ey, a_ey, k_ey = (v[1:-1] for v in prof(grid.ny, 0.0, py))
    b_ex, a_ex, k_ex = (v[1:-1] for v in prof(grid.nx, 0.0, px))
    c1x, c2x, c3x = _axis_poles(grid, eps, poles, poles_x, pole_masks, pole_masks_x,
                                (grid.nx - 1, grid.ny), _avg_to_ex)
    c1y, c2y, c3y = _axis_poles(grid, eps, poles, poles_y, pole_masks, pole_masks_y,
                                (grid.nx, grid.ny - 1), _avg_to_ey)
    extra = {}
    if eps_tensor is not None:
        exx = _as_field(eps_tensor[0], grid, 1.0)
        exy = _as_field(eps_tensor[1], grid, 0.0)
        eyy = _as_field(eps_tensor[2], grid, 1.0)
        det = exx * eyy - exy * exy
        extra.update(inv_xx_x=_avg_to_ex(eyy / det), inv_xy_x=_avg_to_ex(-exy / det),
                     inv_yy_y=_avg_to_ey(exx / det), inv_xy_y=_avg_to_ey(-exy / det))
    if len(poles_tensor):
        # oriented poles: one more pole on each axis; the off-diagonal part drives Px
        # from the averaged Ey and Py from the averaged Ex
        nt = len(poles_tensor)
        t = {k: grid.zeros(nt, grid.nx - 1, grid.ny) for k in ("c1x", "c2x", "c3x", "c3xy")}
        t.update({k: grid.zeros(nt, grid.nx, grid.ny - 1) for k in ("c1y", "c2y", "c3y", "c3yx")})
        for k, pole in enumerate(poles_tensor):
            fn, gamma, (sxx, sxy, syy) = pole[0], pole[1], pole[2]
            fc = pole[3] if len(pole) > 3 else fn
            cv1, cv2, cv3 = _pole_recurrence((fn, gamma, 1.0, fc), dt)
            m = (pole_masks_tensor[k] if pole_masks_tensor is not None
                 else torch.ones_like(eps)).to(eps)
            mx, my = _avg_to_ex(m), _avg_to_ey(m)
            t["c1x"][k], t["c2x"][k] = cv1, cv2
            t["c1y"][k], t["c2y"][k] = cv1, cv2
            t["c3x"][k], t["c3xy"][k] = cv3 * sxx * mx, cv3 * sxy * mx
            t["c3y"][k], t["c3yx"][k] = cv3 * syy * my, cv3 * sxy * my
        n0x, n0y = c1x.shape[0], c1y.shape[0]
        c1x, c2x, c3x = (torch.cat([a, t[k]]) for a, k in ((c1x, "c1x"), (c2x, "c2x"),
                                                           (c3x, "c3x")))
        c1y, c2y, c3y = (torch.cat([a, t[k]]) for a, k in ((c1y, "c1y"), (c2y, "c2y"),
                                                           (c3y, "c3y")))
        extra.update(c3xy=torch.cat([grid.zeros(n0x, grid.nx - 1, grid.ny), t["c3xy"]]),
                     c3yx=torch.cat([grid.zeros(n0y, grid.nx, grid.ny - 1), t["c3yx"]]))
    return TECoeffs(
        dt=dt, dx=dx, eps_x=_avg_to_ex(eps), eps_y=_avg_to_ey(eps),
        chi3_x=_avg_to_ex(x3), chi3_y=_avg_to_ey(x3), has_kerr=bool((x3 != 0).any()),
        c1x=c1x, c2x=c2x, c3x=c3x, c1y=c1y, c2y=c2y, c3y=c3y,
        b_hx=b_hx[:, None], a_hx=a_hx[:, None], k_hx=k_hx[:, None],
        b_hy=b_hy[None, :], a_hy=a_hy[None, :], k_hy=k_hy[None, :],
        b_ey=b_ey[None, :], a_ey=a_ey[None, :], k_ey=k_ey[None, :],
        b_ex=b_ex[:, None], a_ex=a_ex[:, None], k_ex=k_ex[:, None],
        chi2_x=_avg_to_ex(x2), chi2_y=_avg_to_ey(x2), has_chi2=bool((x2 != 0).any()),
        y_mirror_lo=y_mirror, x_mirror_lo=x_mirror,
        **_cond_te(grid, sigma_d, sigma_b, mu), **extra)
