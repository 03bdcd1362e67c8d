"""numpy restatement of meep_torch's FDTD hot path (TEST INFRASTRUCTURE ONLY).

This is the oracle the CUDA path is checked against. It is never imported by
the product package. Arrays are numpy; ``dtype`` (float32 or float64) is the
grid dtype, and every arithmetic step runs in that dtype in the same order as
the reference so that float32 runs round like the reference's float32 runs.

Scope (what the benchmark workloads use): PEC or PMC-in-y walls, CPML, scalar
eps, no dispersion / conductivity / nonlinearity / symmetry folds.
"""
from __future__ import annotations

import math

import numpy as np


# ---------------------------------------------------------------- CPML / grid

def side_counts(n_or_pair):
    """(lo, hi) cell counts from an int or a pair (core/pml.py:8-14)."""
    if isinstance(n_or_pair, (tuple, list)):
        lo, hi = n_or_pair
        return int(lo), int(hi)
    return int(n_or_pair), int(n_or_pair)


def cpml_profiles(n, npml, offset, dt, dx, m=3, R0=1e-6, alpha_max=0.05,
                  dtype=np.float64):
    """CFS-PML 1D profiles (b, a, kappa) at positions i + offset.

    Follows core/pml.py:17-59: polynomial grading u^m of sigma with
    sigma_max = -(m+1) ln R0 / (2 n dx); alpha = alpha_max (1-u) inside the
    layer; kappa = 1; b = exp(-(sigma/kappa + alpha) dt);
    a = sigma (b-1) / (kappa (sigma + kappa alpha)) where sigma > 0.
    The high wall is anchored at n-1+2*offset (core/pml.py:43-49).
    """
    dtype = np.dtype(dtype)
    n_lo, n_hi = side_counts(npml)
    x = np.arange(n, dtype=dtype) + dtype.type(offset)
    u = np.zeros(n, dtype=dtype)
    sigma = np.zeros(n, dtype=dtype)
    if n_lo > 0:
        u_lo = np.maximum((dtype.type(n_lo) - x) / dtype.type(n_lo), dtype.type(0))
        u = u + u_lo
        smax = -(m + 1) * math.log(R0) / (2.0 * n_lo * dx)
        sigma = sigma + dtype.type(smax) * u_lo ** m
    if n_hi > 0:
        wall = n - 1 + 2.0 * offset
        u_hi = np.maximum((x - dtype.type(wall - n_hi)) / dtype.type(n_hi), dtype.type(0))
        u = u + u_hi
        smax = -(m + 1) * math.log(R0) / (2.0 * n_hi * dx)
        sigma = sigma + dtype.type(smax) * u_hi ** m
    u = np.minimum(u, dtype.type(1.0))
    alpha = np.where(u > 0, dtype.type(alpha_max) * (dtype.type(1.0) - u),
                     np.zeros_like(u)).astype(dtype)
    kappa = np.ones_like(u)
    b = np.exp(-(sigma / kappa + alpha) * dtype.type(dt)).astype(dtype)
    denom = kappa * (sigma + kappa * alpha)
    with np.errstate(divide="ignore", invalid="ignore"):
        a = np.where(sigma > 0, sigma * (b - dtype.type(1.0)) /
                     np.maximum(denom, dtype.type(1e-300) if dtype == np.float64
                                else np.finfo(dtype).tiny),
                     np.zeros_like(b)).astype(dtype)
    return b, a, kappa


def _axis_sides(npml):
    """((x_lo, x_hi), (y_lo, y_hi)) from an int or pair-of-pairs (core/coeffs.py:12-18)."""
    if isinstance(npml, (tuple, list)):
        px, py = npml
        return side_counts(px), side_counts(py)
    return (int(npml), int(npml)), (int(npml), int(npml))


# ---------------------------------------------------------------- 2D TM

def _cond_pair(sd, dt):
    """(d1, d2) of an electric conductivity map (core/coeffs.py:165-166, :406-409)."""
    return (1 - sd * dt / 2) / (1 + sd * dt / 2), dt / (1 + sd * dt / 2)


def _mag_pair(sb, mu, dt):
    """(h1, h2) of a magnetic conductivity / permeability pair on the H nodes
    (core/coeffs.py:171-175, :413-414)."""
    return (1 - sb * dt / 2) / (1 + sb * dt / 2), dt / (mu * (1 + sb * dt / 2))


def pole_recurrence(pole, dt):
    """(c1, c2, c3) of one ADE pole (core/coeffs.py:87-106): pole = (fn, gamma,
    sigma[, fc]); Lorentz with fc = fn, Drude with fn = 0 and fc the plasma
    frequency."""
    fn, gamma, sig = pole[0], pole[1], pole[2]
    fc = pole[3] if len(pole) > 3 else fn
    w0, wc, G = 2 * math.pi * fn, 2 * math.pi * fc, 2 * math.pi * gamma
    den = 1.0 + G * dt / 2.0
    return (2.0 - w0 * w0 * dt * dt) / den, -(1.0 - G * dt / 2.0) / den, \
        sig * wc * wc * dt * dt / den


def tm_coeffs(nx, ny, dx, eps=None, npml=0, courant=0.5, y_pmc=False,
              dtype=np.float64, sigma=None, poles=(), pole_masks=None, sigma_b=None, mu=None,
              y_mirror=0, x_mirror=0, y_rot2=0, rot4=0, chi2=None, chi3=None,
              m_poles=(), m_pole_masks=None):
    """TM coefficient set (core/coeffs.py:134-291, PEC/PMC path only).

    Profiles are sliced to the live derivative nodes exactly as
    core/coeffs.py:251-278: H side at half nodes (n-1 long); E side on the
    interior [1:-1] (or the full axis under y_pmc). ``sigma`` (nx, ny): the
    electric conductivity pair (d1, d2) of :161-166 on Dz; ``sigma_b`` and ``mu``
    (nx, ny): the magnetic pairs of :167-175, averaged onto Hx along y and onto Hy
    along x. Any of the three builds all the pairs, as the reference does.

    Symmetry folds (:213-278): ``y_mirror`` / ``x_mirror`` (+1 even, -1 odd) cut the
    low-y / low-x edge; ``y_rot2`` (C2 about the low-y cut) and ``rot4`` (C4, both low
    edges, square grids) likewise. A cut replaces the low-side PML, and the D-side
    profiles then keep the cut row / column (0 .. n-2) instead of the interior.
    ``chi2`` / ``chi3`` (nx, ny): the instantaneous nonlinearity of :154-158.
    ``m_poles`` = [(fn, gamma, sigma), ...] with ``m_pole_masks``: magnetic Lorentz
    poles (:177-193), the masks averaged onto Hx (along y) and Hy (along x)."""
    dtype = np.dtype(dtype)
    dt = courant * dx
    e = (np.ones((nx, ny), dtype=dtype) if eps is None
         else np.asarray(eps, dtype=dtype).copy())
    for v in (y_mirror, x_mirror, y_rot2, rot4):
        if v not in (0, 1, -1):
            raise ValueError("symmetry parity must be 0, +1 or -1")
    if y_mirror and y_rot2:
        raise ValueError("y_mirror and y_rot2 both cut the low-y edge")
    if rot4 and (y_mirror or x_mirror or y_rot2):
        raise ValueError("rot4 cuts both low edges on its own")
    if rot4 and nx != ny:
        raise ValueError("rot4 needs a square grid")
    if y_pmc and (y_mirror or x_mirror or y_rot2 or rot4):
        raise ValueError("symmetry cuts and y_pmc are mutually exclusive")
    ycut, xcut = bool(y_mirror or y_rot2 or rot4), bool(x_mirror or rot4)
    px, py = _axis_sides(npml)
    if ycut:
        py = (0, py[1])
    if xcut:
        px = (0, px[1])
    if sum(px) >= nx or (sum(py) >= ny and not y_pmc):
        raise ValueError("npml too large for grid")
    yprof = py if not y_pmc else 0
    b_hy, a_hy, k_hy = cpml_profiles(ny - 1, yprof, 0.5, dt, dx, dtype=dtype)
    b_hx, a_hx, k_hx = cpml_profiles(nx - 1, px, 0.5, dt, dx, dtype=dtype)
    b_exf, a_exf, k_exf = cpml_profiles(nx, px, 0.0, dt, dx, dtype=dtype)
    if xcut:
        b_ex, a_ex, k_ex = b_exf[:-1], a_exf[:-1], k_exf[:-1]
    else:
        b_ex, a_ex, k_ex = b_exf[1:-1], a_exf[1:-1], k_exf[1:-1]
    b_eyf, a_eyf, k_eyf = cpml_profiles(ny, yprof, 0.0, dt, dx, dtype=dtype)
    if y_pmc:
        b_ey, a_ey, k_ey = b_eyf, a_eyf, k_eyf
    elif ycut:
        b_ey, a_ey, k_ey = b_eyf[:-1], a_eyf[:-1], k_eyf[:-1]
    else:
        b_ey, a_ey, k_ey = b_eyf[1:-1], a_eyf[1:-1], k_eyf[1:-1]
    cond = {}
    if sigma is not None or sigma_b is not None or mu is not None:
        z, one = np.zeros((nx, ny), dtype=dtype), np.ones((nx, ny), dtype=dtype)
        sd = z if sigma is None else np.asarray(sigma, dtype=dtype)
        sb = z if sigma_b is None else np.asarray(sigma_b, dtype=dtype)
        mu_ = one if mu is None else np.asarray(mu, dtype=dtype)
        h = dtype.type(0.5)
        cond["d1"], cond["d2"] = _cond_pair(sd, dt)
        cond["h1x"], cond["h2x"] = _mag_pair(h * (sb[:, :-1] + sb[:, 1:]),
                                             h * (mu_[:, :-1] + mu_[:, 1:]), dt)
        cond["h1y"], cond["h2y"] = _mag_pair(h * (sb[:-1, :] + sb[1:, :]),
                                             h * (mu_[:-1, :] + mu_[1:, :]), dt)
    n_p = len(poles)
    c1, c2, c3 = (np.zeros((n_p, nx, ny), dtype=dtype) for _ in range(3))
    for k, pole in enumerate(poles):        # core/coeffs.py:195-203
        cv1, cv2, cv3 = pole_recurrence(pole, dt)
        m = (np.ones((nx, ny), dtype=dtype) if pole_masks is None
             else np.asarray(pole_masks[k], dtype=dtype))
        c1[k] = dtype.type(cv1)
        c2[k] = dtype.type(cv2)
        c3[k] = dtype.type(cv3) * m
    cond.update(c1=c1, c2=c2, c3=c3)
    nl = {}
    if chi2 is not None or chi3 is not None:
        z = np.zeros((nx, ny), dtype=dtype)
        x2 = z if chi2 is None else np.asarray(chi2, dtype=dtype)
        x3 = z if chi3 is None else np.asarray(chi3, dtype=dtype)
        if (x2 != 0).any() or (x3 != 0).any():
            nl = dict(chi2=x2, chi3=x3)
    if m_poles:
        if "d1" in cond:
            raise NotImplementedError("m_poles with sigma_d / sigma_b / mu")
        nm, h = len(m_poles), dtype.type(0.5)
        for suf, shape, avg in (("x", (nx, ny - 1), lambda v: h * (v[:, :-1] + v[:, 1:])),
                                ("y", (nx - 1, ny), lambda v: h * (v[:-1, :] + v[1:, :]))):
            c1m, c2m, c3m = (np.zeros((nm,) + shape, dtype=dtype) for _ in range(3))
            for k, pole in enumerate(m_poles):
                fn, gamma, sig = pole[0], pole[1], pole[2]
                w0, G = 2 * math.pi * fn, 2 * math.pi * gamma
                den = 1.0 + G * dt / 2.0
                msk = (np.ones((nx, ny), dtype=dtype) if m_pole_masks is None
                       else np.asarray(m_pole_masks[k], dtype=dtype))
                c1m[k] = dtype.type((2.0 - w0 * w0 * dt * dt) / den)
                c2m[k] = dtype.type(-(1.0 - G * dt / 2.0) / den)
                c3m[k] = dtype.type(sig * w0 * w0 * dt * dt / den) * avg(msk)
            nl.update({"mc1" + suf: c1m, "mc2" + suf: c2m, "mc3" + suf: c3m})
    return dict(pol="tm", dt=dt, dx=dx, nx=nx, ny=ny, dtype=dtype, eps=e, y_pmc=y_pmc, **cond,
                **nl, y_mirror=y_mirror, x_mirror=x_mirror, y_rot2=y_rot2, rot4=rot4,
                b_hy=b_hy[None, :], a_hy=a_hy[None, :], k_hy=k_hy[None, :],
                b_hx=b_hx[:, None], a_hx=a_hx[:, None], k_hx=k_hx[:, None],
                b_ex=b_ex[:, None], a_ex=a_ex[:, None], k_ex=k_ex[:, None],
                b_ey=b_ey[None, :], a_ey=a_ey[None, :], k_ey=k_ey[None, :])


def tm_state(c):
    """Zero TM state with the reference's shapes (core/stepper_tm.py:37-71): with a
    low-y (low-x) cut the E-side CPML memory keeps the cut row (column); an odd y
    mirror, Rotate2 or Rotate4 carries the live on-plane Hx row (Hx0, (nx,)), an odd x
    mirror or Rotate4 the on-plane Hy column (Hy0, (ny,))."""
    nx, ny, dt = c["nx"], c["ny"], c["dtype"]
    ym, xm, r2, r4 = (c.get(k, 0) for k in ("y_mirror", "x_mirror", "y_rot2", "rot4"))
    ny_e = ny if c["y_pmc"] else (ny - 1 if (ym or r2 or r4) else ny - 2)
    nx_e = nx - 1 if (xm or r4) else nx - 2
    z = lambda *s: np.zeros(s, dtype=dt)
    n_p = c["c1"].shape[0]
    st = dict(Ez=z(nx, ny), Hx=z(nx, ny - 1), Hy=z(nx - 1, ny), Dz=z(nx, ny),
              P_cur=z(n_p, nx, ny), P_prev=z(n_p, nx, ny),
              psi_Ezy=z(nx, ny - 1), psi_Ezx=z(nx - 1, ny),
              psi_Hyx=z(nx_e, ny_e), psi_Hxy=z(nx_e, ny_e))
    if ym == -1 or r2 or r4:
        st["Hx0"] = z(nx)
    if xm == -1 or r4:
        st["Hy0"] = z(ny)
    if "mc1x" in c:                     # magnetic poles: B and the M histories
        nm = c["mc1x"].shape[0]
        st.update(Bx=z(nx, ny - 1), By=z(nx - 1, ny), Mx_cur=z(nm, nx, ny - 1),
                  Mx_prev=z(nm, nx, ny - 1), My_cur=z(nm, nx - 1, ny),
                  My_prev=z(nm, nx - 1, ny))
    return st


def tm_step(s, c, amp=0.0, mask=None, amp_h=0.0, hy_mask=None, hx_mask=None):
    """One TM step in the phase order of core/stepper_tm.py:234-254.

    step_db(B) (:85-128) -> step_source(B) (:186-196) -> step_db(D)
    (:130-166) -> step_source(D) (:197-200) -> update_eh(E) (:224-231).
    Returns a new state dict."""
    dt, dx, T = c["dt"], c["dx"], c["dtype"].type
    Ez = s["Ez"]
    dEz_dy = (Ez[:, 1:] - Ez[:, :-1]) / T(dx)
    psi_Ezy = c["b_hy"] * s["psi_Ezy"] + c["a_hy"] * dEz_dy
    curl_hx = dEz_dy / c["k_hy"] + psi_Ezy
    dEz_dx = (Ez[1:, :] - Ez[:-1, :]) / T(dx)
    psi_Ezx = c["b_hx"] * s["psi_Ezx"] + c["a_hx"] * dEz_dx
    curl_hy = dEz_dx / c["k_hx"] + psi_Ezx
    mpol = {}
    if "mc1x" in c:
        # magnetic poles: B integrates the curl (core/stepper_tm.py:115-119); H is
        # formed below by update_eh(H)
        Bx = s["Bx"] - T(dt) * curl_hx
        By = s["By"] + T(dt) * curl_hy
    elif "h1x" in c:
        # magnetic conductivity / permeability (core/stepper_tm.py:121-125)
        Hx = c["h1x"] * s["Hx"] - c["h2x"] * curl_hx
        Hy = c["h1y"] * s["Hy"] + c["h2y"] * curl_hy
    else:
        Hx = s["Hx"] - T(dt) * curl_hx
        Hy = s["Hy"] + T(dt) * curl_hy
    # on-plane H of an odd mirror / Rotate2 / Rotate4 cut (core/stepper_tm.py:94-115):
    # the ghost Ez beyond the cut is -Ez (odd), the cut row reversed times the parity
    # (C2), or the other cut's line times the parity (C4)
    r2, r4 = c.get("y_rot2", 0), c.get("rot4", 0)
    mir = {}
    if "Hx0" in s:
        ez0 = Ez[:, 0]
        ghost = r4 * Ez[0, :] if r4 else (r2 * ez0[::-1] if r2 else -ez0)
        mir["Hx0"] = s["Hx0"] - T(dt) * (ez0 - ghost) / T(dx)
    if "Hy0" in s:
        ez0x = Ez[0, :]
        ghost_x = r4 * Ez[:, 0] if r4 else -ez0x
        mir["Hy0"] = s["Hy0"] + T(dt) * (ez0x - ghost_x) / T(dx)
    # magnetic sheet current (mode sources), subtracted (core/stepper_tm.py:186-196),
    # into B when magnetic poles carry it
    if "mc1x" in c:
        if hy_mask is not None:
            By = By - T(dt * amp_h) * hy_mask
        if hx_mask is not None:
            Bx = Bx - T(dt * amp_h) * hx_mask
        # update_eh(H) (:215-224): M(n+1) = mc1 M(n) + mc2 M(n-1) + mc3 H(n-1/2),
        # H = B - sum M
        Mx = c["mc1x"] * s["Mx_cur"] + c["mc2x"] * s["Mx_prev"] + c["mc3x"] * s["Hx"]
        My = c["mc1y"] * s["My_cur"] + c["mc2y"] * s["My_prev"] + c["mc3y"] * s["Hy"]
        Hx, Hy = Bx - Mx.sum(0), By - My.sum(0)
        mpol = dict(Bx=Bx, By=By, Mx_cur=Mx, Mx_prev=s["Mx_cur"], My_cur=My,
                    My_prev=s["My_cur"])
    else:
        if hy_mask is not None:
            Hy = Hy - T(dt * amp_h) * hy_mask
        if hx_mask is not None:
            Hx = Hx - T(dt * amp_h) * hx_mask
    # D update (core/stepper_tm.py:130-166): ghost / plane H beyond each wall, then
    # differences over the live Ez region -- interior (PEC), all rows (y-PMC), or from
    # the cut up (even mirror: H = 0 ghost; odd / C2 / C4: the plane node)
    ym, xm = c.get("y_mirror", 0), c.get("x_mirror", 0)
    if c["y_pmc"]:
        Hxg = np.pad(Hx, ((0, 0), (1, 1)))
        pad_y, ys = (0, 0), slice(None)
    elif ym == 1:
        Hxg = np.pad(Hx, ((0, 0), (1, 0)))
        pad_y, ys = (0, 1), slice(None, -1)
    elif ym == -1 or r2 or r4:
        Hxg = np.concatenate([mir["Hx0"][:, None], Hx], axis=1)
        pad_y, ys = (0, 1), slice(None, -1)
    else:
        Hxg = Hx
        pad_y, ys = (1, 1), slice(1, -1)
    if xm == 1:
        Hyg = np.pad(Hy, ((1, 0), (0, 0)))
        pad_x, xs = (0, 1), slice(None, -1)
    elif xm == -1 or r4:
        Hyg = np.concatenate([mir["Hy0"][None, :], Hy], axis=0)
        pad_x, xs = (0, 1), slice(None, -1)
    else:
        Hyg = Hy
        pad_x, xs = (1, 1), slice(1, -1)
    dHx_dy = (Hxg[xs, 1:] - Hxg[xs, :-1]) / T(dx)
    dHy_dx = (Hyg[1:, ys] - Hyg[:-1, ys]) / T(dx)
    pad = (pad_x, pad_y)
    psi_Hyx = c["b_ex"] * s["psi_Hyx"] + c["a_ex"] * dHy_dx
    psi_Hxy = c["b_ey"] * s["psi_Hxy"] + c["a_ey"] * dHx_dy
    curl = dHy_dx / c["k_ex"] + psi_Hyx - dHx_dy / c["k_ey"] - psi_Hxy
    if "d1" in c:
        # conductivity (core/stepper_tm.py:158-161); the source scaled by d2 (:197-200)
        Dz = c["d1"] * s["Dz"] + c["d2"] * np.pad(curl, pad)
        if mask is not None:
            Dz = Dz - c["d2"] * T(amp) * mask
    else:
        Dz = s["Dz"] + T(dt) * np.pad(curl, pad)
        if mask is not None:
            Dz = Dz - T(dt * amp) * mask
    out = dict(Hx=Hx, Hy=Hy, Dz=Dz, psi_Ezy=psi_Ezy, psi_Ezx=psi_Ezx, psi_Hyx=psi_Hyx,
               psi_Hxy=psi_Hxy, **mir, **mpol)
    if c["c1"].shape[0]:
        # update_pols (core/stepper_tm.py:203-207) on the old Ez, then
        # update_eh(E): Ez = (Dz - sum P) / eps_inf (:220-224)
        P_new = c["c1"] * s["P_cur"] + c["c2"] * s["P_prev"] + c["c3"] * Ez
        rhs = Dz - P_new.sum(0)
        out.update(P_cur=P_new, P_prev=s["P_cur"])
    else:
        rhs = Dz
        out.update(P_cur=s.get("P_cur"), P_prev=s.get("P_prev"))
    Ez_new = rhs / c["eps"]
    if "chi3" in c:
        # instantaneous chi2 / chi3: three fixed-point sweeps of
        # E = rhs / (eps + chi2 E + chi3 E^2) (core/stepper_tm.py:225-230)
        for _ in range(3):
            Ez_new = rhs / (c["eps"] + c["chi2"] * Ez_new + c["chi3"] * Ez_new * Ez_new)
    out["Ez"] = Ez_new
    return out


# ---------------------------------------------------------------- 2D TE

def te_coeffs(nx, ny, dx, eps=None, npml=0, courant=0.5, dtype=np.float64, sigma=None,
              poles=(), pole_masks=None, sigma_b=None, mu=None, y_mirror=0, x_mirror=0,
              chi2=None, chi3=None, eps_tensor=None, poles_tensor=(), pole_masks_tensor=None):
    """TE coefficient set (core/coeffs.py:357-503, PEC path only).

    eps is Yee-averaged to Ex (nx-1, ny) and Ey (nx, ny-1) positions
    (core/coeffs.py:347-354); so is ``sigma`` for the conductivity pairs of
    :401-409 on Dx and Dy. ``sigma_b`` and ``mu`` give the Hz pair of :410-414,
    averaged over the four nodes around each Hz. Any of the three builds all pairs.
    ``y_mirror`` / ``x_mirror`` (+1 even, -1 odd) replace the low-side PML with the
    mirror wall (:457-469). ``chi2`` / ``chi3`` (nx, ny) are Yee-averaged to Ex / Ey
    (:382-387). ``eps_tensor`` = (exx, exy, eyy) at cell centres: the in-plane
    inverse tensor's components Yee-averaged to the E nodes (:390-400).
    ``poles_tensor`` = [(fn, gamma, (sxx, sxy, syy)[, fc]), ...]: oriented poles
    (:426-452) appended to both axis stacks, sxx / syy on the diagonal c3 and sxy in
    the cross terms c3xy (Px from Ey) and c3yx (Py from Ex)."""
    dtype = np.dtype(dtype)
    dt = courant * dx
    e = (np.ones((nx, ny), dtype=dtype) if eps is None
         else np.asarray(eps, dtype=dtype).copy())
    h = dtype.type(0.5)
    eps_x = h * (e[:-1, :] + e[1:, :])
    eps_y = h * (e[:, :-1] + e[:, 1:])
    if y_mirror not in (0, 1, -1) or x_mirror not in (0, 1, -1):
        raise ValueError("mirror parity must be 0, +1 or -1")
    px, py = _axis_sides(npml)
    if y_mirror:
        py = (0, py[1])
    if x_mirror:
        px = (0, px[1])
    if sum(px) >= nx or sum(py) >= ny:
        raise ValueError("npml too large for grid")
    b_hx, a_hx, k_hx = cpml_profiles(nx - 1, px, 0.5, dt, dx, dtype=dtype)
    b_hy, a_hy, k_hy = cpml_profiles(ny - 1, py, 0.5, dt, dx, dtype=dtype)
    b_ey, a_ey, k_ey = (v[1:-1] for v in cpml_profiles(ny, py, 0.0, dt, dx, dtype=dtype))
    b_ex, a_ex, k_ex = (v[1:-1] for v in cpml_profiles(nx, px, 0.0, dt, dx, dtype=dtype))
    cond = {}
    if sigma is not None or sigma_b is not None or mu is not None:
        z, one = np.zeros((nx, ny), dtype=dtype), np.ones((nx, ny), dtype=dtype)
        sd = z if sigma is None else np.asarray(sigma, dtype=dtype)
        sb = z if sigma_b is None else np.asarray(sigma_b, dtype=dtype)
        mu_ = one if mu is None else np.asarray(mu, dtype=dtype)
        q = dtype.type(0.25)
        cond["d1x"], cond["d2x"] = _cond_pair(h * (sd[:-1, :] + sd[1:, :]), dt)
        cond["d1y"], cond["d2y"] = _cond_pair(h * (sd[:, :-1] + sd[:, 1:]), dt)
        cond["hz1"], cond["hz2"] = _mag_pair(
            q * (sb[:-1, :-1] + sb[1:, :-1] + sb[:-1, 1:] + sb[1:, 1:]),
            q * (mu_[:-1, :-1] + mu_[1:, :-1] + mu_[:-1, 1:] + mu_[1:, 1:]), dt)
    # shared ADE poles on both E axes, masks Yee-averaged (core/coeffs.py:109-131, :416-425)
    for ax, shape in (("x", (nx - 1, ny)), ("y", (nx, ny - 1))):
        n_p = len(poles)
        c1, c2, c3 = (np.zeros((n_p,) + shape, dtype=dtype) for _ in range(3))
        for k, pole in enumerate(poles):
            cv1, cv2, cv3 = pole_recurrence(pole, dt)
            m = (np.ones((nx, ny), dtype=dtype) if pole_masks is None
                 else np.asarray(pole_masks[k], dtype=dtype))
            mavg = h * (m[:-1, :] + m[1:, :]) if ax == "x" else h * (m[:, :-1] + m[:, 1:])
            c1[k] = dtype.type(cv1)
            c2[k] = dtype.type(cv2)
            c3[k] = dtype.type(cv3) * mavg
        cond.update({"c1" + ax: c1, "c2" + ax: c2, "c3" + ax: c3})
    if len(poles_tensor):
        # oriented poles (core/coeffs.py:426-452): one extra pole per axis stack, the
        # cross drive zero for the plain poles before them
        for ax, shape in (("x", (nx - 1, ny)), ("y", (nx, ny - 1))):
            nt = len(poles_tensor)
            t1, t2, t3, tc = (np.zeros((nt,) + shape, dtype=dtype) for _ in range(4))
            for k, pole in enumerate(poles_tensor):
                fn, gamma, (sxx, sxy, syy) = pole[0], pole[1], pole[2]
                fc = pole[3] if len(pole) > 3 else fn
                cv1, cv2, cv3 = pole_recurrence((fn, gamma, 1.0, fc), dt)
                m = (np.ones((nx, ny), dtype=dtype) if pole_masks_tensor is None
                     else np.asarray(pole_masks_tensor[k], dtype=dtype))
                mavg = h * (m[:-1, :] + m[1:, :]) if ax == "x" else h * (m[:, :-1] + m[:, 1:])
                t1[k], t2[k] = dtype.type(cv1), dtype.type(cv2)
                t3[k] = dtype.type(cv3 * (sxx if ax == "x" else syy)) * mavg
                tc[k] = dtype.type(cv3 * sxy) * mavg
            n0 = cond["c1" + ax].shape[0]
            for key, t in (("c1", t1), ("c2", t2), ("c3", t3)):
                cond[key + ax] = np.concatenate([cond[key + ax], t])
            cond["c3xy" if ax == "x" else "c3yx"] = np.concatenate(
                [np.zeros((n0,) + shape, dtype=dtype), tc])
    nl = {}
    if chi2 is not None or chi3 is not None:
        z = np.zeros((nx, ny), dtype=dtype)
        x2 = z if chi2 is None else np.asarray(chi2, dtype=dtype)
        x3 = z if chi3 is None else np.asarray(chi3, dtype=dtype)
        if (x2 != 0).any() or (x3 != 0).any():
            nl = dict(chi2_x=h * (x2[:-1, :] + x2[1:, :]), chi2_y=h * (x2[:, :-1] + x2[:, 1:]),
                      chi3_x=h * (x3[:-1, :] + x3[1:, :]), chi3_y=h * (x3[:, :-1] + x3[:, 1:]))
    if eps_tensor is not None:
        exx, exy, eyy = (np.asarray(v, dtype=dtype) for v in eps_tensor)
        det = exx * eyy - exy * exy
        ax = lambda v: h * (v[:-1, :] + v[1:, :])          # noqa: E731
        ay = lambda v: h * (v[:, :-1] + v[:, 1:])          # noqa: E731
        nl.update(inv_xx_x=ax(eyy / det), inv_xy_x=ax(-exy / det),
                  inv_yy_y=ay(exx / det), inv_xy_y=ay(-exy / det))
    return dict(pol="te", dt=dt, dx=dx, nx=nx, ny=ny, dtype=dtype, eps=e, **cond, **nl,
                eps_x=eps_x, eps_y=eps_y, y_mirror=y_mirror, x_mirror=x_mirror,
                b_hx=b_hx[:, None], a_hx=a_hx[:, None], k_hx=k_hx[:, None],
                b_hy=b_hy[None, :], a_hy=a_hy[None, :], k_hy=k_hy[None, :],
                b_ey=b_ey[None, :], a_ey=a_ey[None, :], k_ey=k_ey[None, :],
                b_ex=b_ex[:, None], a_ex=a_ex[:, None], k_ex=k_ex[:, None])


def _avg4_to_ex(Ey):
    """Ey (nx, ny-1) at the Ex nodes (nx-1, ny), zero beyond the y walls
    (core/stepper_te.py:52-55)."""
    p = np.pad(Ey, ((0, 0), (1, 1)))
    return Ey.dtype.type(0.25) * (p[:-1, :-1] + p[:-1, 1:] + p[1:, :-1] + p[1:, 1:])


def _avg4_to_ey(Ex):
    """Ex (nx-1, ny) at the Ey nodes (nx, ny-1), zero beyond the x walls (:58-61)."""
    p = np.pad(Ex, ((1, 1), (0, 0)))
    return Ex.dtype.type(0.25) * (p[:-1, :-1] + p[:-1, 1:] + p[1:, :-1] + p[1:, 1:])


def te_state(c):
    """Zero TE state with the reference's shapes (core/stepper_te.py:27-49)."""
    nx, ny, dt = c["nx"], c["ny"], c["dtype"]
    z = lambda *s: np.zeros(s, dtype=dt)
    npx, npy = c["c1x"].shape[0], c["c1y"].shape[0]
    return dict(Hz=z(nx - 1, ny - 1), Ex=z(nx - 1, ny), Ey=z(nx, ny - 1),
                Dx=z(nx - 1, ny), Dy=z(nx, ny - 1),
                Px_cur=z(npx, nx - 1, ny), Px_prev=z(npx, nx - 1, ny),
                Py_cur=z(npy, nx, ny - 1), Py_prev=z(npy, nx, ny - 1),
                psi_Eyx=z(nx - 1, ny - 1), psi_Exy=z(nx - 1, ny - 1),
                psi_Hzy=z(nx - 1, ny - 2), psi_Hzx=z(nx - 2, ny - 1))


def te_step(s, c, amp=0.0, mask_ey=None, amp_h=0.0, hz_mask=None):
    """One TE step, entered at the D half (core/stepper_te.py:178-190):
    step_db(D) (:79-111) -> step_source(D) into Dy (:120-134) -> update_eh(E)
    (:150-175) -> step_db(B) Hz (:113-117) -> step_source(B) into Hz."""
    dt, dx, T = c["dt"], c["dx"], c["dtype"].type
    Hz = s["Hz"]
    dHz_dy = (Hz[:, 1:] - Hz[:, :-1]) / T(dx)
    psi_Hzy = c["b_ey"] * s["psi_Hzy"] + c["a_ey"] * dHz_dy
    curl_x = np.pad(dHz_dy / c["k_ey"] + psi_Hzy, ((0, 0), (1, 1)))
    dHz_dx = (Hz[1:, :] - Hz[:-1, :]) / T(dx)
    psi_Hzx = c["b_ex"] * s["psi_Hzx"] + c["a_ex"] * dHz_dx
    curl_y = np.pad(dHz_dx / c["k_ex"] + psi_Hzx, ((1, 1), (0, 0)))
    # even mirror: the on-plane tangential E row / column is live, its curl from the
    # odd Hz ghost 2 Hz[0] / dx (core/stepper_te.py:87-96); odd: the zero pad stays
    if c.get("y_mirror", 0) == 1:
        curl_x = np.concatenate([T(2.0) * Hz[:, :1] / T(dx), curl_x[:, 1:]], axis=1)
    if c.get("x_mirror", 0) == 1:
        curl_y = np.concatenate([T(2.0) * Hz[:1, :] / T(dx), curl_y[1:, :]], axis=0)
    if "d1x" in c:
        # conductivity (core/stepper_te.py D update); the source scaled by d2y
        Dx = c["d1x"] * s["Dx"] + c["d2x"] * curl_x
        Dy = c["d1y"] * s["Dy"] - c["d2y"] * curl_y
        if mask_ey is not None:
            Dy = Dy - c["d2y"] * T(amp) * mask_ey
    else:
        Dx = s["Dx"] + T(dt) * curl_x
        Dy = s["Dy"] - T(dt) * curl_y
        if mask_ey is not None:
            Dy = Dy - T(dt * amp) * mask_ey
    pol = {}
    if c["c1x"].shape[0] or c["c1y"].shape[0]:
        # update_pols on the old E (core/stepper_te.py:136-146), update_eh(E) (:159-169)
        Px = c["c1x"] * s["Px_cur"] + c["c2x"] * s["Px_prev"] + c["c3x"] * s["Ex"]
        Py = c["c1y"] * s["Py_cur"] + c["c2y"] * s["Py_prev"] + c["c3y"] * s["Ey"]
        if "c3xy" in c:
            # oriented poles: the off-diagonal drive (core/stepper_te.py:142-145)
            Px = Px + c["c3xy"] * _avg4_to_ex(s["Ey"])
            Py = Py + c["c3yx"] * _avg4_to_ey(s["Ex"])
        pol = dict(Px_cur=Px, Px_prev=s["Px_cur"], Py_cur=Py, Py_prev=s["Py_cur"])
        rhs_x, rhs_y = Dx - Px.sum(0), Dy - Py.sum(0)
    else:
        pol = {k: s.get(k) for k in ("Px_cur", "Px_prev", "Py_cur", "Py_prev")}
        rhs_x, rhs_y = Dx, Dy
    if "inv_xx_x" in c:
        # in-plane tensor eps (core/stepper_te.py:162-165): E = eps^-1 (D - P), the
        # cross terms from the other component averaged over four nodes
        Ex = c["inv_xx_x"] * rhs_x + c["inv_xy_x"] * _avg4_to_ex(rhs_y)
        Ey = c["inv_yy_y"] * rhs_y + c["inv_xy_y"] * _avg4_to_ey(rhs_x)
    else:
        Ex = rhs_x / c["eps_x"]
        Ey = rhs_y / c["eps_y"]
    if "chi3_x" in c:
        # instantaneous chi2 / chi3 (core/stepper_te.py:157-174): three fixed-point
        # sweeps with |E|^2 from the other component averaged over four nodes
        for _ in range(3):
            E2x = Ex * Ex + _avg4_to_ex(Ey) ** 2
            E2y = Ey * Ey + _avg4_to_ey(Ex) ** 2
            Ex = rhs_x / (c["eps_x"] + c["chi2_x"] * Ex + c["chi3_x"] * E2x)
            Ey = rhs_y / (c["eps_y"] + c["chi2_y"] * Ey + c["chi3_y"] * E2y)
    dEy_dx = (Ey[1:, :] - Ey[:-1, :]) / T(dx)
    dEx_dy = (Ex[:, 1:] - Ex[:, :-1]) / T(dx)
    psi_Eyx = c["b_hx"] * s["psi_Eyx"] + c["a_hx"] * dEy_dx
    psi_Exy = c["b_hy"] * s["psi_Exy"] + c["a_hy"] * dEx_dy
    curl_z = dEy_dx / c["k_hx"] + psi_Eyx - dEx_dy / c["k_hy"] - psi_Exy
    if "hz1" in c:
        # magnetic conductivity / permeability (core/stepper_te.py:112-114)
        Hz_new = c["hz1"] * Hz - c["hz2"] * curl_z
    else:
        Hz_new = Hz - T(dt) * curl_z
    if hz_mask is not None:
        Hz_new = Hz_new - T(dt * amp_h) * hz_mask
    return dict(Hz=Hz_new, Ex=Ex, Ey=Ey, Dx=Dx, Dy=Dy, psi_Eyx=psi_Eyx,
                psi_Exy=psi_Exy, psi_Hzy=psi_Hzy, psi_Hzx=psi_Hzx, **pol)


# ---------------------------------------------------------------- sources

def gaussian_pulse(fcen, fwidth, cutoff=5.0):
    """Time profile cos(2 pi f (t-t0)) exp(-(t-t0)^2/(2 w^2)), w = 1/fwidth,
    t0 = cutoff*w (core/sources.py:26-36). Returns a float -> float callable."""
    w = 1.0 / fwidth
    t0 = cutoff * w

    def amplitude(t):
        return math.cos(2 * math.pi * fcen * (t - t0)) * math.exp(-((t - t0) ** 2) / (2 * w ** 2))
    return amplitude


def line_source_mask(nx, ny, dx, ix, j0, j1, dtype=np.float64):
    """LineSource mask (core/sources.py:49-91): 1 on x=ix, y in [j0, j1),
    scaled by dx/dx^2 for an extended line and 1/dx^2 for a single cell."""
    dtype = np.dtype(dtype)
    mask = np.zeros((nx, ny), dtype=dtype)
    mask[ix, j0:j1] = 1.0
    per_cell = dx if (j1 - j0) > 1 else 1.0
    return (mask * dtype.type(per_cell / dx ** 2)).astype(dtype)


def src_time(t_idx, dt):
    """Soft sources sample their profile at (t_idx + 1/2) dt (core/sources.py:90-91)."""
    return (t_idx + 0.5) * dt


# ---------------------------------------------------------------- 2D monitors

def dft_sample(F, t_idx, dt, freqs, component, dtype):
    """DFTFieldsMonitor.sample (core/monitors.py:40-46): dt*[cos(wt) F, -sin(wt) F]
    with t = (t_idx + 1) dt for E components and (t_idx + 1/2) dt for H; the
    phase is evaluated in the grid dtype like the reference."""
    T = np.dtype(dtype).type
    off = 1.0 if component.startswith("E") else 0.5
    t = (t_idx + off) * dt
    w = (T(2 * math.pi) * np.asarray(freqs, dtype=dtype))[:, None, None]
    wt = w * T(t)
    return T(dt) * np.stack([np.cos(wt) * F, -np.sin(wt) * F], axis=1)


def _line_dft(E, H, tE, tH, dt, freqs, dtype):
    T = np.dtype(dtype).type
    w = (T(2 * math.pi) * np.asarray(freqs, dtype=dtype))[:, None]
    wE, wH = w * T(tE), w * T(tH)
    return T(dt) * np.stack([np.cos(wE) * E, -np.sin(wE) * E,
                             np.cos(wH) * H, -np.sin(wH) * H], axis=1)


def flux_tm_sample(s, t_idx, dt, freqs, x_normal, idx, lo, hi, dtype):
    """FluxMonitorTM.sample (core/monitors.py:71-95): Ez on the line and the
    2-point average of Hy (x-normal) or Hx (y-normal); E at (t+1)dt, H at (t+1/2)dt."""
    T = np.dtype(dtype).type
    if x_normal:
        E = s["Ez"][idx, lo:hi]
        H = T(0.5) * (s["Hy"][idx - 1, lo:hi] + s["Hy"][idx, lo:hi])
    else:
        E = s["Ez"][lo:hi, idx]
        H = T(0.5) * (s["Hx"][lo:hi, idx - 1] + s["Hx"][lo:hi, idx])
    return _line_dft(E, H, (t_idx + 1.0) * dt, (t_idx + 0.5) * dt, dt, freqs, dtype)


def flux_te_sample(s, t_idx, dt, freqs, ix, lo, hi, dtype):
    """FluxMonitorTE.sample (core/monitors.py:112-122): Ey and the averaged Hz,
    E at (t+1/2)dt, H at (t+1)dt."""
    T = np.dtype(dtype).type
    E = s["Ey"][ix, lo:hi]
    H = T(0.5) * (s["Hz"][ix - 1, lo:hi] + s["Hz"][ix, lo:hi])
    return _line_dft(E, H, (t_idx + 0.5) * dt, (t_idx + 1.0) * dt, dt, freqs, dtype)


def flux_tey_sample(s, t_idx, dt, freqs, iy, lo, hi, dtype):
    """FluxMonitorTEY.sample (core/monitors.py:141-151): Ex and Hz averaged in y."""
    T = np.dtype(dtype).type
    E = s["Ex"][lo:hi, iy]
    H = T(0.5) * (s["Hz"][lo:hi, iy - 1] + s["Hz"][lo:hi, iy])
    return _line_dft(E, H, (t_idx + 0.5) * dt, (t_idx + 1.0) * dt, dt, freqs, dtype)


def line_flux(acc, dx, sign):
    """Flux from 4 line accumulators: sign*1/2*sum(ReE ReH + ImE ImH)*dx
    (core/monitors.py:97-100, :124-126, :153-155)."""
    ReE, ImE, ReH, ImH = (acc[:, k] for k in range(4))
    return sign * 0.5 * (ReE * ReH + ImE * ImH).sum(-1) * dx


def run_2d(step, s, c, n_steps, amp_fn=None, mask=None, monitors=(), t0=0):
    """Per-step loop of core/run.py:10-40: step, then every monitor samples the
    new state and sum-folds. ``monitors`` are callables (state, t_idx) -> sample."""
    acc = [None] * len(monitors)
    for k in range(n_steps):
        t = t0 + k
        if amp_fn is not None:
            s = step(s, c, amp_fn(t), mask)
        else:
            s = step(s, c)
        for i, mon in enumerate(monitors):
            smp = mon(s, t)
            acc[i] = smp if acc[i] is None else acc[i] + smp
    return s, acc


# ---------------------------------------------------------------- 3D

def _avg(v, axis):
    a = [slice(None)] * 3
    b = [slice(None)] * 3
    a[axis] = slice(None, -1)
    b[axis] = slice(1, None)
    return v.dtype.type(0.5) * (v[tuple(a)] + v[tuple(b)])


def _d(v, axis):
    a = [slice(None)] * 3
    b = [slice(None)] * 3
    a[axis] = slice(None, -1)
    b[axis] = slice(1, None)
    return v[tuple(b)] - v[tuple(a)]


def _bc(v, ax):
    sh = [1, 1, 1]
    sh[ax] = v.shape[0]
    return v.reshape(sh)


def _per_axis3(v):
    """Per-axis layer counts of a 3D box (core/stepper_3d.py:142-147): an int (or a
    (lo, hi) pair) for all three axes, or a 3-sequence of int-or-pair."""
    if isinstance(v, (tuple, list)):
        return tuple(v)
    return (v, v, v)


def absorber_sigma(n, nabs, dx, R0=1e-15, m=2, dtype=np.float64):
    """Matched-sigma absorber profile along one axis (core/pml.py:62-80): a
    quadratic (order m) ramp on each edge's nabs cells, peak -(m+1) ln R0 / (2 nc dx)."""
    n_lo, n_hi = side_counts(nabs)
    p = np.zeros(n, dtype=dtype)

    def ramp(nc):
        smax = -(m + 1) * math.log(R0) / (2.0 * nc * dx)
        i = np.arange(nc, dtype=dtype)
        return smax * ((nc - i - 0.5) / nc) ** m
    if n_lo > 0:
        p[:n_lo] = ramp(n_lo)
    if n_hi > 0:
        p[n - n_hi:] = ramp(n_hi)[::-1]
    return p


def coeffs_3d(nx, ny, nz, dx, eps=None, npml=0, dtype=np.float64, sigma_d=None,
              sigma_b=None, poles=(), pole_masks=None, n_abs=0, absorber_axes=(),
              absorber_m=2, absorber_R0=1e-15, pmc_axes=()):
    """3D coefficient set (core/stepper_3d.py:150-266). dt = 0.5 dx / sqrt(3). H-side
    CPML profiles on the n-1 half nodes, E-side on the interior [1:-1].

    Boundary modes (:170-215): CPML (npml > 0); the matched-sigma absorber (npml = 0,
    ``n_abs`` > 0) -- plain derivatives and the absorber sigma added to both the
    electric and magnetic damping; or mixed (both), the absorber on ``absorber_axes``
    and CPML on the others. A plain derivative is written here as the identity
    profile (b = 0, a = 0, k = 1): the memory then stays 0 and d / 1 + 0 = d exactly,
    the reference's own form for the absorber axes of mixed mode (:132-147).
    ``pmc_axes``: PMC walls instead of PEC on those axes (plain derivatives there; the
    E update keeps the wall values, see _term_pmc)."""
    dtype = np.dtype(dtype)
    dt = 0.5 * dx / math.sqrt(3.0)
    e = (np.ones((nx, ny, nz), dtype=dtype) if eps is None
         else np.asarray(eps, dtype=dtype).copy())
    dims = (nx, ny, nz)
    npml_ax = [side_counts(v) for v in _per_axis3(npml)]
    nabs_ax = [side_counts(v) for v in _per_axis3(n_abs)]
    has_pml = any(lo or hi for lo, hi in npml_ax)
    has_abs = any(lo or hi for lo, hi in nabs_ax)
    mixed = has_pml and has_abs
    plain_axes = set(absorber_axes) if mixed else ({0, 1, 2} if not has_pml else set())
    plain_axes |= set(pmc_axes)
    cp = {}
    for ax, kh, ke in ((0, "hx", "ex"), (1, "hy", "ey"), (2, "hz", "ez")):
        n = dims[ax]
        if ax in plain_axes:
            ident = lambda L: tuple(_bc(v, ax) for v in (np.zeros(L, dtype=dtype),  # noqa: E731
                                                          np.zeros(L, dtype=dtype),
                                                          np.ones(L, dtype=dtype)))
            cp[kh], cp[ke] = ident(n - 1), ident(n - 2)
            continue
        b, a, k = cpml_profiles(n - 1, npml_ax[ax], 0.5, dt, dx, dtype=dtype)
        cp[kh] = (_bc(b, ax), _bc(a, ax), _bc(k, ax))
        b, a, k = cpml_profiles(n, npml_ax[ax], 0.0, dt, dx, dtype=dtype)
        cp[ke] = (_bc(b[1:-1], ax), _bc(a[1:-1], ax), _bc(k[1:-1], ax))
    sig_bound = None
    if has_abs:
        sig_bound = np.zeros((nx, ny, nz), dtype=dtype)
        for ax in (absorber_axes if mixed else (0, 1, 2)):
            sa = absorber_sigma(dims[ax], nabs_ax[ax], dx, R0=absorber_R0, m=absorber_m,
                                dtype=dtype)
            sig_bound = np.maximum(sig_bound, _bc(sa, ax))
    # damping pairs (core/stepper_3d.py:217-235): (1, dt) without conductivity, else
    # (1 - s dt/2)/(1 + s dt/2), dt/(1 + s dt/2) with sigma_d (+ the absorber) Yee-averaged
    # onto each E component and sigma_b (+ the absorber) onto each H component
    if sigma_d is None and sigma_b is None and sig_bound is None:
        one, d2 = dtype.type(1.0), dtype.type(dt)
        damp = {k: (one, d2) for k in ("ex", "ey", "ez", "hx", "hy", "hz")}
    else:
        z = np.zeros((nx, ny, nz), dtype=dtype)
        sd = z if sigma_d is None else np.asarray(sigma_d, dtype=dtype)
        sb = z if sigma_b is None else np.asarray(sigma_b, dtype=dtype)
        if sig_bound is not None:
            sd, sb = sig_bound + sd, sig_bound + sb
        pair = lambda sg: ((1 - sg * dt / 2) / (1 + sg * dt / 2), dt / (1 + sg * dt / 2))  # noqa: E731
        damp = {"ex": pair(_avg(sd, 0)), "ey": pair(_avg(sd, 1)), "ez": pair(_avg(sd, 2)),
                "hx": pair(_avg(_avg(sb, 1), 2)), "hy": pair(_avg(_avg(sb, 0), 2)),
                "hz": pair(_avg(_avg(sb, 0), 1))}
    # ADE pole stacks per E component (core/stepper_3d.py:236-266): c1, c2 per pole,
    # c3 = v3 x the Yee-averaged mask
    pols = None
    if len(poles):
        pols = {}
        for key, shape, ax in (("x", (nx - 1, ny, nz), 0), ("y", (nx, ny - 1, nz), 1),
                               ("z", (nx, ny, nz - 1), 2)):
            n_p = len(poles)
            c3 = np.zeros((n_p,) + shape, dtype=dtype)
            c1 = np.zeros((n_p, 1, 1, 1), dtype=dtype)
            c2 = np.zeros((n_p, 1, 1, 1), dtype=dtype)
            for q, pole in enumerate(poles):
                v1, v2, v3 = pole_recurrence(pole, dt)
                m = (np.ones((nx, ny, nz), dtype=dtype) if pole_masks is None
                     else np.asarray(pole_masks[q], dtype=dtype))
                c3[q] = dtype.type(v3) * _avg(m, ax)
                c1[q], c2[q] = v1, v2
            pols[key] = (c1, c2, c3)
    return dict(dt=dt, dx=dx, dims=dims, dtype=dtype, eps=e, cpml=cp, damp=damp, pols=pols,
                pmc=tuple(pmc_axes))


def state_3d(c):
    """Zero 3D state with CPML memory and pole stacks (core/stepper_3d.py:269-292)."""
    nx, ny, nz = c["dims"]
    z = lambda *s: np.zeros(s, dtype=c["dtype"])
    pol = {}
    if c.get("pols"):
        n_p = c["pols"]["x"][2].shape[0]
        pol = dict(Px_cur=z(n_p, nx - 1, ny, nz), Px_prev=z(n_p, nx - 1, ny, nz),
                   Py_cur=z(n_p, nx, ny - 1, nz), Py_prev=z(n_p, nx, ny - 1, nz),
                   Pz_cur=z(n_p, nx, ny, nz - 1), Pz_prev=z(n_p, nx, ny, nz - 1))
    return dict(**pol,
        Ex=z(nx - 1, ny, nz), Ey=z(nx, ny - 1, nz), Ez=z(nx, ny, nz - 1),
        Hx=z(nx, ny - 1, nz - 1), Hy=z(nx - 1, ny, nz - 1), Hz=z(nx - 1, ny - 1, nz),
        psi_Ez_y=z(nx, ny - 1, nz - 1), psi_Ey_z=z(nx, ny - 1, nz - 1),
        psi_Ex_z=z(nx - 1, ny, nz - 1), psi_Ez_x=z(nx - 1, ny, nz - 1),
        psi_Ey_x=z(nx - 1, ny - 1, nz), psi_Ex_y=z(nx - 1, ny - 1, nz),
        psi_Hz_y=z(nx - 1, ny - 2, nz), psi_Hy_z=z(nx - 1, ny, nz - 2),
        psi_Hx_z=z(nx, ny - 1, nz - 2), psi_Hz_x=z(nx - 2, ny - 1, nz),
        psi_Hy_x=z(nx - 2, ny, nz - 1), psi_Hx_y=z(nx, ny - 2, nz - 1))


def _pad_interior(t, axes, pmc=()):
    """Zero pad of one cell on both sides of each axis in ``axes`` (the PEC edge of the
    tangential E), skipping PMC axes, whose terms _term_pmc already brought to full
    length (core/stepper_3d.py:86-96)."""
    pad = [(0, 0)] * 3
    for a in axes:
        if a not in pmc:
            pad[a] = (1, 1)
    return np.pad(t, pad)


def _term_pmc(t, padaxes, fullax, pmc):
    """One curl term of an E update (core/stepper_3d.py:99-121): the term that is
    full-length along ``fullax`` keeps its wall values on a PMC axis and is trimmed to
    the interior otherwise; a term along a PMC axis is zero-padded to the wall."""
    sl = [slice(None)] * 3
    pad = [(0, 0)] * 3
    for a in padaxes:
        if a == fullax:
            if a not in pmc:
                sl[a] = slice(1, -1)
        elif a in pmc:
            pad[a] = (1, 1)
    t = t[tuple(sl)]
    return np.pad(t, pad) if any(p != (0, 0) for p in pad) else t


def _ce3(c):
    dx, T = c["dx"], c["dtype"].type
    cp = c["cpml"]
    X = T(dx)

    def ce(F, ax, key, psi):
        b, a, k = cp[key]
        d = _d(F, ax) / X
        p = b * psi + a * d
        return d / k + p, p
    return ce


def step_3d(s, c, amp=0.0, src=None, point_sign=+1.0):
    """One 3D leapfrog step, CPML path of core/stepper_3d.py:363-445, then the
    soft source of :448-482. ``src`` is ("Ez", i, j, k) for a point current
    (the functional stepper ADDS dt*amp/eps there, :474-480; ``point_sign=-1``
    gives the lean stepper's subtraction, core/stepper_3d_lean.py:293-296) or
    ("Ez", mask) for an area current (subtracted, :452-461)."""
    out = step_3d_h(s, c)
    out.update(step_3d_e(s, c, out, amp, src, point_sign))
    return out


def step_3d_h(s, c):
    """H(n+1/2) and the H-side CPML memory of step_3d (core/stepper_3d.py:367-393)."""
    ce = _ce3(c)
    dm = c["damp"]
    out = {}
    ce_y, out["psi_Ez_y"] = ce(s["Ez"], 1, "hy", s["psi_Ez_y"])
    ce_z, out["psi_Ey_z"] = ce(s["Ey"], 2, "hz", s["psi_Ey_z"])
    Hx = dm["hx"][0] * s["Hx"] - dm["hx"][1] * (ce_y - ce_z)
    ce_z2, out["psi_Ex_z"] = ce(s["Ex"], 2, "hz", s["psi_Ex_z"])
    ce_x, out["psi_Ez_x"] = ce(s["Ez"], 0, "hx", s["psi_Ez_x"])
    Hy = dm["hy"][0] * s["Hy"] - dm["hy"][1] * (ce_z2 - ce_x)
    ce_x2, out["psi_Ey_x"] = ce(s["Ey"], 0, "hx", s["psi_Ey_x"])
    ce_y2, out["psi_Ex_y"] = ce(s["Ex"], 1, "hy", s["psi_Ex_y"])
    Hz = dm["hz"][0] * s["Hz"] - dm["hz"][1] * (ce_x2 - ce_y2)
    out.update(Hx=Hx, Hy=Hy, Hz=Hz)
    return out


def _e_update(s, c, key, pair, eps_c, curl, out):
    """E(n+1) of one component: (d1 E eps + d2 curl) / eps, or with poles the folded-D
    form (d1 (eps E + sum P(n)) + d2 curl - sum P(n+1)) / eps after the ADE step
    P(n+1) = c1 P(n) + c2 P(n-1) + c3 E(n) (core/stepper_3d.py:295-300, :312-325)."""
    d1, d2 = pair
    E = s["E" + key]
    if not c.get("pols"):
        return (d1 * E * eps_c + d2 * curl) / eps_c
    c1, c2, c3 = c["pols"][key]
    pc, pp = s[f"P{key}_cur"], s[f"P{key}_prev"]
    pn = c1 * pc + c2 * pp + c3 * E
    out[f"P{key}_cur"], out[f"P{key}_prev"] = pn, pc
    return (d1 * (E * eps_c + pc.sum(0)) + d2 * curl - pn.sum(0)) / eps_c


def step_3d_e(s, c, h, amp=0.0, src=None, point_sign=+1.0):
    """E(n+1), the E-side CPML memory and the soft source of step_3d
    (core/stepper_3d.py:395-482) from the state ``s`` and H(n+1/2) in ``h``."""
    ce = _ce3(c)
    dm = c["damp"]
    T = c["dtype"].type
    Hx, Hy, Hz = h["Hx"], h["Hy"], h["Hz"]
    out = {}
    eps = c["eps"]
    eps_x = _avg(eps, 0)
    pmc = c.get("pmc", ())
    ch_y, out["psi_Hz_y"] = ce(Hz, 1, "ey", s["psi_Hz_y"])
    ch_z, out["psi_Hy_z"] = ce(Hy, 2, "ez", s["psi_Hy_z"])
    curl_x = _pad_interior(_term_pmc(ch_y, (1, 2), 2, pmc) - _term_pmc(ch_z, (1, 2), 1, pmc),
                           (1, 2), pmc)
    Ex = _e_update(s, c, "x", dm["ex"], eps_x, curl_x, out)
    eps_y = _avg(eps, 1)
    ch_z2, out["psi_Hx_z"] = ce(Hx, 2, "ez", s["psi_Hx_z"])
    ch_x, out["psi_Hz_x"] = ce(Hz, 0, "ex", s["psi_Hz_x"])
    curl_y = _pad_interior(_term_pmc(ch_z2, (0, 2), 0, pmc) - _term_pmc(ch_x, (0, 2), 2, pmc),
                           (0, 2), pmc)
    Ey = _e_update(s, c, "y", dm["ey"], eps_y, curl_y, out)
    eps_z = _avg(eps, 2)
    ch_x2, out["psi_Hy_x"] = ce(Hy, 0, "ex", s["psi_Hy_x"])
    ch_y2, out["psi_Hx_y"] = ce(Hx, 1, "ey", s["psi_Hx_y"])
    curl_z = _pad_interior(_term_pmc(ch_x2, (0, 1), 1, pmc) - _term_pmc(ch_y2, (0, 1), 0, pmc),
                           (0, 1), pmc)
    Ez = _e_update(s, c, "z", dm["ez"], eps_z, curl_z, out)
    out.update(Ex=Ex, Ey=Ey, Ez=Ez)
    if src is not None and amp != 0.0:
        comp = src[0]
        epsc = {"Ex": eps_x, "Ey": eps_y, "Ez": eps_z}[comp]
        F = out[comp]
        if isinstance(src[1], np.ndarray):
            out[comp] = F - T(c["dt"] * amp) * src[1] / epsc
        else:
            i, j, k = src[1], src[2], src[3]
            F = F.copy()
            if point_sign > 0:
                F[i, j, k] = F[i, j, k] + T(c["dt"] * amp) / epsc[i, j, k]
            else:
                F[i, j, k] = F[i, j, k] - T(c["dt"] * amp) * (T(1.0) / epsc[i, j, k])
            out[comp] = F
    return out


def flux3d_planes(s, normal, idx, win=None, ap=0):
    """FluxMonitor3D._plane (core/monitors_3d.py:124-162): the two tangential
    E/H pairs on the plane (H averaged across it), cropped to the common
    min shape and then to ``win`` = (l0, h0, l1, h1) or the ``ap`` margin."""
    h = s["Ex"].dtype.type(0.5)
    if normal == "z":
        k = idx
        Ea = s["Ex"][:, :, k]; Ha = h * (s["Hy"][:, :, k - 1] + s["Hy"][:, :, k])
        Eb = s["Ey"][:, :, k]; Hb = h * (s["Hx"][:, :, k - 1] + s["Hx"][:, :, k])
    elif normal == "x":
        i = idx
        Ea = s["Ey"][i]; Ha = h * (s["Hz"][i - 1] + s["Hz"][i])
        Eb = s["Ez"][i]; Hb = h * (s["Hy"][i - 1] + s["Hy"][i])
    else:
        j = idx
        Ea = s["Ez"][:, j, :]; Ha = h * (s["Hx"][:, j - 1, :] + s["Hx"][:, j, :])
        Eb = s["Ex"][:, j, :]; Hb = h * (s["Hz"][:, j - 1, :] + s["Hz"][:, j, :])
    ts = [Ea, Ha, Eb, Hb]
    m0 = min(t.shape[0] for t in ts)
    m1 = min(t.shape[1] for t in ts)
    if win is not None:
        l0, h0, l1, h1 = win
    else:
        l0, h0, l1, h1 = ap, m0 - ap, ap, m1 - ap
    l0 = max(0, l0); l1 = max(0, l1)
    h0 = min(m0, h0); h1 = min(m1, h1)
    return [t[l0:h0, l1:h1] for t in ts]


def flux3d_sample(s, t_idx, dt, freqs, normal, idx, win=None, ap=0):
    """FluxMonitor3D.sample (core/monitors_3d.py:164-182): 8 accumulators,
    E at (t+1)dt and H at (t+1/2)dt, phase in the field dtype."""
    Ea, Ha, Eb, Hb = flux3d_planes(s, normal, idx, win, ap)
    dtype = Ea.dtype
    T = dtype.type
    f = np.asarray(freqs, dtype=dtype)
    w = (T(2 * math.pi) * f)[:, None, None]
    wE, wH = w * T((t_idx + 1.0) * dt), w * T((t_idx + 0.5) * dt)
    cE, sE, cH, sH = np.cos(wE), -np.sin(wE), np.cos(wH), -np.sin(wH)
    return T(dt) * np.stack([cE * Ea, sE * Ea, cH * Ha, sH * Ha,
                             cE * Eb, sE * Eb, cH * Hb, sH * Hb], axis=1)


def flux3d(acc, dx):
    """FluxMonitor3D.flux (core/monitors_3d.py:184-189): 1/2 sum(sa - sb) dx^2."""
    sa = acc[:, 0] * acc[:, 2] + acc[:, 1] * acc[:, 3]
    sb = acc[:, 4] * acc[:, 6] + acc[:, 5] * acc[:, 7]
    return 0.5 * (sa - sb).sum(axis=(1, 2)) * dx * dx


def run_3d(s, c, n_steps, amp_fn=None, src=None, monitors=(), point_sign=+1.0):
    """Loop of core/monitors_3d.py:192-210: step_3d, then sample and sum-fold."""
    acc = [None] * len(monitors)
    for t in range(n_steps):
        amp = amp_fn(t) if amp_fn is not None else 0.0
        s = step_3d(s, c, amp, src, point_sign=point_sign)
        for i, mon in enumerate(monitors):
            smp = mon(s, t)
            acc[i] = smp if acc[i] is None else acc[i] + smp
    return s, acc


# ---------------------------------------------------------------- CW solve (2D TM)

def bicgstab_l(ell, A, b, x, tol=1e-8, maxiters=10000, breaktol=1e-30):
    """BiCGSTAB(ell) of Sleijpen and Fokkema (ETNA 1, 11-32, 1993), in place on the
    complex vector ``x``, with the real inner product <p, q> = Re(conj(p) . q) that
    meep's solver uses (the reference's core/bicgstab.py). Stops when
    |r| <= tol |b|; returns (ierr, outer iterations): 0 converged, 1 out of
    iterations, -1 breakdown."""
    if ell < 1:
        raise ValueError("ell >= 1")

    def ip(p, q):
        return float(np.vdot(p, q).real)

    def nrm(p):
        return float(np.linalg.norm(p))
    bn = nrm(b) or 1.0
    r = [np.zeros_like(b) for _ in range(ell + 1)]
    u = [np.zeros_like(b) for _ in range(ell + 1)]
    r[0] = b - A(x)
    n0 = nrm(r[0])
    if n0 == 0.0:
        return 0, 0
    rt = r[0] / n0                                   # shadow residual, normalised
    rho0, alpha, omega = 1.0, 0.0, 1.0
    it = 0
    while nrm(r[0]) > tol * bn:
        if it >= maxiters:
            return 1, it
        it += 1
        rho0 = -omega * rho0
        # BiCG part: ell steps, building r_0..r_ell and u_0..u_ell
        for j in range(ell):
            if abs(rho0) < breaktol:
                return -1, it
            rho1 = ip(r[j], rt)
            beta = alpha * rho1 / rho0
            rho0 = rho1
            for i in range(j + 1):
                u[i] = r[i] - beta * u[i]
            u[j + 1] = A(u[j])
            alpha = rho0 / ip(u[j + 1], rt)
            for i in range(j + 1):
                r[i] = r[i] - alpha * u[i + 1]
            r[j + 1] = A(r[j])
            x += alpha * u[0]
        # minimal-residual part: modified Gram-Schmidt on r_1..r_ell
        tau = np.zeros((ell + 1, ell + 1))
        sig = np.zeros(ell + 1)
        gp = np.zeros(ell + 1)
        for j in range(1, ell + 1):
            for i in range(1, j):
                tau[i, j] = ip(r[j], r[i]) / sig[i]
                r[j] = r[j] - tau[i, j] * r[i]
            sig[j] = ip(r[j], r[j])
            gp[j] = ip(r[0], r[j]) / sig[j]
        g = np.zeros(ell + 1)
        g[ell] = gp[ell]
        omega = g[ell]
        for j in range(ell - 1, 0, -1):
            g[j] = gp[j] - sum(tau[j, i] * g[i] for i in range(j + 1, ell + 1))
        gpp = np.zeros(ell + 1)
        for j in range(1, ell):
            gpp[j] = g[j + 1] + sum(tau[j, i] * g[i + 1] for i in range(j + 1, ell))
        x += g[1] * r[0]
        r[0] = r[0] - gp[ell] * r[ell]
        u[0] = u[0] - g[ell] * u[ell]
        for j in range(1, ell):
            u[0] = u[0] - g[j] * u[j]
            x += gpp[j] * r[j]
            r[0] = r[0] - gp[j] * r[j]
    return 0, it


def cw_tm(c, freq):
    """meep's CW operator on a 2D TM coefficient set (mp/cpp/core.py:721-778):
    A x = (step(x) - x) / dt + i Omega x, Omega = (1 - exp(-2 pi i f dt)) / i dt, over
    the unknowns the step carries forward (every state array but Ez, which update_eh
    re-derives from Dz - sum P after each unpack). Returns (names, pack, unpack, A)."""
    s0 = tm_state(c)
    names = tuple(k for k in ("Hx", "Hy", "Dz", "P_cur", "P_prev", "psi_Ezy", "psi_Ezx",
                              "psi_Hyx", "psi_Hxy", "Hx0", "Hy0") if k in s0)
    shapes = {k: s0[k].shape for k in names}
    dt = c["dt"]
    iomega = (1.0 - np.exp(-2j * np.pi * freq * dt)) / dt

    def pack(re, im):
        return np.concatenate([re[k].ravel() for k in names]) + \
            1j * np.concatenate([im[k].ravel() for k in names])

    def unpack(x):
        re, im, i = dict(tm_state(c)), dict(tm_state(c)), 0
        for k in names:
            n = int(np.prod(shapes[k]))
            re[k] = x[i:i + n].real.reshape(shapes[k]).astype(c["dtype"])
            im[k] = x[i:i + n].imag.reshape(shapes[k]).astype(c["dtype"])
            i += n
        for st in (re, im):
            st["Ez"] = (st["Dz"] - st["P_cur"].sum(0)) / c["eps"]
        return re, im

    def A(x):
        re, im = unpack(x)
        return (pack(tm_step(re, c), tm_step(im, c)) - x) / dt + iomega * x
    return names, pack, unpack, A


def cw_rhs_tm(c, names, pack, amp, mask):
    """meep's right-hand side (mp/cpp/core.py:704-719): one step of source current
    into zero fields, read back and scaled by -1/dt -- amp * mask on Dz."""
    re, im = dict(tm_state(c)), dict(tm_state(c))
    re["Dz"] = re["Dz"] - c["dt"] * amp.real * mask
    im["Dz"] = im["Dz"] - c["dt"] * amp.imag * mask
    return pack(re, im) * (-1.0 / c["dt"])
