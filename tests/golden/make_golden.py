"""Generate the golden fixtures in this folder by running the REFERENCE itself.

Imports meep_torch from the reference checkout named by ``MEEP_TORCH_REF`` (read-only,
no bytecode written) and runs small seeded
cases of the hot path through its own public functions:

* ``Grid`` / ``build_tm_coeffs`` / ``LineSource`` / ``FluxMonitorTM`` /
  ``DFTFieldsMonitor`` / ``run_tm``            (core/run.py:125)
* ``build_te_coeffs`` / ``FluxMonitorTE`` / ``FluxMonitorTEY`` / ``run_te``
* ``build_3d_coeffs`` / ``PointSource3D`` / ``FluxMonitor3D`` / ``run_3d``
  (core/monitors_3d.py:192) and ``build_lean`` / ``run_3d_lean``
* ``cpml_profiles``                              (core/pml.py:17)
* d J / d eps through the reference's autograd of ``run_tm`` with
  ``checkpoint_every`` (``python make_golden.py grad`` writes only these)
* the design chain (``conic_filter``, ``tanh_projection``, ``MaterialGrid``,
  ``DesignRegion``, ``OptimizationProblem``; ``python make_golden.py design``)
* d J / d eps of ``run_3d_adjoint`` (core/adjoint3d.py:56; ``make_golden.py grad3d``,
  with conductive damping ``grad3d_sigma``, with poles ``grad3d_poles``, with PMC walls
  ``grad3d_pmc``) and of ``run_te``
  (``make_golden.py grad_te``)
* the TM and TE cases with an electric conductivity map (``sigma_d``;
  ``make_golden.py sigma``) and with magnetic conductivity and permeability maps
  (``sigma_b``, ``mu``; ``make_golden.py magnetic``), and the symmetry-folded TM and TE
  runs (mirrors, Rotate2, Rotate4; ``make_golden.py folds``), chi2 / chi3 runs
  (``make_golden.py nonlinear``), a TM run with magnetic Lorentz poles
  (``make_golden.py mpoles``), a TE run with an in-plane tensor eps
  (``make_golden.py tensor``) and the 3D matched-sigma absorber, alone and beside CPML,
  and PMC walls (``make_golden.py absorber3d``), and meep's CW solve on a 2D TM
  cell (``make_golden.py cw``), the lean 3D stepper with poles
  (``make_golden.py lean_poles``), and the TM gradient of lossy and dispersive runs
  (``make_golden.py grad_extra``) and the TM and TE cases with a Lorentz and a Drude pole
  (``make_golden.py poles``); the 3D cases with sigma_d and sigma_b
  (``make_golden.py sigma3d``) and with poles (``make_golden.py poles3d``)

in float64 and float32. Inputs (eps maps, parameters) and outputs (final
state, monitor accumulators, fluxes) are stored as ``golden_*.npz``. The
fixtures are what pins the oracle (tests/test_oracle_golden.py) and the CUDA
path (tests/test_gpu_parity.py); this script is only re-run by hand.
"""
from __future__ import annotations

import json
import math
import os
import sys

import numpy as np

sys.dont_write_bytecode = True
sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
from reference_path import reference_root  # noqa: E402
sys.path.insert(0, reference_root())

import torch  # noqa: E402

from meep_torch.core.coeffs import build_te_coeffs, build_tm_coeffs  # noqa: E402
from meep_torch.core.grid import Grid  # noqa: E402
from meep_torch.core.monitors import (DFTFieldsMonitor, FluxMonitorTE,  # noqa: E402
                                      FluxMonitorTEY, FluxMonitorTM)
from meep_torch.core.monitors_3d import FluxMonitor3D, PointSource3D, run_3d  # noqa: E402
from meep_torch.core.pml import cpml_profiles  # noqa: E402
from meep_torch.core.run import run_te, run_tm  # noqa: E402
from meep_torch.core.sources import GaussianPulse, LineSource  # noqa: E402
from meep_torch.core.stepper_3d import build_3d_coeffs, init_3d_state  # noqa: E402
from meep_torch.core.stepper_3d_lean import build_lean, run_3d_lean  # noqa: E402
from meep_torch.core.stepper_te import init_te_state  # noqa: E402
from meep_torch.core.stepper_tm import init_tm_state  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
DT = {"f64": torch.float64, "f32": torch.float32}


def _np(t):
    return t.detach().cpu().to(torch.float64).numpy()


def sigma_map(nx, ny, seed):
    """Electric conductivity: a lossy slab across the grid and a graded patch."""
    rng = np.random.default_rng(seed)
    sig = np.zeros((nx, ny))
    sig[26:31, :] = 1.5
    sig[14:20, 24:30] = rng.uniform(0.5, 4.0, (6, 6))
    return sig


def magnetic_maps(nx, ny, seed):
    """Magnetic conductivity (a lossy slab and a graded patch) and permeability (a
    block of mu in [1.5, 3])."""
    rng = np.random.default_rng(seed)
    sb = np.zeros((nx, ny))
    sb[30:34, :] = 2.0
    sb[10:16, 22:28] = rng.uniform(0.5, 3.0, (6, 6))
    mu = np.ones((nx, ny))
    mu[18:26, 6:14] = rng.uniform(1.5, 3.0, (8, 8))
    return sb, mu


POLES = [(0.7, 0.05, 1.5), (0.0, 0.1, 1.0, 0.9)]   # a Lorentz and a Drude pole


def pole_masks(nx, ny):
    """The Lorentz pole on a block across the guide, the Drude pole on a patch."""
    m0 = np.zeros((nx, ny))
    m0[22:30, 12:24] = 1.0
    m1 = np.zeros((nx, ny))
    m1[32:38, 6:12] = 1.0
    return [m0, m1]


def chi_maps(nx, ny, seed):
    """Kerr chi3 along a band and chi2 on a patch (instantaneous nonlinearity), strong
    enough at these field amplitudes to change the run well beyond the tolerances."""
    rng = np.random.default_rng(seed)
    x3 = np.zeros((nx, ny))
    x3[:, 14:22] = 100.0
    x2 = np.zeros((nx, ny))
    x2[24:32, 8:16] = rng.uniform(5.0, 20.0, (8, 8))
    return x2, x3


M_POLES = [(0.6, 0.05, 0.8), (0.9, 0.1, 0.4)]      # two magnetic Lorentz poles


def tm_case(prec, y_pmc=False, point=False, sigma=False, poles=False, magnetic=False,
            nonlinear=False, mpoles=False):
    rng = np.random.default_rng(11)
    nx, ny, dx, npml = 48, 36, 0.05, 8
    if extra == "rot4":                          # Rotate4 needs a square grid
        nx = ny = 40
    eps = np.ones((nx, ny))
    eps[:, 15:21] = 12.0                          # guide along x
    eps[20:30, 8:14] = rng.uniform(2.0, 6.0)      # a block
    g = Grid(nx=nx, ny=ny, dx=dx, dtype=DT[prec], device="cpu")
    sig = sigma_map(nx, ny, 21) if sigma else None
    kw = {} if sig is None else {"sigma_d": torch.tensor(sig, dtype=DT[prec])}
    sbm, mum = magnetic_maps(nx, ny, 23) if magnetic else (None, None)
    if magnetic:
        kw.update(sigma_b=torch.tensor(sbm, dtype=DT[prec]), mu=torch.tensor(mum, dtype=DT[prec]))
    x2m, x3m = chi_maps(nx, ny, 25) if nonlinear else (None, None)
    if nonlinear:
        kw.update(chi2=torch.tensor(x2m, dtype=DT[prec]), chi3=torch.tensor(x3m, dtype=DT[prec]))
    mpm = pole_masks(nx, ny) if mpoles else None
    if mpoles:
        kw.update(m_poles=M_POLES, m_pole_masks=[torch.tensor(m, dtype=DT[prec]) for m in mpm])
    pm = pole_masks(nx, ny) if poles else None
    if poles:
        kw.update(poles=POLES, pole_masks=[torch.tensor(m, dtype=DT[prec]) for m in pm])
    m = build_tm_coeffs(g, eps_inf=torch.tensor(eps, dtype=DT[prec]), npml=npml,
                        y_pmc=y_pmc, **kw)
    prof = GaussianPulse(0.65, 0.4)
    if point:
        src = LineSource(g, ix=12, j0=18, j1=19, profile=prof)
    else:
        src = LineSource(g, ix=12, j0=10, j1=26, profile=prof)
    freqs = [0.55, 0.65, 0.75]
    monx = FluxMonitorTM(g, freqs, x_normal=True, idx=36, lo=9, hi=27)
    mony = FluxMonitorTM(g, freqs, x_normal=False, idx=26, lo=10, hi=38)
    dft = DFTFieldsMonitor(g, freqs, component="Ez")
    s0 = init_tm_state(g, y_pmc=y_pmc, n_poles=len(POLES) if poles else 0,
                       n_mpoles=len(M_POLES) if mpoles else 0)
    n = 300
    with torch.no_grad():
        st, (ax, ay, ad) = run_tm(s0, m, n, source=src, monitors=[monx, mony, dft])
    out = dict(nx=nx, ny=ny, dx=dx, npml=npml, n_steps=n, eps=eps, freqs=np.array(freqs),
               fcen=0.65, fwidth=0.4, src_ix=12, src_j0=18 if point else 10,
               src_j1=19 if point else 26, y_pmc=int(y_pmc),
               monx=np.array([36, 9, 27]), mony=np.array([26, 10, 38]),
               acc_x=_np(ax), acc_y=_np(ay), acc_dft=_np(ad),
               flux_x=_np(monx.flux(ax, dx)), flux_y=_np(mony.flux(ay, dx)),
               mask=_np(src.mask))
    if sig is not None:
        out["sigma"] = sig
    if magnetic:
        out["sigma_b"], out["mu"] = sbm, mum
    if nonlinear:
        out["chi2"], out["chi3"] = x2m, x3m
    if mpoles:
        out["m_poles"] = json.dumps(M_POLES)
        out["m_pole_masks"] = np.stack(mpm)
    if poles:
        out["poles"] = json.dumps(POLES)
        out["pole_masks"] = np.stack(pm)
    for k in st._fields:
        v = getattr(st, k)
        if v is not None and v.numel():
            out["s_" + k] = _np(v)
    for k in ("b_hy", "a_hy", "b_hx", "a_hx", "b_ex", "a_ex", "b_ey", "a_ey"):
        out["c_" + k] = _np(getattr(m, k))
    return out


def tensor_maps(eps):
    """An in-plane anisotropic block: exx raised, a 0.5 off-diagonal on a patch."""
    exx, exy, eyy = eps.copy(), np.zeros_like(eps), eps.copy()
    exx[10:30, 6:16] += 2.0
    exy[14:26, 8:14] = 0.5
    return exx, exy, eyy


_TH = math.radians(30.0)
POLES_T = [(0.65, 0.05, (math.cos(_TH) ** 2, math.cos(_TH) * math.sin(_TH),
                         math.sin(_TH) ** 2))]              # one pole, optic axis at 30 deg


def te_case(prec, sigma=False, poles=False, magnetic=False, nonlinear=False, tensor=False,
            tensor_poles=False):
    rng = np.random.default_rng(12)
    nx, ny, dx, npml = 44, 40, 0.05, 8
    eps = np.ones((nx, ny))
    eps[:, 17:23] = 12.0
    eps[18:28, 26:32] = rng.uniform(2.0, 6.0)
    g = Grid(nx=nx, ny=ny, dx=dx, dtype=DT[prec], device="cpu")
    sig = sigma_map(nx, ny, 22) if sigma else None
    kw = {} if sig is None else {"sigma_d": torch.tensor(sig, dtype=DT[prec])}
    sbm, mum = magnetic_maps(nx, ny, 24) if magnetic else (None, None)
    if magnetic:
        kw.update(sigma_b=torch.tensor(sbm, dtype=DT[prec]), mu=torch.tensor(mum, dtype=DT[prec]))
    x2m, x3m = chi_maps(nx, ny, 26) if nonlinear else (None, None)
    if nonlinear:
        kw.update(chi2=torch.tensor(x2m, dtype=DT[prec]), chi3=torch.tensor(x3m, dtype=DT[prec]))
    tens = tensor_maps(eps) if tensor else None
    if tensor:
        kw.update(eps_tensor=tuple(torch.tensor(v, dtype=DT[prec]) for v in tens))
    tpm = pole_masks(nx, ny) if tensor_poles else None
    if tensor_poles:                      # a plain shared pole, then the oriented one
        kw.update(poles=POLES[:1], pole_masks=[torch.tensor(tpm[0], dtype=DT[prec])],
                  poles_tensor=POLES_T, pole_masks_tensor=[torch.tensor(tpm[1], dtype=DT[prec])])
    pm = pole_masks(nx, ny) if poles else None
    if poles:
        kw.update(poles=POLES, pole_masks=[torch.tensor(m, dtype=DT[prec]) for m in pm])
    m = build_te_coeffs(g, eps_inf=torch.tensor(eps, dtype=DT[prec]), npml=npml, **kw)
    prof = GaussianPulse(0.65, 0.4)
    src = LineSource(g, ix=12, j0=12, j1=28, profile=prof)

    class _TESrc:                                   # Simulation's TE binding:
        mask = src.mask[:, :-1]                     # mask[:, :-1] -> Dy (mp/simulation.py:867-869)
        amplitude = staticmethod(src.amplitude)

    freqs = [0.55, 0.65, 0.75]
    monx = FluxMonitorTE(g, freqs, ix=32, lo=9, hi=31)
    mony = FluxMonitorTEY(g, freqs, iy=30, lo=9, hi=35)
    dft = DFTFieldsMonitor(g, freqs, component="Hz")
    s0 = init_te_state(g, n_poles=len(POLES) if poles else (2 if tensor_poles else 0))
    n = 300
    with torch.no_grad():
        st, (ax, ay, ad) = run_te(s0, m, n, source=_TESrc(), monitors=[monx, mony, dft])
    out = dict(nx=nx, ny=ny, dx=dx, npml=npml, n_steps=n, eps=eps, freqs=np.array(freqs),
               fcen=0.65, fwidth=0.4, src_ix=12, src_j0=12, src_j1=28,
               monx=np.array([32, 9, 31]), mony=np.array([30, 9, 35]),
               acc_x=_np(ax), acc_y=_np(ay), acc_dft=_np(ad),
               flux_x=_np(monx.flux(ax, dx)), flux_y=_np(mony.flux(ay, dx)),
               mask=_np(_TESrc.mask))
    if sig is not None:
        out["sigma"] = sig
    if magnetic:
        out["sigma_b"], out["mu"] = sbm, mum
    if nonlinear:
        out["chi2"], out["chi3"] = x2m, x3m
    if tensor:
        out["eps_tensor"] = np.stack(tens)
    if tensor_poles:
        out["poles"] = json.dumps(POLES[:1])
        out["pole_masks"] = tpm[:1]
        out["poles_tensor"] = json.dumps(POLES_T)
        out["pole_masks_tensor"] = tpm[1:]
    if poles:
        out["poles"] = json.dumps(POLES)
        out["pole_masks"] = np.stack(pm)
    for k in st._fields:
        v = getattr(st, k)
        if v is not None and v.numel():
            out["s_" + k] = _np(v)
    return out


TM_FOLDS = {"ym_even": dict(y_mirror=1), "ym_odd": dict(y_mirror=-1),
            "xm_even": dict(x_mirror=1), "xm_odd_ym_even": dict(x_mirror=-1, y_mirror=1),
            "rot2_even": dict(y_rot2=1), "rot2_odd": dict(y_rot2=-1),
            "rot4_even": dict(rot4=1), "rot4_odd": dict(rot4=-1)}
TE_FOLDS = {"ym_even_xm_odd": dict(y_mirror=1, x_mirror=-1),
            "ym_odd_xm_even": dict(y_mirror=-1, x_mirror=1)}


def fold_case(prec, pol, fold):
    """A symmetry-folded 2D run (the low-x / low-y edges are the cuts): 40 x 40 cells,
    PML on the far sides, a dielectric block and a line source near the cut, 250
    steps, the full-grid DFT of the main component at three frequencies."""
    rng = np.random.default_rng(31)
    nx = ny = 40
    dx, npml, n = 0.05, 8, 250
    eps = np.ones((nx, ny))
    eps[6:16, 4:12] = rng.uniform(2.0, 6.0)
    eps[:, 20:24] = 8.0
    g = Grid(nx=nx, ny=ny, dx=dx, dtype=DT[prec], device="cpu")
    e = torch.tensor(eps, dtype=DT[prec])
    freqs = [0.55, 0.65, 0.75]
    src = LineSource(g, ix=5, j0=3, j1=18, profile=GaussianPulse(0.65, 0.4))
    if pol == "tm":
        m = build_tm_coeffs(g, eps_inf=e, npml=npml, **fold)
        s0 = init_tm_state(g, **fold)
        dft = DFTFieldsMonitor(g, freqs, component="Ez")
        with torch.no_grad():
            st, (ad,) = run_tm(s0, m, n, source=src, monitors=[dft])
        mask = _np(src.mask)
    else:
        m = build_te_coeffs(g, eps_inf=e, npml=npml, **fold)
        s0 = init_te_state(g)

        class _TESrc:
            mask = src.mask[:, :-1]
            amplitude = staticmethod(src.amplitude)
        dft = DFTFieldsMonitor(g, freqs, component="Hz")
        with torch.no_grad():
            st, (ad,) = run_te(s0, m, n, source=_TESrc(), monitors=[dft])
        mask = _np(_TESrc.mask)
    out = dict(nx=nx, ny=ny, dx=dx, npml=npml, n_steps=n, eps=eps, freqs=np.array(freqs),
               fcen=0.65, fwidth=0.4, src_ix=5, src_j0=3, src_j1=18, mask=mask,
               acc_dft=_np(ad), fold=json.dumps(fold))
    for k in st._fields:
        v = getattr(st, k)
        if v is not None and v.numel():
            out["s_" + k] = _np(v)
    return out


def cw_case():
    """meep's CW solve on a small 2D TM cell, assembled from the reference's own parts the
    way its Simulation.solve_cw does (mp/cpp/core.py:667-778): the unknowns are every
    state array but Ez, A x = (step(x) - x) / dt + i Omega x with update_eh(E) after each
    unpack, b = amp * mask on Dz, and its bicgstabL (L = 2). FP64. Also A applied to two
    seeded random vectors, which pins the operator itself."""
    from meep_torch.core.bicgstab import bicgstabL
    from meep_torch.core.stepper_tm import step_tm, update_eh
    nx, ny, dx, npml, freq = 40, 30, 0.05, 6, 0.6
    eps = np.ones((nx, ny))
    eps[:, 12:18] = 6.0
    g = Grid(nx=nx, ny=ny, dx=dx, dtype=torch.float64, device="cpu")
    m = build_tm_coeffs(g, eps_inf=torch.tensor(eps), npml=npml)
    st0 = init_tm_state(g)
    names = tuple(n for n in st0._fields if n != "Ez" and getattr(st0, n) is not None)
    shapes = tuple(tuple(getattr(st0, n).shape) for n in names)
    dt = m.dt
    iomega = complex((1.0 - np.exp(-2j * np.pi * freq * dt)) / dt)

    def pack(re, im):
        return (torch.cat([getattr(re, n).reshape(-1) for n in names])
                + 1j * torch.cat([getattr(im, n).reshape(-1) for n in names]))

    def unpack(x):
        out_re, out_im, i = {}, {}, 0
        for n, sh in zip(names, shapes):
            k = int(np.prod(sh))
            out_re[n] = x[i:i + k].real.reshape(sh).contiguous()
            out_im[n] = x[i:i + k].imag.reshape(sh).contiguous()
            i += k
        return (update_eh(st0._replace(**out_re), m, "E"),
                update_eh(st0._replace(**out_im), m, "E"))

    def A(x):
        re, im = unpack(x)
        return (pack(step_tm(re, m), step_tm(im, m)) - x) / dt + iomega * x

    src = LineSource(g, ix=10, j0=13, j1=17, profile=GaussianPulse(freq, 0.2))
    mask = src.mask
    b = pack(st0._replace(Dz=mask.clone()), st0._replace(Dz=torch.zeros_like(mask)))
    x = torch.zeros_like(b)
    ierr, iters = bicgstabL(2, A, b, x, tol=1e-8, maxiters=5000)
    rng = np.random.default_rng(41)
    n = b.numel()
    vs = [torch.tensor(rng.standard_normal(n) + 1j * rng.standard_normal(n)) for _ in range(2)]
    re, im = unpack(x)
    out = dict(nx=nx, ny=ny, dx=dx, npml=npml, eps=eps, freq=freq, src_ix=10, src_j0=13,
               src_j1=17, mask=_np(mask), ierr=ierr, iters=iters, names=json.dumps(names),
               b=b.numpy(), v0=vs[0].numpy(), v1=vs[1].numpy(), Av0=A(vs[0]).numpy(),
               Av1=A(vs[1]).numpy())
    for k in names:
        out["re_" + k], out["im_" + k] = _np(getattr(re, k)), _np(getattr(im, k))
    out["re_Ez"], out["im_Ez"] = _np(re.Ez), _np(im.Ez)
    return out


FACES = [("x", 5), ("x", 18), ("y", 5), ("y", 16), ("z", 5), ("z", 14)]


POLES3 = [(0.5, 0.05, 2.0), (0.0, 0.1, 1.0, 0.8)]     # a Lorentz and a Drude pole


def case_3d(prec, lean=False, sigma=False, poles=False, absorber=None, pmc=False):
    rng = np.random.default_rng(13)
    nx, ny, nz, dx, npml = 24, 22, 20, 1.0 / 16, 4
    # matched-sigma absorber on every face (npml 0), or on z beside x / y CPML
    ab = {None: {}, "abs": dict(n_abs=5), "mixed": dict(n_abs=5, absorber_axes=(2,))}[absorber]
    if pmc:                                           # PMC walls on y beside x / z CPML
        ab = dict(ab, pmc_axes=(1,))
    if absorber == "abs":
        npml = 0
    eps = np.ones((nx, ny, nz))
    for _ in range(6):                                # a few spheres, draw order
        c = rng.uniform(4, [nx - 4, ny - 4, nz - 4])
        r = rng.uniform(1.5, 3.5)
        e = rng.uniform(2, 12)
        X, Y, Z = np.meshgrid(np.arange(nx) + 0.5, np.arange(ny) + 0.5,
                              np.arange(nz) + 0.5, indexing="ij")
        eps[(X - c[0]) ** 2 + (Y - c[1]) ** 2 + (Z - c[2]) ** 2 <= r * r] = e
    epst = torch.tensor(eps, dtype=DT[prec])
    freqs = [0.4, 0.5, 0.6, 0.7]
    win = (4, 17, 4, 15)
    prof = GaussianPulse(0.5, 0.3)
    n = 120
    src_ijk = (12, 11, 10)
    if lean:
        lk = {}
        if poles:                                     # the same pole masks as the functional case
            pm3 = [np.zeros((nx, ny, nz)), np.zeros((nx, ny, nz))]
            pm3[0][8:16, 6:14, 6:14] = 1.0
            pm3[1][14:19, 12:17, 9:15] = 1.0
            lk = dict(poles=POLES3, pole_masks=[torch.tensor(m, dtype=DT[prec]) for m in pm3])
        c = build_lean(nx, ny, nz, dx, epst, npml, dtype=DT[prec], device="cpu", **lk)
        src = PointSource3D(c.dt, "Ez", *src_ijk, prof)
        mons = [FluxMonitor3D(c.dt, freqs, normal=a, idx=i, win=win, dtype=DT[prec])
                for a, i in FACES]
        view, accs = run_3d_lean(c, n, source=src, monitors=mons)
        st = {k: getattr(view, k) for k in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")}
    else:
        kw = {}
        if sigma:                                     # lossy slab (E) and a lossy patch (H)
            sd = np.zeros((nx, ny, nz))
            sd[14:18] = 2.0
            sb = np.zeros((nx, ny, nz))
            sb[6:10, 6:12, 8:14] = 3.0
            kw = dict(sigma_d=torch.tensor(sd, dtype=DT[prec]),
                      sigma_b=torch.tensor(sb, dtype=DT[prec]))
        pm3 = None
        if poles:                                     # masks off the absorbing layers
            pm3 = [np.zeros((nx, ny, nz)), np.zeros((nx, ny, nz))]
            pm3[0][8:16, 6:14, 6:14] = 1.0
            pm3[1][14:19, 12:17, 9:15] = 1.0
            kw.update(poles=POLES3, pole_masks=[torch.tensor(m, dtype=DT[prec]) for m in pm3])
        c = build_3d_coeffs(nx, ny, nz, dx, eps=epst, npml=npml, dtype=DT[prec], **kw, **ab)
        src = PointSource3D(c.dt, "Ez", *src_ijk, prof)
        mons = [FluxMonitor3D(c.dt, freqs, normal=a, idx=i, win=win, dtype=DT[prec])
                for a, i in FACES]
        s0 = init_3d_state(nx, ny, nz, npml=npml, dtype=DT[prec],
                           n_poles=len(POLES3) if poles else 0)
        with torch.no_grad():
            stt, accs = run_3d(s0, c, n, source=src, monitors=mons)
        st = {k: getattr(stt, k) for k in stt._fields if getattr(stt, k) is not None}
    out = dict(nx=nx, ny=ny, nz=nz, dx=dx, npml=npml, n_steps=n, eps=eps,
               freqs=np.array(freqs), fcen=0.5, fwidth=0.3, src=np.array(src_ijk),
               faces=json.dumps(FACES), win=np.array(win))
    if sigma:
        out["sigma_d"], out["sigma_b"] = sd, sb
    if "n_abs" in ab:
        out["n_abs"] = ab["n_abs"]
        out["absorber_axes"] = np.array(ab.get("absorber_axes", ()), dtype=np.int64)
    if pmc:
        out["pmc_axes"] = np.array(ab["pmc_axes"], dtype=np.int64)
    if poles:
        out["poles"] = json.dumps(POLES3)
        out["pole_masks"] = np.stack(pm3)
    for k, v in st.items():
        out["s_" + k] = _np(v)
    for i, (a, mon) in enumerate(zip(accs, mons)):
        out[f"acc_{i}"] = _np(a)
        out[f"flux_{i}"] = _np(mon.flux(a, dx))
    return out


def pml_case():
    out = {}
    cases = [(40, 8, 0.5, 0.025, 0.05), (40, 8, 0.0, 0.025, 0.05),
             (33, (5, 9), 0.5, 0.02, 0.04), (64, 16, 0.0, 0.018042, 1 / 16),
             (30, (0, 6), 0.0, 0.025, 0.05)]
    for i, (n, npml, off, dt, dx) in enumerate(cases):
        for prec in ("f64", "f32"):
            b, a, k = cpml_profiles(n, npml, off, dt, dx, dtype=DT[prec])
            out[f"{i}_{prec}_b"], out[f"{i}_{prec}_a"], out[f"{i}_{prec}_k"] = _np(b), _np(a), _np(k)
    out["cases"] = json.dumps(cases)
    return out


def grad_loss(st, ax, ay, ad, mx, my, dx):
    """The scalar loss of the gradient fixtures: both flux lines (frequency
    weights), the energy of the full-grid DFT and of the final fields."""
    w = torch.tensor([1.0, -0.5, 0.25], dtype=ax.dtype)
    J = ((w * mx.flux(ax, dx)).sum() + (w.flip(0) * my.flux(ay, dx)).sum()
         + 1e-3 * (ad * ad).sum() + 0.1 * (st.Ez * st.Ez).sum()
         + 0.05 * (st.Hy * st.Hy).sum() - 0.02 * (st.Hx * st.Hx).sum())
    for k, c in (("Hx0", 0.3), ("Hy0", -0.2)):     # the live on-plane lines of odd cuts
        if getattr(st, k, None) is not None:
            J = J + c * (getattr(st, k) ** 2).sum()
    return J


def grad_tm_case(prec, extra=None):
    """d J / d eps through the reference's autograd (run_tm with
    checkpoint_every, core/run.py:81-120) on the TM case's geometry; ``extra`` =
    "lossy" adds sigma_d, sigma_b and mu maps, "poles" a Lorentz and a Drude pole,
    "mpoles" two magnetic Lorentz poles,
    "pmc" PMC walls in y, "mirror" / "mirror_odd" even / odd mirror cuts on the low x and
    y edges (the CPML only on the far sides), "rot2" / "rot4" an odd Rotate2 (y cut) /
    Rotate4 (both cuts, 40 x 40)."""
    rng = np.random.default_rng(11)
    nx, ny, dx, npml = 48, 36, 0.05, 8
    if extra == "rot4":                          # Rotate4 needs a square grid
        nx = ny = 40
    eps = np.ones((nx, ny))
    eps[:, 15:21] = 12.0
    eps[20:30, 8:14] = rng.uniform(2.0, 6.0)
    eps[30:38, 20:30] = 1.0 + 4.0 * rng.random((8, 10))       # a pixelated design patch
    g = Grid(nx=nx, ny=ny, dx=dx, dtype=DT[prec], device="cpu")
    e = torch.tensor(eps, dtype=DT[prec], requires_grad=True)
    kw, out_extra = {}, {}
    if extra == "lossy":
        sd = sigma_map(nx, ny, 21)
        sbm, mum = magnetic_maps(nx, ny, 23)
        kw = dict(sigma_d=torch.tensor(sd, dtype=DT[prec]), sigma_b=torch.tensor(sbm, dtype=DT[prec]),
                  mu=torch.tensor(mum, dtype=DT[prec]))
        out_extra = dict(sigma=sd, sigma_b=sbm, mu=mum)
    elif extra == "poles":
        pm = pole_masks(nx, ny)
        kw = dict(poles=POLES, pole_masks=[torch.tensor(v, dtype=DT[prec]) for v in pm])
        out_extra = dict(poles=json.dumps(POLES), pole_masks=np.stack(pm))
    elif extra == "mpoles":
        pm = pole_masks(nx, ny)
        kw = dict(m_poles=M_POLES, m_pole_masks=[torch.tensor(v, dtype=DT[prec]) for v in pm])
        out_extra = dict(m_poles=json.dumps(M_POLES), m_pole_masks=np.stack(pm))
    if extra == "pmc":
        kw, out_extra = dict(y_pmc=True), dict(y_pmc=1)
    folds = {"mirror": dict(y_mirror=1, x_mirror=1), "mirror_odd": dict(y_mirror=-1, x_mirror=-1),
             "rot2": dict(y_rot2=-1), "rot4": dict(rot4=-1)}.get(extra, {})
    if folds:
        kw, out_extra = dict(folds), dict(fold=json.dumps(folds))
    m = build_tm_coeffs(g, eps_inf=e, npml=npml, **kw)
    src = LineSource(g, ix=12, j0=10, j1=26, profile=GaussianPulse(0.65, 0.4))
    freqs = [0.55, 0.65, 0.75]
    monx = FluxMonitorTM(g, freqs, x_normal=True, idx=36, lo=9, hi=27)
    mony = FluxMonitorTM(g, freqs, x_normal=False, idx=26, lo=10, hi=38)
    dft = DFTFieldsMonitor(g, freqs, component="Ez")
    n, ce = 200, 50
    s0 = init_tm_state(g, n_poles=len(POLES) if extra == "poles" else 0,
                       n_mpoles=len(M_POLES) if extra == "mpoles" else 0,
                       y_pmc=extra == "pmc", **folds)
    st, (ax, ay, ad) = run_tm(s0, m, n, source=src, monitors=[monx, mony, dft],
                              checkpoint_every=ce)
    J = grad_loss(st, ax, ay, ad, monx, mony, dx)
    J.backward()
    return dict(nx=nx, ny=ny, dx=dx, npml=npml, n_steps=n, checkpoint_every=ce, eps=eps,
                freqs=np.array(freqs), fcen=0.65, fwidth=0.4, src_ix=12, src_j0=10, src_j1=26,
                monx=np.array([36, 9, 27]), mony=np.array([26, 10, 38]),
                J=float(J.detach()), grad=_np(e.grad), **out_extra)


def design_case():
    """The design chain (adjoint/filters.py, adjoint/problem.py): conic filter,
    tanh projection, MaterialGrid / DesignRegion paint, and the gradient of an
    OptimizationProblem whose run function is the TM run of grad_tm_case."""
    from meep_torch.adjoint.filters import conic_filter, tanh_projection
    from meep_torch.adjoint.problem import DesignRegion, MaterialGrid, OptimizationProblem
    rng = np.random.default_rng(4)
    rho = rng.uniform(0.0, 1.0, (20, 16))
    r = torch.tensor(rho, dtype=torch.float64)
    filt = conic_filter(r, 0.15, 0.04)
    proj = tanh_projection(filt, 8.0, 0.5)
    mg = MaterialGrid((20, 16), 2.1, 12.0)
    base = torch.full((48, 36), 2.1, dtype=torch.float64)
    base[:, 15:21] = 12.0
    reg = DesignRegion(mg, ix0=22, ix1=32, iy0=10, iy1=26)
    painted = reg.paint(base, proj)
    # problem: TM run on the fixture grid, objective = transmitted flux
    nx, ny, dx, npml = 48, 36, 0.05, 8
    g = Grid(nx=nx, ny=ny, dx=dx, dtype=torch.float64, device="cpu")
    src = LineSource(g, ix=12, j0=12, j1=24, profile=GaussianPulse(0.65, 0.4))
    freqs = [0.6, 0.7]
    mon = FluxMonitorTM(g, freqs, x_normal=True, idx=38, lo=9, hi=27)

    def run_fn(eps):
        m = build_tm_coeffs(g, eps_inf=eps, npml=npml)
        st, (acc,) = run_tm(init_tm_state(g), m, 200, source=src, monitors=[mon],
                            checkpoint_every=50)
        return mon.flux(acc, dx).mean() * 1e9

    rho0 = torch.tensor(rng.uniform(0.3, 0.7, (20, 16)), dtype=torch.float64)
    opt = OptimizationProblem(run_fn, base, reg, filter_radius=0.1, dx=dx, beta=4.0, eta=0.5,
                              rho0=rho0)
    f0, grad = opt()
    return dict(rho=rho, filt=_np(filt), proj=_np(proj), base=_np(base), painted=_np(painted),
                box=np.array(reg.box), rho0=_np(rho0), f0=f0, grad=grad)


def grad3d_case(prec, sigma=False, poles=False, pmc=False):
    """d J / d eps of the reference's run_3d_adjoint (core/adjoint3d.py:56) on a
    small CPML grid with spheres, an Ez point dipole and two flux faces; ``sigma`` adds a
    lossy slab (sigma_d) and a magnetically lossy patch (sigma_b), ``poles`` a Lorentz
    and a Drude pole on two boxes inside the CPML layers, ``pmc`` PMC walls on y (no y
    CPML) with the dipole moved next to the low wall."""
    from meep_torch.core.adjoint3d import run_3d_adjoint
    rng = np.random.default_rng(13)
    n, dx, npml = 20, 1.0 / 16, 4
    eps = np.ones((n, n, n))
    ax = (np.arange(n) + 0.5) * dx
    for _ in range(6):
        cc = rng.uniform(0.35, 0.9, 3)
        r = rng.uniform(0.08, 0.2)
        inside = ((ax[:, None, None] - cc[0]) ** 2 + (ax[None, :, None] - cc[1]) ** 2 +
                  (ax[None, None, :] - cc[2]) ** 2) <= r * r
        eps[inside] = rng.uniform(2.0, 8.0)
    e = torch.tensor(eps, dtype=DT[prec], requires_grad=True)
    kw, out_extra = {}, {}
    if sigma:
        sd = np.zeros((n, n, n))
        sd[12:15] = 2.0
        sb = np.zeros((n, n, n))
        sb[5:9, 6:12, 7:13] = 3.0
        kw = dict(sigma_d=torch.tensor(sd, dtype=DT[prec]), sigma_b=torch.tensor(sb, dtype=DT[prec]))
        out_extra = dict(sigma_d=sd, sigma_b=sb)
    if poles:
        pm = [np.zeros((n, n, n)), np.zeros((n, n, n))]
        pm[0][7:13, 5:12, 8:14] = 1.0
        pm[1][11:15, 9:15, 6:11] = 1.0
        kw = dict(poles=POLES3, pole_masks=[torch.tensor(m, dtype=DT[prec]) for m in pm])
        out_extra = dict(pm0=pm[0], pm1=pm[1], poles=json.dumps(POLES3))
    src_ijk = (10, 9, 11)
    if pmc:
        kw = dict(pmc_axes=(1,))
        out_extra = dict(pmc_axes=np.array([1]))
        src_ijk = (10, 1, 11)
    c = build_3d_coeffs(n, n, n, dx, eps=e, npml=npml, device="cpu", **kw)
    src = PointSource3D(c.dt, "Ez", *src_ijk, GaussianPulse(0.9, 0.6))
    freqs = [0.7, 0.9, 1.1]
    mons = [FluxMonitor3D(c.dt, freqs, normal="x", idx=15, win=(5, 15, 5, 15)),
            FluxMonitor3D(c.dt, freqs, normal="z", idx=6, win=(5, 15, 5, 15))]
    w = torch.tensor([1.0, -0.7, 0.4], dtype=DT[prec])

    def loss_fn(accs):
        return 1e15 * ((w * mons[0].flux(accs[0], dx)).sum()
                       + (w.flip(0) * mons[1].flux(accs[1], dx)).sum()
                       + 1e-3 * sum((a * a).sum() for a in accs))

    s0 = init_3d_state(n, n, n, npml=npml, dtype=DT[prec], device="cpu",
                       n_poles=len(POLES3) if poles else 0)
    n_steps, chunk = 70, 25
    L, accs = run_3d_adjoint(c, n_steps, chunk, src, mons, loss_fn, s0)
    return dict(n=n, dx=dx, npml=npml, eps=eps, freqs=np.array(freqs), src=np.array(src_ijk),
                fcen=0.9, fwidth=0.6, n_steps=n_steps, chunk=chunk, L=float(L),
                grad=_np(e.grad), acc_0=_np(accs[0]), acc_1=_np(accs[1]), **out_extra)


def grad_loss_te(st, ad, ax, ay, mx, my, dx):
    """The loss of the TE gradient fixtures: both flux lines (frequency weights),
    the energy of the full-grid Hz DFT and of the final fields."""
    w = torch.tensor([1.0, -0.5, 0.25], dtype=ax.dtype)
    return 1e6 * ((w * mx.flux(ax, dx)).sum() + (w.flip(0) * my.flux(ay, dx)).sum()
                  + 1e-3 * (ad * ad).sum() + 0.1 * (st.Hz * st.Hz).sum()
                  + 0.05 * (st.Ex * st.Ex).sum() - 0.02 * (st.Ey * st.Ey).sum())


def grad_te_case(prec, extra=None):
    """d J / d eps_inf through the reference's autograd of run_te
    (checkpoint_every, core/run.py:81-120) on the TE case's geometry; ``extra`` =
    "lossy" adds sigma_d, sigma_b and mu maps, "poles" a Lorentz and a Drude pole on
    both E axes, "mirror" / "mirror_even" odd / even mirror cuts on the low x and y
    edges."""
    rng = np.random.default_rng(12)
    nx, ny, dx, npml = 44, 40, 0.05, 8
    eps = np.ones((nx, ny))
    eps[:, 16:24] = 12.0
    eps[26:34, 22:32] = 1.0 + 4.0 * rng.random((8, 10))
    g = Grid(nx=nx, ny=ny, dx=dx, dtype=DT[prec], device="cpu")
    e = torch.tensor(eps, dtype=DT[prec], requires_grad=True)
    kw, out_extra = {}, {}
    if extra == "lossy":
        sd = sigma_map(nx, ny, 21)
        sbm, mum = magnetic_maps(nx, ny, 23)
        kw = dict(sigma_d=torch.tensor(sd, dtype=DT[prec]), sigma_b=torch.tensor(sbm, dtype=DT[prec]),
                  mu=torch.tensor(mum, dtype=DT[prec]))
        out_extra = dict(sigma=sd, sigma_b=sbm, mu=mum)
    elif extra == "poles":
        pm = pole_masks(nx, ny)
        kw = dict(poles=POLES, pole_masks=[torch.tensor(v, dtype=DT[prec]) for v in pm])
        out_extra = dict(poles=json.dumps(POLES), pole_masks=np.stack(pm))
    elif extra in ("mirror", "mirror_even"):
        folds = dict(y_mirror=-1, x_mirror=-1) if extra == "mirror" else dict(y_mirror=1,
                                                                              x_mirror=1)
        kw, out_extra = dict(folds), dict(fold=json.dumps(folds))
    m = build_te_coeffs(g, eps_inf=e, npml=npml, **kw)
    line = LineSource(g, ix=12, j0=14, j1=26, profile=GaussianPulse(0.65, 0.4))

    class _TESrc:                                   # TE binding: mask[:, :-1] -> Dy
        mask = line.mask[:, :-1]
        amplitude = staticmethod(line.amplitude)

    src = _TESrc()
    freqs = [0.55, 0.65, 0.75]
    dft = DFTFieldsMonitor(g, freqs, component="Hz")
    monx = FluxMonitorTE(g, freqs, ix=33, lo=10, hi=30)
    mony = FluxMonitorTEY(g, freqs, iy=30, lo=10, hi=34)
    n, ce = 180, 60
    s0 = init_te_state(g, n_poles=len(POLES) if extra == "poles" else 0)
    st, (ad, ax, ay) = run_te(s0, m, n, source=src, monitors=[dft, monx, mony],
                              checkpoint_every=ce)
    J = grad_loss_te(st, ad, ax, ay, monx, mony, dx)
    J.backward()
    return dict(nx=nx, ny=ny, dx=dx, npml=npml, n_steps=n, checkpoint_every=ce, eps=eps,
                freqs=np.array(freqs), fcen=0.65, fwidth=0.4, src_ix=12, src_j0=14, src_j1=26,
                monx=np.array([33, 10, 30]), mony=np.array([30, 10, 34]),
                J=float(J.detach()), grad=_np(e.grad), **out_extra)


def main():
    if sys.argv[1:] == ["sigma3d"]:
        for prec in ("f64", "f32"):
            np.savez_compressed(os.path.join(HERE, f"golden_3d_sigma_{prec}.npz"),
                                **case_3d(prec, sigma=True))
        return
    if sys.argv[1:] == ["poles3d"]:
        for prec in ("f64", "f32"):
            np.savez_compressed(os.path.join(HERE, f"golden_3d_poles_{prec}.npz"),
                                **case_3d(prec, poles=True))
        return
    if sys.argv[1:] == ["poles"]:
        for prec in ("f64", "f32"):
            np.savez_compressed(os.path.join(HERE, f"golden_tm_poles_{prec}.npz"),
                                **tm_case(prec, poles=True))
            np.savez_compressed(os.path.join(HERE, f"golden_te_poles_{prec}.npz"),
                                **te_case(prec, poles=True))
        return
    if sys.argv[1:] == ["folds"]:
        for prec in ("f64", "f32"):
            for pol, folds in (("tm", TM_FOLDS), ("te", TE_FOLDS)):
                for name, fold in folds.items():
                    np.savez_compressed(os.path.join(HERE, f"golden_{pol}_fold_{name}_{prec}.npz"),
                                        **fold_case(prec, pol, fold))
        return
    if sys.argv[1:] == ["grad3d_sigma"]:
        np.savez_compressed(os.path.join(HERE, "golden_grad3d_sigma_f64.npz"),
                            **grad3d_case("f64", sigma=True))
        return
    if sys.argv[1:] == ["grad3d_poles"]:
        np.savez_compressed(os.path.join(HERE, "golden_grad3d_poles_f64.npz"),
                            **grad3d_case("f64", poles=True))
        return
    if sys.argv[1:] == ["grad3d_pmc"]:
        np.savez_compressed(os.path.join(HERE, "golden_grad3d_pmc_f64.npz"),
                            **grad3d_case("f64", pmc=True))
        return
    if sys.argv[1:] == ["grad_mpoles"]:
        np.savez_compressed(os.path.join(HERE, "golden_grad_tm_mpoles_f64.npz"),
                            **grad_tm_case("f64", "mpoles"))
        return
    if sys.argv[1:] == ["grad_cut_lines"]:
        for name in ("mirror_odd", "rot2", "rot4"):
            np.savez_compressed(os.path.join(HERE, f"golden_grad_tm_{name}_f64.npz"),
                                **grad_tm_case("f64", name))
        return
    if sys.argv[1:] == ["grad_mirror"]:
        np.savez_compressed(os.path.join(HERE, "golden_grad_tm_mirror_f64.npz"),
                            **grad_tm_case("f64", "mirror"))
        np.savez_compressed(os.path.join(HERE, "golden_grad_te_mirror_f64.npz"),
                            **grad_te_case("f64", "mirror"))
        np.savez_compressed(os.path.join(HERE, "golden_grad_te_mirror_even_f64.npz"),
                            **grad_te_case("f64", "mirror_even"))
        return
    if sys.argv[1:] == ["grad_pmc"]:
        np.savez_compressed(os.path.join(HERE, "golden_grad_tm_pmc_f64.npz"),
                            **grad_tm_case("f64", "pmc"))
        return
    if sys.argv[1:] == ["grad_extra"]:
        for extra in ("lossy", "poles"):
            np.savez_compressed(os.path.join(HERE, f"golden_grad_tm_{extra}_f64.npz"),
                                **grad_tm_case("f64", extra))
        return
    if sys.argv[1:] == ["grad_extra_te"]:
        for extra in ("lossy", "poles"):
            np.savez_compressed(os.path.join(HERE, f"golden_grad_te_{extra}_f64.npz"),
                                **grad_te_case("f64", extra))
        return
    if sys.argv[1:] == ["lean_poles"]:
        for prec in ("f64", "f32"):
            np.savez_compressed(os.path.join(HERE, f"golden_3d_lean_poles_{prec}.npz"),
                                **case_3d(prec, lean=True, poles=True))
        return
    if sys.argv[1:] == ["cw"]:
        np.savez_compressed(os.path.join(HERE, "golden_cw_tm_f64.npz"), **cw_case())
        return
    if sys.argv[1:] == ["absorber3d"]:
        for prec in ("f64", "f32"):
            for mode in ("abs", "mixed"):
                np.savez_compressed(os.path.join(HERE, f"golden_3d_{mode}_{prec}.npz"),
                                    **case_3d(prec, absorber=mode))
            np.savez_compressed(os.path.join(HERE, f"golden_3d_pmc_{prec}.npz"),
                                **case_3d(prec, pmc=True))
        return
    if sys.argv[1:] == ["tensor"]:
        for prec in ("f64", "f32"):
            np.savez_compressed(os.path.join(HERE, f"golden_te_tensor_{prec}.npz"),
                                **te_case(prec, tensor=True))
            np.savez_compressed(os.path.join(HERE, f"golden_te_tensor_poles_{prec}.npz"),
                                **te_case(prec, tensor_poles=True))
        return
    if sys.argv[1:] == ["mpoles"]:
        for prec in ("f64", "f32"):
            np.savez_compressed(os.path.join(HERE, f"golden_tm_mpoles_{prec}.npz"),
                                **tm_case(prec, mpoles=True))
        return
    if sys.argv[1:] == ["nonlinear"]:
        for prec in ("f64", "f32"):
            np.savez_compressed(os.path.join(HERE, f"golden_tm_nonlinear_{prec}.npz"),
                                **tm_case(prec, nonlinear=True))
            np.savez_compressed(os.path.join(HERE, f"golden_te_nonlinear_{prec}.npz"),
                                **te_case(prec, nonlinear=True))
        return
    if sys.argv[1:] == ["magnetic"]:
        for prec in ("f64", "f32"):
            np.savez_compressed(os.path.join(HERE, f"golden_tm_magnetic_{prec}.npz"),
                                **tm_case(prec, magnetic=True))
            np.savez_compressed(os.path.join(HERE, f"golden_te_magnetic_{prec}.npz"),
                                **te_case(prec, magnetic=True))
        return
    if sys.argv[1:] == ["sigma"]:
        for prec in ("f64", "f32"):
            np.savez_compressed(os.path.join(HERE, f"golden_tm_sigma_{prec}.npz"),
                                **tm_case(prec, sigma=True))
            np.savez_compressed(os.path.join(HERE, f"golden_te_sigma_{prec}.npz"),
                                **te_case(prec, sigma=True))
        return
    if sys.argv[1:] == ["grad_te"]:
        for prec in ("f64", "f32"):
            np.savez_compressed(os.path.join(HERE, f"golden_grad_te_{prec}.npz"),
                                **grad_te_case(prec))
        return
    if sys.argv[1:] == ["grad3d"]:
        for prec in ("f64", "f32"):
            np.savez_compressed(os.path.join(HERE, f"golden_grad3d_{prec}.npz"),
                                **grad3d_case(prec))
        return
    if sys.argv[1:] == ["design"]:
        np.savez_compressed(os.path.join(HERE, "golden_design.npz"), **design_case())
        return
    if sys.argv[1:] == ["grad"]:
        for prec in ("f64", "f32"):
            np.savez_compressed(os.path.join(HERE, f"golden_grad_tm_{prec}.npz"),
                                **grad_tm_case(prec))
        return
    torch.set_num_threads(4)
    np.savez_compressed(os.path.join(HERE, "golden_pml.npz"), **pml_case())
    for prec in ("f64", "f32"):
        np.savez_compressed(os.path.join(HERE, f"golden_tm_{prec}.npz"), **tm_case(prec))
        np.savez_compressed(os.path.join(HERE, f"golden_tm_point_pmc_{prec}.npz"),
                            **tm_case(prec, y_pmc=True, point=True))
        np.savez_compressed(os.path.join(HERE, f"golden_te_{prec}.npz"), **te_case(prec))
        np.savez_compressed(os.path.join(HERE, f"golden_3d_{prec}.npz"), **case_3d(prec))
        np.savez_compressed(os.path.join(HERE, f"golden_3d_lean_{prec}.npz"),
                            **case_3d(prec, lean=True))
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
