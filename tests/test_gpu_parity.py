"""Parity of the CUDA path with the reference (golden fixtures made by running
meep_torch itself) and with the oracle, through the package's public API and
therefore the C ABI.

Bar (the parity tolerance): relative L2 <= 1e-4 against the reference's
float32 run on fields, DFT accumulators and fluxes. The error against the
reference's float64 run is computed and printed for each case.
"""
import json

import numpy as np
import pytest
import torch

from oracle import fdtd as O
from tests.conftest import load_golden, rel_l2

pytestmark = pytest.mark.gpu

TOL = 1e-4


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    from meep_torch_b200 import build
    build.build()


def dev():
    return "cuda"


def _report(name, errs32, errs64):
    print(f"\n[{name}] max relL2 vs ref fp32: {max(errs32.values()):.2e}  "
          f"vs ref fp64: {max(errs64.values()):.2e}")


def run_tm_case(case, phase_mode="exact"):
    from meep_torch_b200.core.coeffs import build_tm_coeffs
    from meep_torch_b200.core.grid import Grid
    from meep_torch_b200.core.monitors import DFTFieldsMonitor, FluxMonitorTM
    from meep_torch_b200.core.run import run_tm
    from meep_torch_b200.core.sources import GaussianPulse, LineSource
    from meep_torch_b200.core.stepper_tm import init_tm_state
    g = load_golden(f"{case}_f32")
    nx, ny, dx = int(g["nx"]), int(g["ny"]), float(g["dx"])
    pmc = bool(g["y_pmc"])
    grid = Grid(nx=nx, ny=ny, dx=dx, device=dev())
    sig = g.get("sigma")
    poles = json.loads(str(g["poles"])) if "poles" in g else ()
    pm = [torch.tensor(x, dtype=torch.float32) for x in g["pole_masks"]] if poles else None
    mag = {k: torch.tensor(g[k], dtype=torch.float32)
           for k in ("sigma_b", "mu", "chi2", "chi3") if k in g}
    n_mp = 0
    if "m_poles" in g:
        mag.update(m_poles=json.loads(str(g["m_poles"])),
                   m_pole_masks=[torch.tensor(x, dtype=torch.float32) for x in g["m_pole_masks"]])
        n_mp = len(mag["m_poles"])
    m = build_tm_coeffs(grid, eps_inf=torch.tensor(g["eps"], dtype=torch.float32),
                        npml=int(g["npml"]), y_pmc=pmc,
                        sigma_d=None if sig is None else torch.tensor(sig, dtype=torch.float32),
                        poles=poles, pole_masks=pm, **mag)
    src = LineSource(grid, ix=int(g["src_ix"]), j0=int(g["src_j0"]), j1=int(g["src_j1"]),
                     profile=GaussianPulse(float(g["fcen"]), float(g["fwidth"])))
    freqs = [float(f) for f in g["freqs"]]
    mx, my = (int(v) for v in g["monx"]), (int(v) for v in g["mony"])
    ix, xlo, xhi = mx
    iy, ylo, yhi = my
    monx = FluxMonitorTM(grid, freqs, x_normal=True, idx=ix, lo=xlo, hi=xhi)
    mony = FluxMonitorTM(grid, freqs, x_normal=False, idx=iy, lo=ylo, hi=yhi)
    dft = DFTFieldsMonitor(grid, freqs, "Ez")
    st, accs = run_tm(init_tm_state(grid, y_pmc=pmc, n_poles=len(poles), n_mpoles=n_mp), m,
                      int(g["n_steps"]),
                      source=src, monitors=[monx, mony, dft], phase_mode=phase_mode)
    fx, fy = monx.flux(accs[0], dx), mony.flux(accs[1], dx)
    return st, accs, (fx, fy)


@pytest.mark.parametrize("case", ["tm", "tm_point_pmc", "tm_sigma", "tm_poles",
                                  "tm_magnetic", "tm_nonlinear", "tm_mpoles"])
def test_tm_matches_reference(case):
    st, accs, (fx, fy) = run_tm_case(case)
    e32, e64 = {}, {}
    for prec, errs in (("f32", e32), ("f64", e64)):
        g = load_golden(f"{case}_{prec}")
        names = ["Ez", "Hx", "Hy", "Dz", "psi_Ezy", "psi_Ezx", "psi_Hyx", "psi_Hxy"]
        if "s_P_cur" in g:
            names += ["P_cur", "P_prev"]
        names += [k for k in ("Bx", "By", "Mx_cur", "Mx_prev", "My_cur", "My_prev")
                  if "s_" + k in g]
        for k in names:
            errs[k] = rel_l2(getattr(st, k).cpu().numpy(), g["s_" + k])
        for a, key in zip(accs, ("acc_x", "acc_y", "acc_dft")):
            errs[key] = rel_l2(a.cpu().numpy(), g[key])
        errs["flux_x"] = rel_l2(fx.cpu().numpy(), g["flux_x"])
        errs["flux_y"] = rel_l2(fy.cpu().numpy(), g["flux_y"])
    _report(case, e32, e64)
    bad = {k: v for k, v in e32.items() if not v < TOL}
    assert not bad, bad


FOLD_CASES = [("tm", "ym_even"), ("tm", "ym_odd"), ("tm", "xm_even"), ("tm", "xm_odd_ym_even"),
              ("tm", "rot2_even"), ("tm", "rot2_odd"), ("tm", "rot4_even"), ("tm", "rot4_odd"),
              ("te", "ym_even_xm_odd"), ("te", "ym_odd_xm_even")]


@pytest.mark.parametrize("pol,fold", FOLD_CASES)
def test_fold_matches_reference(pol, fold):
    """Symmetry-folded runs (core/stepper_tm.py:85-166, core/stepper_te.py:73-111):
    mirrors, Rotate2 and Rotate4 at the low-x / low-y edges, absorber on the far sides, a
    line source beside the cut; every state array (the on-plane Hx0 / Hy0 lines and the
    CPML memory from the cut row included) and the full-grid DFT, 250 steps."""
    from meep_torch_b200.core.coeffs import build_te_coeffs, build_tm_coeffs
    from meep_torch_b200.core.grid import Grid
    from meep_torch_b200.core.monitors import DFTFieldsMonitor
    from meep_torch_b200.core.run import run_te, run_tm
    from meep_torch_b200.core.sources import GaussianPulse, LineSource, TESource
    from meep_torch_b200.core.stepper_te import init_te_state
    from meep_torch_b200.core.stepper_tm import init_tm_state
    name = f"{pol}_fold_{fold}"
    g = load_golden(f"{name}_f32")
    kw = json.loads(str(g["fold"]))
    nx, ny, dx = int(g["nx"]), int(g["ny"]), float(g["dx"])
    grid = Grid(nx=nx, ny=ny, dx=dx, device=dev())
    eps = torch.tensor(g["eps"], dtype=torch.float32)
    src = LineSource(grid, ix=int(g["src_ix"]), j0=int(g["src_j0"]), j1=int(g["src_j1"]),
                     profile=GaussianPulse(float(g["fcen"]), float(g["fwidth"])))
    freqs = [float(f) for f in g["freqs"]]
    if pol == "tm":
        m = build_tm_coeffs(grid, eps_inf=eps, npml=int(g["npml"]), **kw)
        dft = DFTFieldsMonitor(grid, freqs, "Ez")
        st, (acc,) = run_tm(init_tm_state(grid, **kw), m, int(g["n_steps"]), source=src,
                            monitors=[dft])
    else:
        m = build_te_coeffs(grid, eps_inf=eps, npml=int(g["npml"]), **kw)
        src = TESource(src)
        dft = DFTFieldsMonitor(grid, freqs, "Hz")
        st, (acc,) = run_te(init_te_state(grid), m, int(g["n_steps"]), source=src,
                            monitors=[dft])
    np.testing.assert_array_equal(src.mask.cpu().numpy(), g["mask"])
    e32, e64 = {}, {}
    for prec, errs in (("f32", e32), ("f64", e64)):
        gg = load_golden(f"{name}_{prec}")
        keys = [k[2:] for k in gg if k.startswith("s_")]
        assert not [k for k in st._fields if getattr(st, k) is not None
                    and getattr(st, k).numel() and k not in keys]
        for k in keys:
            errs[k] = rel_l2(getattr(st, k).cpu().numpy(), gg["s_" + k])
        errs["acc_dft"] = rel_l2(acc.cpu().numpy(), gg["acc_dft"])
    _report(name, e32, e64)
    bad = {k: v for k, v in e32.items() if not v < TOL}
    assert not bad, bad


def test_tm_reference_phase_mode():
    """The float32 phase emulation reproduces the reference's own float32
    DFT phase arithmetic (core/monitors.py:43-46)."""
    st, accs, (fx, fy) = run_tm_case("tm", phase_mode="reference_fp32")
    g = load_golden("tm_f32")
    for a, key in zip(accs, ("acc_x", "acc_y", "acc_dft")):
        assert rel_l2(a.cpu().numpy(), g[key]) < TOL, key


@pytest.mark.parametrize("case", ["te", "te_sigma", "te_poles", "te_magnetic", "te_tensor",
                                  "te_tensor_poles", "te_nonlinear"])
def test_te_matches_reference(case):
    from meep_torch_b200.core.coeffs import build_te_coeffs
    from meep_torch_b200.core.grid import Grid
    from meep_torch_b200.core.monitors import DFTFieldsMonitor, FluxMonitorTE, FluxMonitorTEY
    from meep_torch_b200.core.run import run_te
    from meep_torch_b200.core.sources import GaussianPulse, LineSource, TESource
    from meep_torch_b200.core.stepper_te import init_te_state
    g = load_golden(f"{case}_f32")
    nx, ny, dx = int(g["nx"]), int(g["ny"]), float(g["dx"])
    grid = Grid(nx=nx, ny=ny, dx=dx, device=dev())
    sig = g.get("sigma")
    poles = json.loads(str(g["poles"])) if "poles" in g else ()
    pm = [torch.tensor(x, dtype=torch.float32) for x in g["pole_masks"]] if poles else None
    mag = {k: torch.tensor(g[k], dtype=torch.float32)
           for k in ("sigma_b", "mu", "chi2", "chi3") if k in g}
    # in-plane tensor eps, oriented poles, chi2 / chi3: the three-pass TE kernels
    if "eps_tensor" in g:
        mag["eps_tensor"] = tuple(torch.tensor(v, dtype=torch.float32) for v in g["eps_tensor"])
    n_pt = 0
    if "poles_tensor" in g:
        pt = [(p[0], p[1], tuple(p[2]), *p[3:]) for p in json.loads(str(g["poles_tensor"]))]
        mag.update(poles_tensor=pt, pole_masks_tensor=[torch.tensor(x, dtype=torch.float32)
                                                       for x in g["pole_masks_tensor"]])
        n_pt = len(pt)
    m = build_te_coeffs(grid, eps_inf=torch.tensor(g["eps"], dtype=torch.float32),
                        npml=int(g["npml"]), poles=poles, pole_masks=pm,
                        sigma_d=None if sig is None else torch.tensor(sig, dtype=torch.float32),
                        **mag)
    src = TESource(LineSource(grid, ix=int(g["src_ix"]), j0=int(g["src_j0"]),
                              j1=int(g["src_j1"]),
                              profile=GaussianPulse(float(g["fcen"]), float(g["fwidth"]))))
    freqs = [float(f) for f in g["freqs"]]
    ix, xlo, xhi = (int(v) for v in g["monx"])
    iy, ylo, yhi = (int(v) for v in g["mony"])
    monx = FluxMonitorTE(grid, freqs, ix=ix, lo=xlo, hi=xhi)
    mony = FluxMonitorTEY(grid, freqs, iy=iy, lo=ylo, hi=yhi)
    dft = DFTFieldsMonitor(grid, freqs, "Hz")
    st, accs = run_te(init_te_state(grid, n_poles=len(poles) + n_pt), m, int(g["n_steps"]),
                      source=src, monitors=[monx, mony, dft])
    fx, fy = monx.flux(accs[0], dx), mony.flux(accs[1], dx)
    e32, e64 = {}, {}
    for prec, errs in (("f32", e32), ("f64", e64)):
        gg = load_golden(f"{case}_{prec}")
        names = ["Hz", "Ex", "Ey", "Dx", "Dy", "psi_Eyx", "psi_Exy", "psi_Hzy", "psi_Hzx"]
        if "s_Px_cur" in gg:
            names += ["Px_cur", "Px_prev", "Py_cur", "Py_prev"]
        for k in names:
            errs[k] = rel_l2(getattr(st, k).cpu().numpy(), gg["s_" + k])
        for a, key in zip(accs, ("acc_x", "acc_y", "acc_dft")):
            errs[key] = rel_l2(a.cpu().numpy(), gg[key])
        errs["flux_x"] = rel_l2(fx.cpu().numpy(), gg["flux_x"])
        errs["flux_y"] = rel_l2(fy.cpu().numpy(), gg["flux_y"])
    _report(case, e32, e64)
    bad = {k: v for k, v in e32.items() if not v < TOL}
    assert not bad, bad


def _run3d(lean, variant=0, case=None):
    from meep_torch_b200.core.monitors_3d import FluxMonitor3D, PointSource3D, run_3d
    from meep_torch_b200.core.sources import GaussianPulse
    from meep_torch_b200.core.stepper_3d import build_3d_coeffs, init_3d_state
    from meep_torch_b200.core.stepper_3d_lean import build_lean, run_3d_lean
    g = load_golden(f"{case}_f32" if case else ("3d_lean_f32" if lean else "3d_f32"))
    nx, ny, nz, dx, npml = (int(g["nx"]), int(g["ny"]), int(g["nz"]), float(g["dx"]),
                            int(g["npml"]))
    eps = torch.tensor(g["eps"], dtype=torch.float32)
    freqs = [float(f) for f in g["freqs"]]
    win = tuple(int(v) for v in g["win"])
    faces = json.loads(str(g["faces"]))
    prof = GaussianPulse(float(g["fcen"]), float(g["fwidth"]))
    i, j, k = (int(v) for v in g["src"])
    if lean:
        lk = {}
        if "poles" in g:
            lk = dict(poles=json.loads(str(g["poles"])),
                      pole_masks=[torch.tensor(m, dtype=torch.float32) for m in g["pole_masks"]])
        c = build_lean(nx, ny, nz, dx, eps, npml, device=dev(), **lk)
        dt = c.dt
    else:
        kw = {}
        if "sigma_d" in g:
            kw = dict(sigma_d=torch.tensor(g["sigma_d"], dtype=torch.float32),
                      sigma_b=torch.tensor(g["sigma_b"], dtype=torch.float32))
        if "poles" in g:
            kw = dict(poles=json.loads(str(g["poles"])),
                      pole_masks=[torch.tensor(m, dtype=torch.float32) for m in g["pole_masks"]])
        if "n_abs" in g:
            kw.update(n_abs=int(g["n_abs"]),
                      absorber_axes=tuple(int(a) for a in g["absorber_axes"]))
        if "pmc_axes" in g:
            kw.update(pmc_axes=tuple(int(a) for a in g["pmc_axes"]))
        c = build_3d_coeffs(nx, ny, nz, dx, eps=eps, npml=npml, device=dev(), **kw)
        dt = c.dt
    src = PointSource3D(dt, "Ez", i, j, k, prof)
    mons = [FluxMonitor3D(dt, freqs, normal=a, idx=idx, win=win) for a, idx in faces]
    if lean:
        view, accs = run_3d_lean(c, int(g["n_steps"]), source=src, monitors=mons,
                                 variant=variant)
        st = {kk: getattr(view, kk) for kk in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")}
    else:
        n_p = len(json.loads(str(g["poles"]))) if "poles" in g else 0
        s, accs = run_3d(init_3d_state(nx, ny, nz, npml=npml, device=dev(), n_poles=n_p), c,
                         int(g["n_steps"]), source=src, monitors=mons, variant=variant)
        st = s._asdict()
    return st, accs, mons, dx


@pytest.mark.parametrize("variant,lean,case", [(1, False, None), (2, False, None),
                                                (3, False, None), (1, True, None),
                                                (2, True, None), (3, True, None),
                                                (2, False, "3d_sigma"), (2, False, "3d_poles"),
                                                (2, False, "3d_abs"), (2, False, "3d_mixed"),
                                                (2, False, "3d_pmc"), (3, False, "3d_pmc"),
                                                (2, True, "3d_lean_poles")])
def test_3d_matches_reference(lean, variant, case):
    """3D golden cases; 3d_sigma adds conductive damping (sigma_d on E, sigma_b on H);
    3d_abs is the matched-sigma absorber on every face (no CPML), 3d_mixed the absorber
    on z beside x / y CPML (core/stepper_3d.py:150-235); 3d_pmc puts PMC walls on y
    beside x / z CPML (core/stepper_3d.py _term_pmc / _pad_interior), on the split and the
    one-pass kernels."""
    st, accs, mons, dx = _run3d(lean, variant, case)
    name = case or ("3d_lean" if lean else "3d")
    e32, e64 = {}, {}
    for prec, errs in (("f32", e32), ("f64", e64)):
        g = load_golden(f"{name}_{prec}")
        keys = ["Ex", "Ey", "Ez", "Hx", "Hy", "Hz"]
        if not lean and case != "3d_abs":
            keys += ["psi_Ez_y", "psi_Hx_y", "psi_Hz_x", "psi_Hy_z", "psi_Ex_z"]
            keys += [k[2:] for k in g if k.startswith("s_P")]
        for k in keys:
            errs[k] = rel_l2(st[k].cpu().numpy(), g["s_" + k])
        for n, (a, mon) in enumerate(zip(accs, mons)):
            errs[f"acc_{n}"] = rel_l2(a.cpu().numpy(), g[f"acc_{n}"])
            errs[f"flux_{n}"] = rel_l2(mon.flux(a, dx).cpu().numpy(), g[f"flux_{n}"])
    _report(name, e32, e64)
    bad = {k: v for k, v in e32.items() if not v < TOL}
    assert not bad, bad


# ------------------------------------------------------------------ oracle parity

def _oracle_tm(nx, ny, dx, eps, npml, n, ix, j0, j1, freqs, mons_spec, fcen=0.65, fw=0.3,
               y_pmc=False, s0=None):
    c = O.tm_coeffs(nx, ny, dx, eps=eps, npml=npml, y_pmc=y_pmc, dtype=np.float32)
    mask = O.line_source_mask(nx, ny, dx, ix, j0, j1, dtype=np.float32)
    prof = O.gaussian_pulse(fcen, fw)
    dt = c["dt"]
    mons = []
    for xn, idx, lo, hi in mons_spec:
        mons.append((lambda xn, idx, lo, hi: lambda s, t: O.flux_tm_sample(
            s, t, dt, freqs, xn, idx, lo, hi, np.float32))(xn, idx, lo, hi))
    mons.append(lambda s, t: O.dft_sample(s["Ez"], t, dt, freqs, "Ez", np.float32))
    s, acc = O.run_2d(O.tm_step, s0 if s0 is not None else O.tm_state(c), c, n,
                      amp_fn=lambda t: prof(O.src_time(t, dt)), mask=mask, monitors=mons)
    return s, acc


def _oracle_te(nx, ny, dx, eps, npml, n, ix, j0, j1, freqs, fcen=0.65, fw=0.3, mon=None):
    c = O.te_coeffs(nx, ny, dx, eps=eps, npml=npml, dtype=np.float32)
    mask = O.line_source_mask(nx, ny, dx, ix, j0, j1, dtype=np.float32)[:, :-1]
    prof = O.gaussian_pulse(fcen, fw)
    dt = c["dt"]
    mons = [lambda s, t: O.dft_sample(s["Hz"], t, dt, freqs, "Hz", np.float32)]
    if mon is not None:
        mx, my = mon
        mons.append(lambda s, t: O.flux_te_sample(s, t, dt, freqs, *mx, np.float32))
        mons.append(lambda s, t: O.flux_tey_sample(s, t, dt, freqs, *my, np.float32))
    return O.run_2d(O.te_step, O.te_state(c), c, n,
                    amp_fn=lambda t: prof(O.src_time(t, dt)), mask=mask, monitors=mons)


@pytest.mark.parametrize("variant", [1, 2, 3])
def test_batched_mixed_tm_te_matches_oracle(variant):
    """One plan advancing TM and TE structures of different, odd sizes whose
    widths span several 128-column strips and rows several warp segments."""
    from meep_torch_b200.core.coeffs import build_te_coeffs, build_tm_coeffs
    from meep_torch_b200.core.grid import Grid
    from meep_torch_b200.core.monitors import (DFTFieldsMonitor, FluxMonitorTE, FluxMonitorTEY,
                                               FluxMonitorTM)
    from meep_torch_b200.core.sources import GaussianPulse, LineSource, TESource
    from meep_torch_b200.core.stepper_te import init_te_state
    from meep_torch_b200.core.stepper_tm import init_tm_state
    from meep_torch_b200.engine2d import Engine2D
    rng = np.random.default_rng(5)
    freqs = [0.55, 0.65, 0.75]
    specs = [("tm", 70, 261), ("te", 83, 133), ("tm", 129, 130), ("te", 45, 300)]
    items, refs = [], []
    n = 120
    for pol, nx, ny in specs:
        eps = np.ones((nx, ny))
        eps[10:nx - 10, ny // 2 - 5: ny // 2 + 5] = 12.0
        eps[nx // 3: nx // 3 + 8, 20:40] = rng.uniform(2, 10)
        grid = Grid(nx=nx, ny=ny, dx=0.05, device=dev())
        prof = GaussianPulse(0.65, 0.3)
        src = LineSource(grid, ix=12, j0=ny // 2 - 8, j1=ny // 2 + 8, profile=prof)
        if pol == "tm":
            m = build_tm_coeffs(grid, eps_inf=torch.tensor(eps, dtype=torch.float32), npml=8)
            mspec = [(True, nx - 20, 10, ny - 10), (False, ny - 15, 9, nx - 9)]
            mons = [FluxMonitorTM(grid, freqs, x_normal=a, idx=b, lo=c, hi=d)
                    for a, b, c, d in mspec] + [DFTFieldsMonitor(grid, freqs, "Ez")]
            items.append((init_tm_state(grid), m, src, mons))
            refs.append(_oracle_tm(nx, ny, 0.05, eps, 8, n, 12, ny // 2 - 8, ny // 2 + 8,
                                   freqs, mspec))
        else:
            m = build_te_coeffs(grid, eps_inf=torch.tensor(eps, dtype=torch.float32), npml=8)
            mx, my = (nx - 20, 10, ny - 10), (ny - 15, 9, nx - 9)
            mons = [DFTFieldsMonitor(grid, freqs, "Hz"),
                    FluxMonitorTE(grid, freqs, ix=mx[0], lo=mx[1], hi=mx[2]),
                    FluxMonitorTEY(grid, freqs, iy=my[0], lo=my[1], hi=my[2])]
            items.append((init_te_state(grid), m, TESource(src), mons))
            refs.append(_oracle_te(nx, ny, 0.05, eps, 8, n, 12, ny // 2 - 8, ny // 2 + 8,
                                   freqs, mon=(mx, my)))
    eng = Engine2D(items, rows_per_warp=16, ring_slots=7, variant=variant)
    eng.run(0, 50)
    eng.run(50, n - 50)                      # two calls: t0 continuity
    for b, ((pol, nx, ny), (s_ref, acc_ref)) in enumerate(zip(specs, refs)):
        st = eng.state(b)
        names = ("Ez", "Hx", "Hy", "Dz") if pol == "tm" else ("Hz", "Ex", "Ey", "Dx", "Dy")
        for k in names:
            e = rel_l2(getattr(st, k).cpu().numpy(), s_ref[k])
            assert e < TOL, (b, pol, k, e)
        accs = eng.accumulators(b)
        # the engine accumulators cover both calls only if folded by the caller:
        # each run() call adds into the same accumulators
        for a, r in zip(accs, acc_ref):
            e = rel_l2(a.cpu().numpy(), r)
            assert e < TOL, (b, pol, e)
    eng.close()


def test_explicit_initial_ez_matches_oracle():
    """An imported TM state whose Ez is not Dz/eps (e.g. a user-set initial
    field, tests/analytic/test_te.py style) is honoured on the first step."""
    from meep_torch_b200.core.coeffs import build_tm_coeffs
    from meep_torch_b200.core.grid import Grid
    from meep_torch_b200.core.run import run_tm
    from meep_torch_b200.core.stepper_tm import init_tm_state
    nx, ny = 90, 140
    grid = Grid(nx=nx, ny=ny, dx=0.02, device=dev())
    m = build_tm_coeffs(grid, npml=0)
    x = torch.arange(nx, dtype=torch.float32)[:, None]
    y = torch.arange(ny, dtype=torch.float32)[None, :]
    G = torch.exp(-((x - 45.0) ** 2 + (y - 70.0) ** 2) / (2 * 5.0 ** 2))
    s0 = init_tm_state(grid)._replace(Ez=G.to(dev()), Dz=(0.5 * G).to(dev()))
    st, _ = run_tm(s0, m, 60)
    c = O.tm_coeffs(nx, ny, 0.02, npml=0, dtype=np.float32)
    so = O.tm_state(c)
    so["Ez"], so["Dz"] = G.numpy(), (0.5 * G).numpy()
    for _ in range(60):
        so = O.tm_step(so, c)
    for k in ("Ez", "Hx", "Hy", "Dz"):
        assert rel_l2(getattr(st, k).cpu().numpy(), so[k]) < TOL, k


def test_energy_conserved_in_pec_box():
    """Discrete Yee invariant (tests/analytic/test_energy.py:29-62) through the
    CUDA path: float32 keeps it to ~1e-6 over 2000 steps."""
    from meep_torch_b200.core.coeffs import build_tm_coeffs
    from meep_torch_b200.core.grid import Grid
    from meep_torch_b200.core.run import run_tm
    from meep_torch_b200.core.stepper_tm import init_tm_state
    grid = Grid(nx=120, ny=120, dx=0.02, device=dev())
    m = build_tm_coeffs(grid, npml=0)
    x = torch.arange(120, dtype=torch.float32, device=dev())[:, None]
    G = torch.exp(-((x - 60.0) ** 2 + (x.T - 60.0) ** 2) / (2 * 6.0 ** 2))
    s = init_tm_state(grid)._replace(Ez=G, Dz=G.clone())
    us = []
    for _ in range(20):
        s_prev = s
        s, _ = run_tm(s, m, 1)
        e = 0.5 * (m.eps_inf * s_prev.Ez ** 2).sum()
        h = 0.5 * (s_prev.Hx * s.Hx).sum() + 0.5 * (s_prev.Hy * s.Hy).sum()
        us.append(float((e + h) * grid.dx ** 2))
        s, _ = run_tm(s, m, 99)
    u = np.array(us)
    assert (u.max() - u.min()) / u.mean() < 1e-4


@pytest.mark.parametrize("variant,slab", [(1, 0), (2, 0), (2, 3)])
def test_3d_wide_z_matches_oracle(variant, slab):
    """z extent 300 (three 128-column blocks, a partial last one) with the
    point source and a z flux face on a block boundary, CPML on all faces;
    the split kernels whole-grid and in x slabs of 3 planes."""
    from meep_torch_b200.core.monitors_3d import FluxMonitor3D, PointSource3D, run_3d
    from meep_torch_b200.core.sources import GaussianPulse
    from meep_torch_b200.core.stepper_3d import build_3d_coeffs, init_3d_state
    nx, ny, nz, dx, npml, n = 14, 13, 300, 0.05, 4, 60
    rng = np.random.default_rng(11)
    eps = (1.0 + 3.0 * rng.random((nx, ny, nz))).astype(np.float32)
    c = build_3d_coeffs(nx, ny, nz, dx, eps=torch.from_numpy(eps), npml=npml, device=dev())
    freqs = [0.8, 1.1]
    prof = GaussianPulse(1.0, 2.0)
    src = PointSource3D(c.dt, "Ez", 7, 6, 128, prof)
    mons = [FluxMonitor3D(c.dt, freqs, normal="z", idx=127, win=(2, 12, 2, 11)),
            FluxMonitor3D(c.dt, freqs, normal="x", idx=8, win=(2, 11, 100, 260))]
    oc = O.coeffs_3d(nx, ny, nz, dx, eps=eps, npml=npml, dtype=np.float32)
    s0 = O.state_3d(oc)
    for k in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz"):      # random start: waves in every layer
        s0[k] = rng.standard_normal(s0[k].shape).astype(np.float32)
    init = init_3d_state(nx, ny, nz, npml=npml, device=dev())
    init = init._replace(**{k: torch.from_numpy(s0[k]).to(dev())
                            for k in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")})
    st, accs = run_3d(init, c, n, source=src, monitors=mons, variant=variant, rows_per_seg=slab)
    dt = oc["dt"]
    om = [lambda s, t: O.flux3d_sample(s, t, dt, freqs, "z", 127, (2, 12, 2, 11)),
          lambda s, t: O.flux3d_sample(s, t, dt, freqs, "x", 8, (2, 11, 100, 260))]
    oprof = O.gaussian_pulse(1.0, 2.0)
    os_, oacc = O.run_3d(s0, oc, n, amp_fn=lambda t: oprof(O.src_time(t, dt)),
                         src=("Ez", 7, 6, 128), monitors=om)
    errs = {}
    sd = st._asdict()
    for k in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz", "psi_Hy_z", "psi_Ex_z", "psi_Hz_x",
              "psi_Ez_y", "psi_Hx_y", "psi_Ey_x"):
        errs[k] = rel_l2(sd[k].cpu().numpy(), os_[k])
    for q in range(2):
        errs[f"acc_{q}"] = rel_l2(accs[q].cpu().numpy(), oacc[q])
    bad = {k: v for k, v in errs.items() if not v < TOL}
    assert not bad, bad


@pytest.mark.parametrize("variant", [1, 2, 3])
def test_random_state_batched_matches_oracle(variant):
    """Random initial fields (waves in every CPML layer from the first step),
    a batch of TM, TM with PMC y walls and TE structures whose widths are not
    multiples of 128 and whose heights are not multiples of the tile rows;
    fields and CPML memory against the oracle. The temporally blocked kernels
    (variant 3) take PEC structures only, so their batch swaps the PMC one for a
    PEC one of the same shape; it runs 41 steps (a first single step, then ten
    4-step launches)."""
    from meep_torch_b200.core.coeffs import build_te_coeffs, build_tm_coeffs
    from meep_torch_b200.core.grid import Grid
    from meep_torch_b200.core.stepper_te import init_te_state
    from meep_torch_b200.core.stepper_tm import init_tm_state
    from meep_torch_b200.engine2d import Engine2D
    rng = np.random.default_rng(17)
    specs = [("tm", 37, 300, False), ("te", 50, 261, False), ("tm", 29, 131, variant != 3),
             ("te", 19, 45, False)]
    n, npml, dx = (41 if variant == 3 else 40), 8, 0.05
    items, refs = [], []
    for pol, nx, ny, pmc in specs:
        eps = (1.0 + 5.0 * rng.random((nx, ny))).astype(np.float32)
        grid = Grid(nx=nx, ny=ny, dx=dx, device=dev())
        if pol == "tm":
            c = O.tm_coeffs(nx, ny, dx, eps=eps, npml=npml, y_pmc=pmc, dtype=np.float32)
            so = O.tm_state(c)
            for k in ("Dz", "Hx", "Hy"):
                so[k] = rng.standard_normal(so[k].shape).astype(np.float32)
            m = build_tm_coeffs(grid, eps_inf=torch.from_numpy(eps), npml=npml, y_pmc=pmc)
            so["Ez"] = (torch.from_numpy(so["Dz"]) / m.eps_inf.cpu()).numpy()
            s0 = init_tm_state(grid, y_pmc=pmc)._replace(
                **{k: torch.from_numpy(so[k]).to(dev()) for k in ("Ez", "Dz", "Hx", "Hy")})
            step = O.tm_step
        else:
            c = O.te_coeffs(nx, ny, dx, eps=eps, npml=npml, dtype=np.float32)
            so = O.te_state(c)
            for k in ("Hz", "Dx", "Dy", "Ex", "Ey"):
                so[k] = rng.standard_normal(so[k].shape).astype(np.float32)
            m = build_te_coeffs(grid, eps_inf=torch.from_numpy(eps), npml=npml)
            s0 = init_te_state(grid)._replace(
                **{k: torch.from_numpy(so[k]).to(dev()) for k in ("Hz", "Dx", "Dy", "Ex", "Ey")})
            step = O.te_step
        items.append((s0, m, None, []))
        refs.append(O.run_2d(step, so, c, n)[0])
    eng = Engine2D(items, variant=variant)
    eng.run(0, n)
    errs = {}
    for b, ((pol, nx, ny, pmc), ref) in enumerate(zip(specs, refs)):
        st = eng.state(b)
        names = (("Ez", "Hx", "Hy", "Dz", "psi_Ezy", "psi_Ezx", "psi_Hyx", "psi_Hxy")
                 if pol == "tm" else
                 ("Hz", "Ex", "Ey", "Dx", "Dy", "psi_Eyx", "psi_Exy", "psi_Hzy", "psi_Hzx"))
        for k in names:
            errs[(b, k)] = rel_l2(getattr(st, k).cpu().numpy(), ref[k])
    eng.close()
    bad = {k: v for k, v in errs.items() if not v < TOL}
    assert not bad, bad


@pytest.mark.parametrize("variant", [1, 2, 3])
def test_graph_replay_bitwise_equal_to_direct_launches(variant):
    """Whole ring flushes replayed as a CUDA graph (coefficient and phase rows
    staged per flush) give bit-identical fields and accumulators to the same
    steps launched one by one, across two run() calls."""
    from meep_torch_b200 import workloads as W
    from meep_torch_b200.engine2d import Engine2D
    specs = W.cfg2_specs(n=4, seed=9, lo=96, hi=200)
    outs = []
    for graph in (False, True):
        items = [W.cfg2_item(s, dev()) for s in specs]
        eng = Engine2D(items, ring_slots=8, variant=variant, graph=graph)
        eng.run(0, 45)
        eng.run(45, 40)
        outs.append(([eng.state(b) for b in range(len(specs))],
                     [[a.clone() for a in eng.accumulators(b)] for b in range(len(specs))]))
        eng.close()
    (s0, a0), (s1, a1) = outs
    for b in range(len(specs)):
        for name in s0[b]._fields:
            x, y = getattr(s0[b], name), getattr(s1[b], name)
            if isinstance(x, torch.Tensor) and x.numel():
                assert torch.equal(x, y), (b, name)
        for x, y in zip(a0[b], a1[b]):
            assert torch.equal(x, y), b


def test_tb_matches_tiles_on_a_cfg2_batch():
    """The temporally blocked kernels (4 steps per launch from TMA-staged tiles)
    against the one-step tile kernels on a cfg2-shaped batch of TM and TE bends
    (line sources, full-grid DFT, two flux lines), over ring flushes of 32 steps
    and a partial last launch: fields, CPML memory and accumulators agree to
    float32 rounding, and the TB plan issues about a quarter of the launches."""
    from meep_torch_b200 import workloads as W
    from meep_torch_b200.engine2d import Engine2D
    specs = W.cfg2_specs(n=6, seed=11, lo=120, hi=420)
    outs, launches = [], []
    for variant in (2, 3):
        items = [W.cfg2_item(s, dev()) for s in specs]
        eng = Engine2D(items, variant=variant, graph=False)
        eng.run(0, 1)
        eng.run(1, 130)
        launches.append(int(eng.last_launches))
        outs.append(([eng.state(b) for b in range(len(specs))],
                     [[a.clone() for a in eng.accumulators(b)] for b in range(len(specs))]))
        eng.close()
    (s0, a0), (s1, a1) = outs
    errs = {}
    for b in range(len(specs)):
        for name in s0[b]._fields:
            x, y = getattr(s0[b], name), getattr(s1[b], name)
            if isinstance(x, torch.Tensor) and x.numel():
                errs[(b, name)] = rel_l2(y.cpu().numpy(), x.cpu().numpy())
        for q, (x, y) in enumerate(zip(a0[b], a1[b])):
            errs[(b, f"acc{q}")] = rel_l2(y.cpu().numpy(), x.cpu().numpy())
    print(f"\n[tb vs tiles] max relL2 {max(errs.values()):.2e}; launches {launches}")
    bad = {k: v for k, v in errs.items() if not v < 1e-5}
    assert not bad, bad
    assert launches[1] < launches[0] / 2, launches


@pytest.mark.parametrize("shape", [(320, 160), (77, 50), (30, 301), (200, 96)])
@pytest.mark.parametrize("graph", [False, True])
def test_cluster_kernel_matches_tiles(shape, graph):
    """The cluster-resident TM kernel (variant 4: the structure's rows split over the
    shared memory of one thread-block cluster, a ring's worth of steps per launch,
    neighbour rows through distributed shared memory) against the one-step tiles from
    a random start: the cfg1 320 x 160 case and shapes whose rows do not split evenly
    over the cluster, a single-cell source, a flux line, a full-grid DFT, run lengths of
    both parities over several calls and ring flushes (graph-replayed or not)."""
    from meep_torch_b200.core.coeffs import build_tm_coeffs
    from meep_torch_b200.core.grid import Grid
    from meep_torch_b200.core.monitors import DFTFieldsMonitor, FluxMonitorTM
    from meep_torch_b200.core.sources import GaussianPulse, LineSource
    from meep_torch_b200.core.stepper_tm import init_tm_state
    from meep_torch_b200.engine2d import Engine2D
    nx, ny = shape
    rng = np.random.default_rng(nx * 7 + ny)
    eps = torch.from_numpy((1.0 + 5.0 * rng.random((nx, ny))).astype(np.float32)).to(dev())
    grid = Grid(nx=nx, ny=ny, dx=0.05, device=dev())
    outs, launches = [], []
    for variant in (2, 4):
        m = build_tm_coeffs(grid, eps_inf=eps, npml=10)
        src = LineSource(grid, ix=nx // 4, j0=ny // 2, j1=ny // 2 + 1,
                         profile=GaussianPulse(0.6, 0.3))
        mons = [FluxMonitorTM(grid, [0.5, 0.6, 0.7], x_normal=True, idx=3 * nx // 4, lo=12,
                              hi=ny - 12),
                DFTFieldsMonitor(grid, [0.55, 0.65], "Ez")]
        s0 = init_tm_state(grid)
        g = torch.Generator().manual_seed(3)
        s0 = s0._replace(**{k: 0.1 * torch.randn(getattr(s0, k).shape, generator=g).to(dev())
                            for k in ("Hx", "Hy")})
        eng = Engine2D([(s0, m, src, mons)], variant=variant, ring_slots=16, graph=graph)
        eng.run(0, 1)
        eng.run(1, 47)
        eng.run(48, 33)
        launches.append(int(eng.last_launches))
        outs.append((eng.state(0), [a.clone() for a in eng.accumulators(0)]))
        eng.close()
    (s0, a0), (s1, a1) = outs
    errs = {}
    for name in s0._fields:
        x, y = getattr(s0, name), getattr(s1, name)
        if isinstance(x, torch.Tensor) and x.numel():
            errs[name] = rel_l2(y.cpu().numpy(), x.cpu().numpy())
    for q, (x, y) in enumerate(zip(a0, a1)):
        errs[f"acc{q}"] = rel_l2(y.cpu().numpy(), x.cpu().numpy())
    print(f"\n[cluster vs tiles {shape}] max relL2 {max(errs.values()):.2e}; launches {launches}")
    bad = {k: v for k, v in errs.items() if not v < 1e-6}
    assert not bad, bad
    assert launches[1] < launches[0] / 4, launches


@pytest.mark.parametrize("variant", [2, 3])
def test_point_probes_stack_every_step(variant):
    """PointProbe (reduce "stack", core/monitors.py:11-21) next to a flux line: the run
    returns Ez at the probe node after every step, over several ring flushes and two
    run calls, equal to the oracle's per-step values; the flux accumulator still sums."""
    from meep_torch_b200.core.coeffs import build_tm_coeffs
    from meep_torch_b200.core.grid import Grid
    from meep_torch_b200.core.monitors import FluxMonitorTM, PointProbe
    from meep_torch_b200.core.run import _run_chunk
    from meep_torch_b200.core.sources import GaussianPulse, LineSource
    from meep_torch_b200.core.stepper_tm import init_tm_state
    nx, ny, dx, npml = 60, 140, 0.05, 8
    rng = np.random.default_rng(31)
    eps = np.ones((nx, ny), dtype=np.float32)
    eps[:, 60:80] = 12.0
    eps[30:40, 20:50] = rng.uniform(2, 8, (10, 30))
    grid = Grid(nx=nx, ny=ny, dx=dx, device=dev())
    m = build_tm_coeffs(grid, eps_inf=torch.from_numpy(eps), npml=npml)
    src = LineSource(grid, ix=12, j0=60, j1=80, profile=GaussianPulse(0.65, 0.3))
    probes = [PointProbe(20, 70), PointProbe(45, 130)]
    freqs = [0.6, 0.7]
    flux = FluxMonitorTM(grid, freqs, x_normal=True, idx=40, lo=10, hi=130)
    c = O.tm_coeffs(nx, ny, dx, eps=eps, npml=npml, dtype=np.float32)
    mask = O.line_source_mask(nx, ny, dx, 12, 60, 80, dtype=np.float32)
    op = O.gaussian_pulse(0.65, 0.3)
    rec = []
    so, (ao,) = O.run_2d(
        O.tm_step, O.tm_state(c), c, 90, amp_fn=lambda t: op(O.src_time(t, c["dt"])),
        mask=mask, monitors=[lambda s, t: (rec.append([s["Ez"][20, 70], s["Ez"][45, 130]]),
                                           O.flux_tm_sample(s, t, c["dt"], freqs, True, 40, 10,
                                                            130, np.float32))[1]])
    rec = np.array(rec, dtype=np.float64)
    from meep_torch_b200.engine2d import Engine2D
    eng = Engine2D([(init_tm_state(grid), m, src, [probes[0], flux, probes[1]])],
                   variant=variant, ring_slots=16)
    eng.run(0, 50)
    p0a, _, p1a = eng.accumulators(0)
    eng.run(50, 40)
    p0b, acc, p1b = eng.accumulators(0)
    eng.close()
    got = np.stack([torch.cat([p0a, p0b]).cpu().double().numpy(),
                    torch.cat([p1a, p1b]).cpu().double().numpy()], axis=1)
    assert got.shape == (90, 2)
    assert rel_l2(got, rec) < TOL, rel_l2(got, rec)
    assert rel_l2(acc.cpu().numpy(), ao) < TOL
    # through the reference's seam: _run_chunk returns the stack as the probe's output
    st, outs = _run_chunk(None, init_tm_state(grid), m, 0, 20, src, [probes[0]])
    assert outs[0].shape == (20,)
    assert rel_l2(outs[0].cpu().numpy(), rec[:20, 0]) < TOL


def _grad_setup(g, dev_, requires_grad=True, extra=None):
    from meep_torch_b200.core.coeffs import build_tm_coeffs
    from meep_torch_b200.core.grid import Grid
    from meep_torch_b200.core.monitors import DFTFieldsMonitor, FluxMonitorTM
    from meep_torch_b200.core.sources import GaussianPulse, LineSource
    from meep_torch_b200.core.stepper_tm import init_tm_state
    nx, ny, dx, npml = int(g["nx"]), int(g["ny"]), float(g["dx"]), int(g["npml"])
    grid = Grid(nx=nx, ny=ny, dx=dx, device=dev_)
    e = torch.tensor(g["eps"], dtype=torch.float32, device=dev_, requires_grad=requires_grad)
    kw, n_p = {}, 0
    if extra == "lossy":
        kw = {k: torch.tensor(g[f], dtype=torch.float32, device=dev_)
              for k, f in (("sigma_d", "sigma"), ("sigma_b", "sigma_b"), ("mu", "mu"))}
    elif extra == "poles":
        poles = json.loads(str(g["poles"]))
        kw = dict(poles=poles, pole_masks=[torch.tensor(v, dtype=torch.float32, device=dev_)
                                           for v in g["pole_masks"]])
        n_p = len(poles)
    elif extra == "mpoles":
        kw = dict(m_poles=[tuple(p) for p in json.loads(str(g["m_poles"]))],
                  m_pole_masks=[torch.tensor(v, dtype=torch.float32, device=dev_)
                                for v in g["m_pole_masks"]])
    n_m = len(kw.get("m_poles", ()))
    pmc = extra == "pmc"
    if pmc:
        kw = dict(y_pmc=True)
    folds = json.loads(str(g["fold"])) if "fold" in g else {}
    kw.update(folds)
    m = build_tm_coeffs(grid, eps_inf=e, npml=npml, **kw)
    src = LineSource(grid, ix=int(g["src_ix"]), j0=int(g["src_j0"]), j1=int(g["src_j1"]),
                     profile=GaussianPulse(float(g["fcen"]), float(g["fwidth"])))
    freqs = [float(f) for f in g["freqs"]]
    mx, my = (int(v) for v in g["monx"]), (int(v) for v in g["mony"])
    mx, my = list(mx), list(my)
    monx = FluxMonitorTM(grid, freqs, x_normal=True, idx=mx[0], lo=mx[1], hi=mx[2])
    mony = FluxMonitorTM(grid, freqs, x_normal=False, idx=my[0], lo=my[1], hi=my[2])
    dft = DFTFieldsMonitor(grid, freqs, "Ez")
    return e, m, src, [monx, mony, dft], init_tm_state(grid, n_poles=n_p, n_mpoles=n_m, y_pmc=pmc,
                                                       **folds), dx


def _grad_loss(st, ax, ay, ad, mx, my, dx):
    """The fixtures' loss (tests/golden/make_golden.py grad_loss)."""
    w = torch.tensor([1.0, -0.5, 0.25], dtype=ax.dtype, device=ax.device)
    J = ((w * mx.flux(ax, dx)).sum() + (w.flip(0) * my.flux(ay, dx)).sum()
         + 1e-3 * (ad * ad).sum() + 0.1 * (st.Ez * st.Ez).sum()
         + 0.05 * (st.Hy * st.Hy).sum() - 0.02 * (st.Hx * st.Hx).sum())
    for k, c in (("Hx0", 0.3), ("Hy0", -0.2)):     # the live on-plane lines of odd cuts
        if getattr(st, k, None) is not None:
            J = J + c * (getattr(st, k) ** 2).sum()
    return J


@pytest.mark.parametrize("chunk", [50, 32, 7])
def test_tm_gradient_matches_reference_autograd(chunk):
    """d J / d eps from the library's discrete-adjoint kernels against the
    reference's own autograd through run_tm(checkpoint_every=50) (fixtures
    made by tests/golden/make_golden.py grad), for several checkpoint lengths."""
    from meep_torch_b200.core.run import run_tm
    g32, g64 = load_golden("grad_tm_f32"), load_golden("grad_tm_f64")
    e, m, src, mons, s0, dx = _grad_setup(g32, dev())
    st, (ax, ay, ad) = run_tm(s0, m, int(g32["n_steps"]), source=src, monitors=mons,
                              checkpoint_every=chunk)
    J = _grad_loss(st, ax, ay, ad, mons[0], mons[1], dx)
    J.backward()
    got = e.grad.cpu().numpy()
    e32, e64 = rel_l2(got, g32["grad"]), rel_l2(got, g64["grad"])
    print(f"grad chunk {chunk}: rel L2 vs reference f32 {e32:.3e}, vs f64 {e64:.3e}; "
          f"J {float(J):.6e} vs {float(g32['J']):.6e}")
    assert abs(float(J) - float(g32["J"])) <= 1e-4 * abs(float(g32["J"]))
    assert e32 < 1e-4, e32


@pytest.mark.parametrize("extra", ["lossy", "poles", "pmc", "mirror", "mirror_odd", "rot2",
                                   "rot4", "mpoles"])
@pytest.mark.parametrize("chunk", [50, 13])
def test_tm_gradient_lossy_and_dispersive_match_reference_autograd(extra, chunk):
    """d J / d eps of lossy (sigma_d on E, sigma_b and mu on H), dispersive (a
    Lorentz and a Drude pole), y-PMC, even- and odd-mirror (cuts on the low x and y edges)
    and odd Rotate2 / Rotate4 TM runs (the live on-plane H lines, their final values in
    the loss) and TM runs with two magnetic Lorentz poles (H = B - sum M) from the adjoint
    kernels, against the reference's
    float64 autograd through run_tm(checkpoint_every=50) (tests/golden/make_golden.py
    grad_extra); the float32 forward and adjoint agree with it to 1e-4."""
    from meep_torch_b200.core.run import run_tm
    g64 = load_golden(f"grad_tm_{extra}_f64")
    e, m, src, mons, s0, dx = _grad_setup(g64, dev(), extra=extra)
    st, (ax, ay, ad) = run_tm(s0, m, int(g64["n_steps"]), source=src, monitors=mons,
                              checkpoint_every=chunk)
    J = _grad_loss(st, ax, ay, ad, mons[0], mons[1], dx)
    J.backward()
    got = e.grad.cpu().numpy()
    e64 = rel_l2(got, g64["grad"])
    print(f"grad {extra} chunk {chunk}: rel L2 vs reference f64 {e64:.3e}; "
          f"J {float(J):.6e} vs {float(g64['J']):.6e}")
    assert abs(float(J) - float(g64["J"])) <= 1e-4 * abs(float(g64["J"]))
    assert e64 < 1e-4, e64


class _Sheets:
    """A TFSF-style source with the shape of the reference's mode sources
    (ports/mode_source.py:21-128): an electric current sheet (``mask``) and a
    magnetic sheet (``h_masks``) half a cell upstream, the magnetic amplitude
    delayed and signed. The kernels see only this protocol."""

    def __init__(self, prof, dt, mask, h_masks, te=False, delay=0.0, hsign=-1.0):
        self.prof, self.dt, self.mask, self.h_masks = prof, dt, mask, h_masks
        self.te, self.delay, self.hsign = te, delay, hsign

    def amplitude(self, t):
        return self.prof.amplitude((t if self.te else t + 0.5) * self.dt)

    def h_amplitude(self, t):
        return self.hsign * self.prof.amplitude((t + 0.5 if self.te else t) * self.dt
                                                - self.delay)


@pytest.mark.parametrize("case", ["tm_x", "tm_y", "te_x"])
def test_magnetic_sheet_sources_match_oracle(case):
    """Electric + magnetic sheet pairs (the mode-source path: src_hy_mask,
    src_hx_mask, src_hz_mask) through run_tm / run_te against the oracle."""
    from meep_torch_b200.core.coeffs import build_te_coeffs, build_tm_coeffs
    from meep_torch_b200.core.grid import Grid
    from meep_torch_b200.core.run import run_te, run_tm
    from meep_torch_b200.core.sources import GaussianPulse
    from meep_torch_b200.core.stepper_te import init_te_state
    from meep_torch_b200.core.stepper_tm import init_tm_state
    nx, ny, dx, npml, n = 70, 58, 0.05, 8, 150
    eps = np.ones((nx, ny), dtype=np.float32)
    eps[:, 24:34] = 12.0
    eps[24:34, :] = np.maximum(eps[24:34, :], 6.0)
    prof = GaussianPulse(0.65, 0.3)
    oprof = O.gaussian_pulse(0.65, 0.3)
    shape = np.sin(np.linspace(0.2, np.pi - 0.2, 14)).astype(np.float32)
    grid = Grid(nx=nx, ny=ny, dx=dx, device=dev())
    delay = 2.5 * dx / 2.0
    if case.startswith("tm"):
        c = O.tm_coeffs(nx, ny, dx, eps=eps, npml=npml, dtype=np.float32)
        m = build_tm_coeffs(grid, eps_inf=torch.from_numpy(eps), npml=npml)
        mask = np.zeros((nx, ny), np.float32)
        if case == "tm_x":
            mask[14, 22:36] = 2.5 * shape / dx
            hm = np.zeros((nx - 1, ny), np.float32)
            hm[13, 22:36] = shape / dx
            key = "src_hy_mask"
        else:
            mask[22:36, 14] = -2.5 * shape / dx
            hm = np.zeros((nx, ny - 1), np.float32)
            hm[22:36, 13] = shape / dx
            key = "src_hx_mask"
        src = _Sheets(prof, c["dt"], torch.from_numpy(mask).to(dev()),
                      {key: torch.from_numpy(hm).to(dev())}, delay=delay)
        st, _ = run_tm(init_tm_state(grid), m, n, source=src)
        s = O.tm_state(c)
        for t in range(n):
            kw = {"hy_mask" if case == "tm_x" else "hx_mask": hm}
            s = O.tm_step(s, c, amp=oprof((t + 0.5) * c["dt"]), mask=mask,
                          amp_h=-oprof(t * c["dt"] - delay), **kw)
        names = ("Ez", "Hx", "Hy", "Dz")
    else:
        c = O.te_coeffs(nx, ny, dx, eps=eps, npml=npml, dtype=np.float32)
        m = build_te_coeffs(grid, eps_inf=torch.from_numpy(eps), npml=npml)
        mask = np.zeros((nx, ny - 1), np.float32)
        mask[14, 22:36] = shape / dx
        hm = np.zeros((nx - 1, ny - 1), np.float32)
        hm[13, 22:36] = 2.0 * shape / dx
        src = _Sheets(prof, c["dt"], torch.from_numpy(mask).to(dev()),
                      {"src_hz_mask": torch.from_numpy(hm).to(dev())}, te=True, delay=delay,
                      hsign=1.0)
        st, _ = run_te(init_te_state(grid), m, n, source=src)
        s = O.te_state(c)
        for t in range(n):
            s = O.te_step(s, c, amp=oprof(t * c["dt"]), mask_ey=mask,
                          amp_h=oprof((t + 0.5) * c["dt"] - delay), hz_mask=hm)
        names = ("Hz", "Ex", "Ey", "Dx", "Dy")
    errs = {k: rel_l2(getattr(st, k).cpu().numpy(), s[k]) for k in names}
    assert all(v < TOL for v in errs.values()), errs


@pytest.mark.parametrize("case", ["sigma", "poles", "pmc"])
def test_3d_lossy_gradient_matches_reference_run_3d_adjoint(case):
    """d J / d eps of run_3d_adjoint with conductive damping (a sigma_d slab, a sigma_b
    patch: H' = d1 H - d2 curl, E' = d1 E + d2 curl / eps), with a Lorentz and a Drude
    pole (P(n+1) = c1 P(n) + c2 P(n-1) + c3 E(n), folded-D E update) or with PMC walls on
    y (the dipole next to one) on the 3D adjoint kernels against the reference's float64
    run_3d_adjoint (tests/golden/make_golden.py grad3d_sigma / grad3d_poles / grad3d_pmc,
    pinned by central differences of the oracle)."""
    from meep_torch_b200.core.adjoint3d import run_3d_adjoint
    from meep_torch_b200.core.monitors_3d import FluxMonitor3D, PointSource3D
    from meep_torch_b200.core.sources import GaussianPulse
    from meep_torch_b200.core.stepper_3d import build_3d_coeffs, init_3d_state
    g64 = load_golden(f"grad3d_{case}_f64")
    n, dx, npml = int(g64["n"]), float(g64["dx"]), int(g64["npml"])
    e = torch.tensor(g64["eps"], dtype=torch.float32, device=dev(), requires_grad=True)
    if case == "sigma":
        kw = dict(sigma_d=torch.tensor(g64["sigma_d"], dtype=torch.float32),
                  sigma_b=torch.tensor(g64["sigma_b"], dtype=torch.float32))
        n_p = 0
    elif case == "pmc":
        kw = dict(pmc_axes=tuple(int(a) for a in g64["pmc_axes"]))
        n_p = 0
    else:
        poles = [tuple(p) for p in json.loads(str(g64["poles"]))]
        kw = dict(poles=poles, pole_masks=[torch.tensor(g64[f"pm{q}"], dtype=torch.float32)
                                           for q in range(2)])
        n_p = len(poles)
    c = build_3d_coeffs(n, n, n, dx, eps=e, npml=npml, device=dev(), **kw)
    i, j, k = (int(v) for v in g64["src"])
    src = PointSource3D(c.dt, "Ez", i, j, k, GaussianPulse(float(g64["fcen"]), float(g64["fwidth"])))
    freqs = [float(f) for f in g64["freqs"]]
    mons = [FluxMonitor3D(c.dt, freqs, normal="x", idx=15, win=(5, 15, 5, 15)),
            FluxMonitor3D(c.dt, freqs, normal="z", idx=6, win=(5, 15, 5, 15))]
    w = torch.tensor([1.0, -0.7, 0.4], dtype=torch.float32, device=dev())

    def loss_fn(accs):
        return 1e15 * ((w * mons[0].flux(accs[0], dx)).sum()
                       + (w.flip(0) * mons[1].flux(accs[1], dx)).sum()
                       + 1e-3 * sum((a * a).sum() for a in accs))

    L, accs = run_3d_adjoint(c, int(g64["n_steps"]), 16, src, mons, loss_fn,
                             init_3d_state(n, n, n, npml=npml, device=dev(), n_poles=n_p))
    got = e.grad.cpu().numpy()
    e64 = rel_l2(got, g64["grad"])
    print(f"3D {case} grad: rel L2 vs reference f64 {e64:.3e}; L {L:.6e} vs "
          f"{float(g64['L']):.6e}")
    assert abs(L - float(g64["L"])) <= 1e-4 * abs(float(g64["L"]))
    assert e64 < 1e-4, e64


def test_3d_gradient_matches_reference_run_3d_adjoint():
    """d J / d eps of run_3d_adjoint on the library's 3D adjoint kernels against the
    reference's own run_3d_adjoint (core/adjoint3d.py:56-115; fixtures made by
    tests/golden/make_golden.py grad3d), chunked differently on each side."""
    from meep_torch_b200.core.adjoint3d import run_3d_adjoint
    from meep_torch_b200.core.monitors_3d import FluxMonitor3D, PointSource3D
    from meep_torch_b200.core.sources import GaussianPulse
    from meep_torch_b200.core.stepper_3d import build_3d_coeffs, init_3d_state
    g32, g64 = load_golden("grad3d_f32"), load_golden("grad3d_f64")
    n, dx, npml = int(g32["n"]), float(g32["dx"]), int(g32["npml"])
    e = torch.tensor(g32["eps"], dtype=torch.float32, device=dev(), requires_grad=True)
    c = build_3d_coeffs(n, n, n, dx, eps=e, npml=npml, device=dev())
    i, j, k = (int(v) for v in g32["src"])
    src = PointSource3D(c.dt, "Ez", i, j, k, GaussianPulse(float(g32["fcen"]), float(g32["fwidth"])))
    freqs = [float(f) for f in g32["freqs"]]
    mons = [FluxMonitor3D(c.dt, freqs, normal="x", idx=15, win=(5, 15, 5, 15)),
            FluxMonitor3D(c.dt, freqs, normal="z", idx=6, win=(5, 15, 5, 15))]
    w = torch.tensor([1.0, -0.7, 0.4], dtype=torch.float32, device=dev())

    def loss_fn(accs):
        return 1e15 * ((w * mons[0].flux(accs[0], dx)).sum()
                       + (w.flip(0) * mons[1].flux(accs[1], dx)).sum()
                       + 1e-3 * sum((a * a).sum() for a in accs))

    L, accs = run_3d_adjoint(c, int(g32["n_steps"]), 16, src, mons, loss_fn,
                             init_3d_state(n, n, n, npml=npml, device=dev()))
    got = e.grad.cpu().numpy()
    e32, e64 = rel_l2(got, g32["grad"]), rel_l2(got, g64["grad"])
    print(f"3D grad: rel L2 vs reference f32 {e32:.3e}, vs f64 {e64:.3e}; "
          f"L {L:.6e} vs {float(g32['L']):.6e}")
    assert abs(L - float(g32["L"])) <= 1e-4 * abs(float(g32["L"]))
    assert rel_l2(accs[0].cpu().numpy(), g32["acc_0"]) < TOL
    assert e32 < TOL, e32


@pytest.mark.parametrize("chunk", [60, 32])
def test_te_gradient_matches_reference_autograd(chunk):
    """d J / d eps_inf of a TE run (gradients through eps_x / eps_y to eps_inf) from
    the adjoint kernels against the reference's autograd through run_te
    (fixtures: tests/golden/make_golden.py grad_te)."""
    from meep_torch_b200.core.coeffs import build_te_coeffs
    from meep_torch_b200.core.grid import Grid
    from meep_torch_b200.core.monitors import DFTFieldsMonitor, FluxMonitorTE, FluxMonitorTEY
    from meep_torch_b200.core.run import run_te
    from meep_torch_b200.core.sources import GaussianPulse, LineSource, TESource
    from meep_torch_b200.core.stepper_te import init_te_state
    g32, g64 = load_golden("grad_te_f32"), load_golden("grad_te_f64")
    nx, ny, dx, npml = int(g32["nx"]), int(g32["ny"]), float(g32["dx"]), int(g32["npml"])
    grid = Grid(nx=nx, ny=ny, dx=dx, device=dev())
    e = torch.tensor(g32["eps"], dtype=torch.float32, device=dev(), requires_grad=True)
    m = build_te_coeffs(grid, eps_inf=e, npml=npml)
    src = TESource(LineSource(grid, ix=int(g32["src_ix"]), j0=int(g32["src_j0"]),
                              j1=int(g32["src_j1"]),
                              profile=GaussianPulse(float(g32["fcen"]), float(g32["fwidth"]))))
    freqs = [float(f) for f in g32["freqs"]]
    mx, my = [int(v) for v in g32["monx"]], [int(v) for v in g32["mony"]]
    dft = DFTFieldsMonitor(grid, freqs, "Hz")
    monx = FluxMonitorTE(grid, freqs, ix=mx[0], lo=mx[1], hi=mx[2])
    mony = FluxMonitorTEY(grid, freqs, iy=my[0], lo=my[1], hi=my[2])
    st, (ad, ax, ay) = run_te(init_te_state(grid), m, int(g32["n_steps"]), source=src,
                              monitors=[dft, monx, mony], checkpoint_every=chunk)
    w = torch.tensor([1.0, -0.5, 0.25], dtype=torch.float32, device=dev())
    J = 1e6 * ((w * monx.flux(ax, dx)).sum() + (w.flip(0) * mony.flux(ay, dx)).sum()
               + 1e-3 * (ad * ad).sum() + 0.1 * (st.Hz * st.Hz).sum()
               + 0.05 * (st.Ex * st.Ex).sum() - 0.02 * (st.Ey * st.Ey).sum())
    J.backward()
    got = e.grad.cpu().numpy()
    e32, e64 = rel_l2(got, g32["grad"]), rel_l2(got, g64["grad"])
    print(f"TE grad chunk {chunk}: rel L2 vs reference f32 {e32:.3e}, vs f64 {e64:.3e}; "
          f"J {float(J):.6e} vs {float(g32['J']):.6e}")
    assert abs(float(J) - float(g32["J"])) <= 1e-4 * abs(float(g32["J"]))
    assert e32 < TOL, e32


@pytest.mark.parametrize("chunk", [60, 32])
@pytest.mark.parametrize("extra", ["lossy", "poles", "mirror", "mirror_even"])
def test_te_gradient_lossy_and_dispersive_match_reference_autograd(extra, chunk):
    """d J / d eps_inf of lossy (sigma_d on Dx / Dy, sigma_b and mu on Hz), dispersive
    (a Lorentz and a Drude pole on Ex and Ey), odd-mirror (cuts on the low x and y edges:
    CPML profiles only) and even-mirror (the cut rows' 2 Hz / dx) TE runs from the
    adjoint kernels,
    against the reference's float64 autograd through run_te(checkpoint_every=60)
    (tests/golden/make_golden.py grad_extra_te, pinned by central differences of the
    oracle); the float32 forward and adjoint agree with it to 1e-4."""
    from meep_torch_b200.core.coeffs import build_te_coeffs
    from meep_torch_b200.core.grid import Grid
    from meep_torch_b200.core.monitors import DFTFieldsMonitor, FluxMonitorTE, FluxMonitorTEY
    from meep_torch_b200.core.run import run_te
    from meep_torch_b200.core.sources import GaussianPulse, LineSource, TESource
    from meep_torch_b200.core.stepper_te import init_te_state
    g64 = load_golden(f"grad_te_{extra}_f64")
    nx, ny, dx, npml = int(g64["nx"]), int(g64["ny"]), float(g64["dx"]), int(g64["npml"])
    grid = Grid(nx=nx, ny=ny, dx=dx, device=dev())
    e = torch.tensor(g64["eps"], dtype=torch.float32, device=dev(), requires_grad=True)
    T = lambda a: torch.tensor(a, dtype=torch.float32)  # noqa: E731
    kw, n_p = {}, 0
    if extra == "lossy":
        kw = dict(sigma_d=T(g64["sigma"]), sigma_b=T(g64["sigma_b"]), mu=T(g64["mu"]))
    elif extra.startswith("mirror"):
        kw = json.loads(str(g64["fold"]))
    else:
        poles = json.loads(str(g64["poles"]))
        kw = dict(poles=poles, pole_masks=[T(x) for x in g64["pole_masks"]])
        n_p = len(poles)
    m = build_te_coeffs(grid, eps_inf=e, npml=npml, **kw)
    src = TESource(LineSource(grid, ix=int(g64["src_ix"]), j0=int(g64["src_j0"]),
                              j1=int(g64["src_j1"]),
                              profile=GaussianPulse(float(g64["fcen"]), float(g64["fwidth"]))))
    freqs = [float(f) for f in g64["freqs"]]
    mx, my = [int(v) for v in g64["monx"]], [int(v) for v in g64["mony"]]
    dft = DFTFieldsMonitor(grid, freqs, "Hz")
    monx = FluxMonitorTE(grid, freqs, ix=mx[0], lo=mx[1], hi=mx[2])
    mony = FluxMonitorTEY(grid, freqs, iy=my[0], lo=my[1], hi=my[2])
    st, (ad, ax, ay) = run_te(init_te_state(grid, n_poles=n_p), m, int(g64["n_steps"]),
                              source=src, monitors=[dft, monx, mony], checkpoint_every=chunk)
    w = torch.tensor([1.0, -0.5, 0.25], dtype=torch.float32, device=dev())
    J = 1e6 * ((w * monx.flux(ax, dx)).sum() + (w.flip(0) * mony.flux(ay, dx)).sum()
               + 1e-3 * (ad * ad).sum() + 0.1 * (st.Hz * st.Hz).sum()
               + 0.05 * (st.Ex * st.Ex).sum() - 0.02 * (st.Ey * st.Ey).sum())
    J.backward()
    got = e.grad.cpu().numpy()
    e64 = rel_l2(got, g64["grad"])
    print(f"TE grad {extra} chunk {chunk}: rel L2 vs reference f64 {e64:.3e}; "
          f"J {float(J):.6e} vs {float(g64['J']):.6e}")
    assert abs(float(J) - float(g64["J"])) <= 1e-4 * abs(float(g64["J"]))
    assert e64 < 1e-4, e64


@pytest.mark.parametrize("geometry", [0, 2])
@pytest.mark.parametrize("shape", [(23, 17, 40), (9, 30, 128), (31, 13, 131), (6, 22, 256),
                                   (40, 8, 77), (48, 256, 256)])
def test_3d_one_pass_bitwise_equal_to_split(shape, geometry):
    """The one-pass x-march (variant 3: H and E of a plane in one kernel, TMA-staged
    planes, a persistent grid cutting the (tile, plane) sequence into segments with
    recomputed halo planes) gives the split kernels' results bit for bit: fields, CPML
    memory and flux / DFT accumulators from a random start, for z widths on both
    kernel shapes (zpitch <= 128 and <= 256), y extents that leave a partial tile and
    grids small enough that every block owns a few planes only; with the default work
    geometry and with the lockstep one asked for (tiles of cost-balanced heights, every
    tile cut at the same x planes)."""
    from meep_torch_b200.core.monitors_3d import (DFTFieldsMonitor3D, FluxMonitor3D,
                                                  PointSource3D, run_3d)
    from meep_torch_b200.core.sources import GaussianPulse
    from meep_torch_b200.core.stepper_3d import build_3d_coeffs, init_3d_state
    nx, ny, nz = shape
    dx, npml, n = 0.05, 3, 24
    rng = np.random.default_rng(nx * 1000 + ny)
    eps = (1.0 + 3.0 * rng.random((nx, ny, nz))).astype(np.float32)
    c = build_3d_coeffs(nx, ny, nz, dx, eps=torch.from_numpy(eps), npml=npml, device=dev())
    freqs = [0.8, 1.1]
    prof = GaussianPulse(1.0, 2.0)
    src = PointSource3D(c.dt, "Ez", nx // 2, ny // 2, nz // 2, prof)
    mons = [FluxMonitor3D(c.dt, freqs, normal="x", idx=nx // 3, ap=1),
            FluxMonitor3D(c.dt, freqs, normal="z", idx=nz - 5, ap=1),
            DFTFieldsMonitor3D(c.dt, freqs, component="Hy", plane=(1, ny // 2))]
    init = init_3d_state(nx, ny, nz, npml=npml, device=dev())
    gen = torch.Generator(device="cpu").manual_seed(nx + ny + nz)
    init = init._replace(**{k: torch.randn(getattr(init, k).shape, generator=gen).to(dev())
                            for k in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")})
    ref_s, ref_a = run_3d(init, c, n, source=src, monitors=mons, variant=2)
    st, accs = run_3d(init, c, n, source=src, monitors=mons, variant=3, geometry=geometry)
    bad = [k for k, v in ref_s._asdict().items()
           if v is not None and not torch.equal(v, getattr(st, k))]
    bad += [f"acc_{q}" for q, (a, b) in enumerate(zip(accs, ref_a)) if not torch.equal(a, b)]
    assert not bad, bad


def test_3d_one_pass_refuses_damping_and_wide_z():
    """Variant 3 asked for explicitly on a plan it does not cover (conductive damping,
    zpitch > 256) is refused before any device work; the default falls back to the
    split kernels there."""
    from meep_torch_b200.core.monitors_3d import run_3d
    from meep_torch_b200.core.stepper_3d import build_3d_coeffs, init_3d_state
    from meep_torch_b200._lib import MtbUnsupported
    c = build_3d_coeffs(8, 8, 300, 0.05, eps=2.0, npml=2, device=dev())
    s0 = init_3d_state(8, 8, 300, npml=2, device=dev())
    with pytest.raises(MtbUnsupported):
        run_3d(s0, c, 2, variant=3)
    run_3d(s0, c, 2)
    sig = torch.full((8, 8, 8), 0.3)
    c = build_3d_coeffs(8, 8, 8, 0.05, eps=2.0, npml=2, sigma_d=sig, sigma_b=sig, device=dev())
    s0 = init_3d_state(8, 8, 8, npml=2, device=dev())
    with pytest.raises(MtbUnsupported):
        run_3d(s0, c, 2, variant=3)
    run_3d(s0, c, 2)


@pytest.mark.parametrize("n_slabs", [1, 2, 3])
@pytest.mark.parametrize("plane_source", [False, True])
def test_3d_slabs_bitwise_equal_to_whole_grid(n_slabs, plane_source):
    """One grid split into x slabs (a plan per slab on its owned planes, halo planes
    copied between the H and E halves) reproduces the whole-grid run bit for bit:
    fields, CPML memory and the flux / DFT accumulators of planes of every
    orientation, some crossing slab boundaries. n_slabs = 1 checks the half-step
    entry points against mtb_yee3d_run."""
    from meep_torch_b200.core.monitors_3d import (DFTFieldsMonitor3D, FluxMonitor3D,
                                                  PlaneSource, PointSource3D, run_3d)
    from meep_torch_b200.core.sources import GaussianPulse
    from meep_torch_b200.core.stepper_3d import build_3d_coeffs, init_3d_state
    from meep_torch_b200.slab3d import run_3d_slabs
    nx, ny, nz, dx, npml, n = 23, 17, 40, 0.05, 4, 50
    rng = np.random.default_rng(12)
    eps = (1.0 + 3.0 * rng.random((nx, ny, nz))).astype(np.float32)
    c = build_3d_coeffs(nx, ny, nz, dx, eps=torch.from_numpy(eps), npml=npml, device=dev())
    freqs = [0.8, 1.1, 1.4]
    prof = GaussianPulse(1.0, 2.0)
    if plane_source:
        src = PlaneSource(nx, ny, nz, c.dt, "Ez", 1, 8, prof, lo=3, hi=19, device=dev())
    else:
        src = PointSource3D(c.dt, "Ez", 11, 8, 20, prof)
    mons = [FluxMonitor3D(c.dt, freqs, normal="x", idx=8, win=(2, 14, 3, 30)),
            FluxMonitor3D(c.dt, freqs, normal="x", idx=16, ap=2),
            FluxMonitor3D(c.dt, freqs, normal="y", idx=10, win=(3, 20, 2, 35)),
            FluxMonitor3D(c.dt, freqs, normal="z", idx=21, ap=1),
            DFTFieldsMonitor3D(c.dt, freqs, component="Ez", plane=(2, 17)),
            DFTFieldsMonitor3D(c.dt, freqs, component="Hy", plane=(0, 12))]
    init = init_3d_state(nx, ny, nz, npml=npml, device=dev())
    init = init._replace(**{k: torch.randn(getattr(init, k).shape, device=dev())
                            for k in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")})
    ref_s, ref_a = run_3d(init, c, n, source=src, monitors=mons)
    st, accs = run_3d_slabs(init, c, n, source=src, monitors=mons, n_slabs=n_slabs)
    bad = [k for k, v in ref_s._asdict().items()
           if v is not None and not torch.equal(v, getattr(st, k))]
    bad += [f"acc_{q}" for q, (a, b) in enumerate(zip(accs, ref_a)) if not torch.equal(a, b)]
    assert not bad, bad


def test_autotune_picks_a_candidate_that_matches_the_default():
    """autotune_2d times every candidate launch shape on the batch and returns the fastest;
    the batch advanced with it agrees with the library default (different kernels, same
    arithmetic up to rounding)."""
    from meep_torch_b200 import workloads as W
    from meep_torch_b200.engine2d import Engine2D
    from meep_torch_b200.tune import DEFAULT_CANDIDATES, autotune_2d
    specs = W.cfg2_specs(n=6, seed=4, lo=96, hi=260)
    items = [W.cfg2_item(s, dev()) for s in specs]
    best, table = autotune_2d(items, steps=40, warmup=8)
    assert len(table) == len(DEFAULT_CANDIDATES) and all(ms > 0 for _, ms in table)
    assert best in [dict(c) for c in DEFAULT_CANDIDATES]
    outs = []
    for kw in ({}, best):
        eng = Engine2D([W.cfg2_item(s, dev()) for s in specs], **kw)
        eng.run(0, 70)
        outs.append([eng.state(b) for b in range(len(specs))])
        eng.close()
    for a, b in zip(*outs):
        main = "Ez" if hasattr(a, "Dz") else "Hz"
        assert rel_l2(getattr(a, main).cpu().numpy(), getattr(b, main).cpu().numpy()) < 1e-5


def test_conductivity_batched_tiles_match_oracle_and_other_paths_refuse():
    """Electric conductivity in a batch large enough for four rows per warp (the tiles
    then run the general rows on every warp of a conductive structure), from random
    fields, against the oracle; the row march refuses it (MTB_UNSUPPORTED)."""
    from meep_torch_b200._lib import MtbUnsupported
    from meep_torch_b200.core.coeffs import build_te_coeffs, build_tm_coeffs
    from meep_torch_b200.core.grid import Grid
    from meep_torch_b200.core.stepper_te import init_te_state
    from meep_torch_b200.core.stepper_tm import init_tm_state
    from meep_torch_b200.engine2d import Engine2D
    rng = np.random.default_rng(23)
    n, npml, dx = 30, 8, 0.05
    specs = [("tm", 300, 260), ("te", 280, 300)] * 40
    items, refs = [], []
    for q, (pol, nx, ny) in enumerate(specs):
        eps = (1.0 + 3.0 * rng.random((nx, ny))).astype(np.float32)
        sig = np.zeros((nx, ny), dtype=np.float32)
        sig[nx // 3: nx // 2, :] = 2.0
        grid = Grid(nx=nx, ny=ny, dx=dx, device=dev())
        kw = dict(eps_inf=torch.from_numpy(eps), npml=npml, sigma_d=torch.from_numpy(sig))
        if pol == "tm":
            c = O.tm_coeffs(nx, ny, dx, eps=eps, npml=npml, dtype=np.float32, sigma=sig)
            so = O.tm_state(c)
            for k in ("Dz", "Hx", "Hy"):
                so[k] = rng.standard_normal(so[k].shape).astype(np.float32)
            m = build_tm_coeffs(grid, **kw)
            so["Ez"] = (torch.from_numpy(so["Dz"]) / m.eps_inf.cpu()).numpy()
            s0 = init_tm_state(grid)._replace(
                **{k: torch.from_numpy(so[k]).to(dev()) for k in ("Ez", "Dz", "Hx", "Hy")})
            step = O.tm_step
        else:
            c = O.te_coeffs(nx, ny, dx, eps=eps, npml=npml, dtype=np.float32, sigma=sig)
            so = O.te_state(c)
            for k in ("Hz", "Dx", "Dy"):
                so[k] = rng.standard_normal(so[k].shape).astype(np.float32)
            so["Ex"], so["Ey"] = so["Dx"] / c["eps_x"], so["Dy"] / c["eps_y"]
            m = build_te_coeffs(grid, **kw)
            s0 = init_te_state(grid)._replace(
                **{k: torch.from_numpy(so[k]).to(dev()) for k in ("Hz", "Dx", "Dy", "Ex", "Ey")})
            step = O.te_step
        items.append((s0, m, None, []))
        if q < 2:
            refs.append(O.run_2d(step, so, c, n)[0])
    eng = Engine2D(items)
    eng.run(0, n)
    for b, ref in enumerate(refs):
        st = eng.state(b)
        for k in (("Ez", "Dz", "Hx", "Hy") if b == 0 else ("Hz", "Dx", "Dy", "Ex", "Ey")):
            assert rel_l2(getattr(st, k).cpu().numpy(), ref[k]) < TOL, (b, k)
    eng.close()
    with pytest.raises(MtbUnsupported):
        Engine2D(items[:1], variant=1)


def test_magnetic_batched_tiles_match_oracle_and_other_paths_refuse():
    """Magnetic conductivity and permeability (with an electric conductivity slab) in
    a batch large enough for four rows per warp, from random fields, against the
    oracle: every H site of the tiles (TM Hx, Hy and the recomputed Hy row and Hx
    column; TE Hz) applies the (h1, h2) pairs. The row march and the TE adjoint refuse
    them (MTB_UNSUPPORTED)."""
    from meep_torch_b200._lib import MtbUnsupported
    from meep_torch_b200.core.coeffs import build_te_coeffs, build_tm_coeffs
    from meep_torch_b200.core.grid import Grid
    from meep_torch_b200.core.monitors import DFTFieldsMonitor
    from meep_torch_b200.core.run import run_te
    from meep_torch_b200.core.sources import GaussianPulse, LineSource
    from meep_torch_b200.core.stepper_te import init_te_state
    from meep_torch_b200.core.stepper_tm import init_tm_state
    from meep_torch_b200.engine2d import Engine2D
    rng = np.random.default_rng(29)
    n, npml, dx = 30, 8, 0.05
    specs = [("tm", 300, 260), ("te", 280, 300)] * 40
    items, refs = [], []
    for q, (pol, nx, ny) in enumerate(specs):
        eps = (1.0 + 3.0 * rng.random((nx, ny))).astype(np.float32)
        sig = np.zeros((nx, ny), dtype=np.float32)
        sig[nx // 3: nx // 2, :] = 1.0
        sb = np.zeros((nx, ny), dtype=np.float32)
        sb[:, ny // 4: ny // 3] = 2.5
        sb[nx // 2:, :] += (2.0 * rng.random((nx - nx // 2, ny))).astype(np.float32)
        mu = (1.0 + 2.0 * rng.random((nx, ny))).astype(np.float32)
        grid = Grid(nx=nx, ny=ny, dx=dx, device=dev())
        kw = dict(eps_inf=torch.from_numpy(eps), npml=npml, sigma_d=torch.from_numpy(sig),
                  sigma_b=torch.from_numpy(sb), mu=torch.from_numpy(mu))
        okw = dict(eps=eps, npml=npml, dtype=np.float32, sigma=sig, sigma_b=sb, mu=mu)
        if pol == "tm":
            c = O.tm_coeffs(nx, ny, dx, **okw)
            so = O.tm_state(c)
            for k in ("Dz", "Hx", "Hy"):
                so[k] = rng.standard_normal(so[k].shape).astype(np.float32)
            m = build_tm_coeffs(grid, **kw)
            so["Ez"] = (torch.from_numpy(so["Dz"]) / m.eps_inf.cpu()).numpy()
            s0 = init_tm_state(grid)._replace(
                **{k: torch.from_numpy(so[k]).to(dev()) for k in ("Ez", "Dz", "Hx", "Hy")})
            step = O.tm_step
        else:
            c = O.te_coeffs(nx, ny, dx, **okw)
            so = O.te_state(c)
            for k in ("Hz", "Dx", "Dy"):
                so[k] = rng.standard_normal(so[k].shape).astype(np.float32)
            so["Ex"], so["Ey"] = so["Dx"] / c["eps_x"], so["Dy"] / c["eps_y"]
            m = build_te_coeffs(grid, **kw)
            s0 = init_te_state(grid)._replace(
                **{k: torch.from_numpy(so[k]).to(dev()) for k in ("Hz", "Dx", "Dy", "Ex", "Ey")})
            step = O.te_step
        items.append((s0, m, None, []))
        if q < 2:
            refs.append(O.run_2d(step, so, c, n)[0])
    eng = Engine2D(items)
    eng.run(0, n)
    for b, ref in enumerate(refs):
        st = eng.state(b)
        for k in (("Ez", "Dz", "Hx", "Hy") if b == 0 else ("Hz", "Dx", "Dy", "Ex", "Ey")):
            assert rel_l2(getattr(st, k).cpu().numpy(), ref[k]) < TOL, (b, k)
    eng.close()
    with pytest.raises(MtbUnsupported):
        Engine2D(items[:1], variant=1)
    # gradients: TE magnetic pairs have an adjoint; a nonlinear (chi3) TE run does not
    grid = Grid(nx=40, ny=40, dx=dx, device=dev())
    eps = torch.ones(40, 40, device=dev(), requires_grad=True)
    m = build_te_coeffs(grid, eps_inf=eps, npml=8, sigma_b=torch.full((40, 40), 0.5))
    _, (acc,) = run_te(init_te_state(grid), m, 10,
                       monitors=[DFTFieldsMonitor(grid, [0.5], "Hz")])
    acc.sum().backward()
    assert bool(torch.isfinite(eps.grad).all())
    eps2 = torch.ones(40, 40, device=dev(), requires_grad=True)
    m = build_te_coeffs(grid, eps_inf=eps2, npml=8, chi3=torch.full((40, 40), 0.5))
    _, (acc,) = run_te(init_te_state(grid), m, 10,
                       monitors=[DFTFieldsMonitor(grid, [0.5], "Hz")])
    with pytest.raises(MtbUnsupported):
        acc.sum().backward()


def test_poles_batched_tiles_match_oracle_from_random_state():
    """Lorentz and Drude poles in a batch that gets four rows per warp, from random
    fields and polarisations, against the oracle (fields, CPML memory, both P buffers);
    a pole-free structure in the same batch keeps the lean rows. The row march refuses
    poles (MTB_UNSUPPORTED)."""
    from meep_torch_b200._lib import MtbUnsupported
    from meep_torch_b200.core.coeffs import build_tm_coeffs
    from meep_torch_b200.core.grid import Grid
    from meep_torch_b200.core.stepper_tm import init_tm_state
    from meep_torch_b200.engine2d import Engine2D
    rng = np.random.default_rng(31)
    n, npml, dx = 30, 8, 0.05
    poles = [(0.7, 0.05, 1.5), (0.0, 0.1, 1.0, 0.9)]
    items, refs = [], []
    for q in range(60):
        nx, ny = (300, 260) if q % 2 == 0 else (260, 300)
        use = q % 3 != 2
        eps = (1.0 + 3.0 * rng.random((nx, ny))).astype(np.float32)
        masks = [(rng.random((nx, ny)) < 0.5).astype(np.float32) for _ in poles] if use else None
        grid = Grid(nx=nx, ny=ny, dx=dx, device=dev())
        pl = poles if use else ()
        c = O.tm_coeffs(nx, ny, dx, eps=eps, npml=npml, dtype=np.float32, poles=pl,
                        pole_masks=masks)
        so = O.tm_state(c)
        for k in ("Dz", "Hx", "Hy", "P_cur", "P_prev"):
            so[k] = (0.1 if k.startswith("P") else 1.0) * \
                rng.standard_normal(so[k].shape).astype(np.float32)
        so["Ez"] = (so["Dz"] - so["P_cur"].sum(0)) / c["eps"]
        m = build_tm_coeffs(grid, eps_inf=torch.from_numpy(eps), npml=npml, poles=pl,
                            pole_masks=None if masks is None else
                            [torch.from_numpy(x) for x in masks])
        s0 = init_tm_state(grid, n_poles=len(pl))._replace(
            **{k: torch.from_numpy(so[k]).to(dev())
               for k in ("Ez", "Dz", "Hx", "Hy", "P_cur", "P_prev")})
        items.append((s0, m, None, []))
        if q < 3:
            refs.append(O.run_2d(O.tm_step, so, c, n)[0])
    eng = Engine2D(items)
    eng.run(0, n)
    for b, ref in enumerate(refs):
        st = eng.state(b)
        names = ["Ez", "Dz", "Hx", "Hy", "psi_Ezy", "psi_Ezx", "psi_Hyx", "psi_Hxy"]
        if b % 3 != 2:
            names += ["P_cur", "P_prev"]
        for k in names:
            assert rel_l2(getattr(st, k).cpu().numpy(), ref[k]) < TOL, (b, k)
    eng.close()
    with pytest.raises(MtbUnsupported):
        Engine2D(items[:1], variant=1)


def test_te_poles_batched_tiles_match_oracle_from_random_state():
    """TE with Lorentz and Drude poles on both E axes in a batch that gets four rows per
    warp, from random fields and polarisations, against the oracle (fields, CPML memory,
    both P buffers of each axis)."""
    from meep_torch_b200.core.coeffs import build_te_coeffs
    from meep_torch_b200.core.grid import Grid
    from meep_torch_b200.core.stepper_te import init_te_state
    from meep_torch_b200.engine2d import Engine2D
    rng = np.random.default_rng(37)
    n, npml, dx = 30, 8, 0.05
    poles = [(0.7, 0.05, 1.5), (0.0, 0.1, 1.0, 0.9)]
    items, refs = [], []
    for q in range(60):
        nx, ny = (300, 260) if q % 2 == 0 else (260, 300)
        use = q % 3 != 2
        eps = (1.0 + 3.0 * rng.random((nx, ny))).astype(np.float32)
        masks = [(rng.random((nx, ny)) < 0.5).astype(np.float32) for _ in poles] if use else None
        grid = Grid(nx=nx, ny=ny, dx=dx, device=dev())
        pl = poles if use else ()
        c = O.te_coeffs(nx, ny, dx, eps=eps, npml=npml, dtype=np.float32, poles=pl,
                        pole_masks=masks)
        so = O.te_state(c)
        for k in ("Hz", "Dx", "Dy", "Px_cur", "Px_prev", "Py_cur", "Py_prev"):
            so[k] = (0.1 if k.startswith("P") else 1.0) * \
                rng.standard_normal(so[k].shape).astype(np.float32)
        so["Ex"] = (so["Dx"] - so["Px_cur"].sum(0)) / c["eps_x"]
        so["Ey"] = (so["Dy"] - so["Py_cur"].sum(0)) / c["eps_y"]
        m = build_te_coeffs(grid, eps_inf=torch.from_numpy(eps), npml=npml, poles=pl,
                            pole_masks=None if masks is None else
                            [torch.from_numpy(x) for x in masks])
        s0 = init_te_state(grid, n_poles=len(pl))._replace(
            **{k: torch.from_numpy(so[k]).to(dev())
               for k in ("Hz", "Dx", "Dy", "Ex", "Ey", "Px_cur", "Px_prev", "Py_cur", "Py_prev")})
        items.append((s0, m, None, []))
        if q < 3:
            refs.append(O.run_2d(O.te_step, so, c, n)[0])
    eng = Engine2D(items)
    eng.run(0, n)
    for b, ref in enumerate(refs):
        st = eng.state(b)
        names = ["Hz", "Dx", "Dy", "Ex", "Ey", "psi_Eyx", "psi_Exy", "psi_Hzy", "psi_Hzx"]
        if b % 3 != 2:
            names += ["Px_cur", "Px_prev", "Py_cur", "Py_prev"]
        for k in names:
            assert rel_l2(getattr(st, k).cpu().numpy(), ref[k]) < TOL, (b, k)
    eng.close()


def test_3d_damping_refused_by_fused_kernel():
    """Conductive damping runs on the split kernels only (the fused x-march refuses it
    with MTB_UNSUPPORTED)."""
    from meep_torch_b200._lib import MtbUnsupported
    from meep_torch_b200.core.monitors_3d import run_3d
    from meep_torch_b200.core.stepper_3d import build_3d_coeffs, init_3d_state
    n = 12
    sd = torch.zeros(n, n, n)
    sd[4:8] = 1.0
    c = build_3d_coeffs(n, n, n, 0.0625, npml=3, device=dev(), sigma_d=sd)
    s0 = init_3d_state(n, n, n, npml=3, device=dev())
    with pytest.raises(MtbUnsupported):
        run_3d(s0, c, 2, variant=1)


def test_3d_poles_slabs_bitwise_equal_to_whole_grid():
    """3D poles (random P stacks and fields) through the x-slab decomposition: two and three
    slabs reproduce the whole-grid run bit for bit, pole stacks included."""
    from meep_torch_b200.core.monitors_3d import FluxMonitor3D, run_3d
    from meep_torch_b200.core.stepper_3d import build_3d_coeffs, init_3d_state
    from meep_torch_b200.slab3d import run_3d_slabs
    nx, ny, nz, dx, npml, n = 21, 15, 24, 0.0625, 4, 30
    g = torch.Generator().manual_seed(5)
    masks = [torch.zeros(nx, ny, nz), torch.zeros(nx, ny, nz)]
    masks[0][6:15, 5:10, 6:18] = 1.0
    masks[1][9:13, 4:11, 8:12] = 1.0
    c = build_3d_coeffs(nx, ny, nz, dx, npml=npml, device=dev(),
                        poles=[(0.5, 0.05, 2.0), (0.0, 0.1, 1.0, 0.8)], pole_masks=masks)
    s0 = init_3d_state(nx, ny, nz, npml=npml, device=dev(), n_poles=2)
    s0 = s0._replace(**{k: 0.1 * torch.randn(getattr(s0, k).shape, generator=g).to(dev())
                        for k in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz", "Px_cur", "Px_prev",
                                  "Py_cur", "Py_prev", "Pz_cur", "Pz_prev")})
    mons = [FluxMonitor3D(c.dt, [0.5, 0.7], normal="y", idx=7, win=(2, 18, 3, 20))]
    ref_s, ref_a = run_3d(s0, c, n, monitors=mons)
    for n_slabs in (2, 3):
        st, accs = run_3d_slabs(s0, c, n, monitors=mons, n_slabs=n_slabs)
        bad = [k for k, v in ref_s._asdict().items()
               if v is not None and not torch.equal(v, getattr(st, k))]
        bad += ["acc"] if not torch.equal(accs[0], ref_a[0]) else []
        assert not bad, (n_slabs, bad)
