"""Config-scale fixtures: the REFERENCE run on the benchmark configurations.

Imports meep_torch from the reference checkout named by ``MEEP_TORCH_REF`` (read-only,
no bytecode written) and runs the configurations at their own sizes and lengths, in
float32 (the parity target) and float64 (the error floor), on all host threads:

* cfg1: 320 x 160 TM waveguide, Gaussian point source, one 50-frequency flux line,
  4000 steps (``build_tm_coeffs`` + ``LineSource`` + ``FluxMonitorTM`` + ``run_tm``,
  core/run.py:125);
* cfg2: four of the 256 seeded bends (two TM, two TE, among them the widest grid of the
  batch), full-grid 3-frequency DFT and two flux lines, 5000 steps (``run_tm`` /
  ``run_te``, core/run.py:125-126);
* cfg3: the 256^3 sphere grid with the centre Ez dipole and the six 20-frequency flux
  faces, ``build_3d_coeffs`` + ``run_3d`` (core/monitors_3d.py:192), 2000 steps;
* cfg4: the 600 x 400 design problem's objective and d J / d rho through the reference's
  ``OptimizationProblem`` (adjoint/problem.py:97) over ``run_tm(checkpoint_every=256)``,
  8000 steps; and (``cfg4fd``, float64 only) central finite differences of the objective on
  32 random design pixels.

The inputs are the seeded synthetic configurations of ``meep_torch_b200.workloads``
(numpy only). The fixtures stay small: monitor accumulators and flux spectra in full
where they are small, strided subsamples of the full-grid arrays (the stride is stored
beside them), and the full arrays' L2 norms. Usage::

    MEEP_TORCH_REF=<checkout> python tests/golden/make_config_golden.py cfg1 cfg2 cfg3 cfg4
"""
from __future__ import annotations

import os
import sys
import time

import numpy as np

sys.dont_write_bytecode = True
HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.abspath(os.path.join(HERE, "..", "..")))
from reference_path import reference_root  # noqa: E402

sys.path.insert(0, reference_root())

import torch  # noqa: E402

from meep_torch.core.coeffs import build_te_coeffs, build_tm_coeffs  # noqa: E402
from meep_torch.core.grid import Grid  # noqa: E402
from meep_torch.core.monitors import (DFTFieldsMonitor, FluxMonitorTE,  # noqa: E402
                                      FluxMonitorTEY, FluxMonitorTM)
from meep_torch.core.monitors_3d import FluxMonitor3D, PointSource3D, run_3d  # noqa: E402
from meep_torch.core.run import run_te, run_tm  # noqa: E402
from meep_torch.core.sources import GaussianPulse, LineSource  # noqa: E402
from meep_torch.core.stepper_3d import build_3d_coeffs, init_3d_state  # noqa: E402
from meep_torch.core.stepper_te import init_te_state  # noqa: E402
from meep_torch.core.stepper_tm import init_tm_state  # noqa: E402

from meep_torch_b200 import workloads as W  # noqa: E402

DT = {"f64": torch.float64, "f32": torch.float32}
# cfg2 variants checked at full length: two TM (even index) and two TE (odd index)
# of the seeded batch; 0 and 1 are the first of each, the others are the TM and TE
# structures with the most cells.
FIELD_STRIDE_2D = 4
DFT_STRIDE_2D = 8
FIELD_STRIDE_3D = 16
FACE_STRIDE_3D = 8


def _np(t):
    return t.detach().cpu().to(torch.float64).numpy()


def _sub(a, stride, lead=0):
    """Strided subsample of the trailing two axes (offset stride // 2), as float32."""
    o = stride // 2
    sl = (slice(None),) * lead + (slice(o, None, stride), slice(o, None, stride))
    return np.ascontiguousarray(a[sl]).astype(np.float32)


def cfg2_variants(specs):
    tm = [b for b in range(len(specs)) if specs[b]["pol"] == "tm"]
    te = [b for b in range(len(specs)) if specs[b]["pol"] == "te"]
    big_tm = max(tm[1:], key=lambda b: specs[b]["nx"] * specs[b]["ny"])
    big_te = max(te[1:], key=lambda b: specs[b]["nx"] * specs[b]["ny"])
    return [tm[0], te[0], big_tm, big_te]


def cfg1_case(prec):
    sp = W.cfg1_spec()
    nx, ny = sp["nx"], sp["ny"]
    g = Grid(nx=nx, ny=ny, dx=W.DX2D, dtype=DT[prec], device="cpu")
    m = build_tm_coeffs(g, eps_inf=torch.tensor(sp["eps"], dtype=DT[prec]), npml=W.NPML2D)
    i, j = sp["src"]
    src = LineSource(g, ix=i, j0=j, j1=j + 1, profile=GaussianPulse(0.15, 0.1))
    ix, lo, hi = sp["flux"]
    mon = FluxMonitorTM(g, list(sp["freqs"]), x_normal=True, idx=ix, lo=lo, hi=hi)
    with torch.no_grad():
        st, (acc,) = run_tm(init_tm_state(g), m, sp["steps"], source=src, monitors=[mon])
    out = dict(n_steps=sp["steps"], acc=_np(acc), flux=_np(mon.flux(acc, W.DX2D)),
               field_stride=FIELD_STRIDE_2D)
    for k in ("Ez", "Hx", "Hy"):
        a = _np(getattr(st, k))
        out["s_" + k] = _sub(a, FIELD_STRIDE_2D)
        out["norm_" + k] = np.linalg.norm(a)
    return out


def cfg2_case(prec, spec):
    nx, ny = spec["nx"], spec["ny"]
    g = Grid(nx=nx, ny=ny, dx=W.DX2D, dtype=DT[prec], device="cpu")
    eps = torch.tensor(spec["eps"], dtype=DT[prec])
    line = LineSource(g, ix=spec["src_ix"], j0=spec["src_j"][0], j1=spec["src_j"][1],
                      profile=GaussianPulse(0.65, 0.2))
    fx, fy = spec["flux_x"], spec["flux_y"]
    freqs = list(W.CFG2_FREQS)
    n = 5000
    with torch.no_grad():
        if spec["pol"] == "tm":
            m = build_tm_coeffs(g, eps_inf=eps, npml=W.NPML2D)
            mons = [DFTFieldsMonitor(g, freqs, "Ez"),
                    FluxMonitorTM(g, freqs, x_normal=True, idx=fx[0], lo=fx[1], hi=fx[2]),
                    FluxMonitorTM(g, freqs, x_normal=False, idx=fy[0], lo=fy[1], hi=fy[2])]
            st, accs = run_tm(init_tm_state(g), m, n, source=line, monitors=mons)
            comps = ("Ez", "Hx", "Hy")
        else:
            m = build_te_coeffs(g, eps_inf=eps, npml=W.NPML2D)

            class _TESrc:                       # Simulation's TE binding: mask[:, :-1] -> Dy
                mask = line.mask[:, :-1]        # (mp/simulation.py:867-869)
                amplitude = staticmethod(line.amplitude)

            mons = [DFTFieldsMonitor(g, freqs, "Hz"),
                    FluxMonitorTE(g, freqs, ix=fx[0], lo=fx[1], hi=fx[2]),
                    FluxMonitorTEY(g, freqs, iy=fy[0], lo=fy[1], hi=fy[2])]
            st, accs = run_te(init_te_state(g), m, n, source=_TESrc(), monitors=mons)
            comps = ("Hz", "Ex", "Ey")
    dft = _np(accs[0])
    out = dict(n_steps=n, nx=nx, ny=ny, pol=spec["pol"], field_stride=FIELD_STRIDE_2D,
               dft_stride=DFT_STRIDE_2D, dft=_sub(dft, DFT_STRIDE_2D, lead=2),
               norm_dft=np.linalg.norm(dft), acc_x=_np(accs[1]), acc_y=_np(accs[2]),
               flux_x=_np(mons[1].flux(accs[1], W.DX2D)),
               flux_y=_np(mons[2].flux(accs[2], W.DX2D)))
    for k in comps:
        a = _np(getattr(st, k))
        out["s_" + k] = _sub(a, FIELD_STRIDE_2D)
        out["norm_" + k] = np.linalg.norm(a)
    return out


def cfg3_case(prec, n_steps=2000):
    n, npml, dx = 256, 16, 1.0 / 16
    eps = torch.tensor(W.cfg3_eps(n), dtype=DT[prec])
    c = build_3d_coeffs(n, n, n, dx, eps=eps, npml=npml, dtype=DT[prec])
    s0 = init_3d_state(n, n, n, npml=npml, dtype=DT[prec])
    src = PointSource3D(c.dt, "Ez", n // 2, n // 2, n // 2, GaussianPulse(0.5, 0.3))
    freqs = np.linspace(0.35, 0.65, 20).tolist()
    mons = [FluxMonitor3D(c.dt, freqs, normal=a, idx=i, win=(24, 232, 24, 232),
                          dtype=DT[prec]) for a, i in W.CFG3_FACES]
    with torch.no_grad():
        st, accs = run_3d(s0, c, n_steps, source=src, monitors=mons)
    out = dict(n_steps=n_steps, field_stride=FIELD_STRIDE_3D, face_stride=FACE_STRIDE_3D)
    for k in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz"):
        a = _np(getattr(st, k))
        o = FIELD_STRIDE_3D // 2
        out["s_" + k] = np.ascontiguousarray(
            a[o::FIELD_STRIDE_3D, o::FIELD_STRIDE_3D, o::FIELD_STRIDE_3D]).astype(np.float32)
        out["norm_" + k] = np.linalg.norm(a)
    out["ez_mid"] = _np(st.Ez)[:, :, n // 2].astype(np.float32)
    for i, (a, mon) in enumerate(zip(accs, mons)):
        an = _np(a)
        out[f"flux_{i}"] = _np(mon.flux(a, dx))
        out[f"acc_{i}"] = _sub(an, FACE_STRIDE_3D, lead=2)
        out[f"norm_acc_{i}"] = np.linalg.norm(an)
    return out


def cfg4_case(prec, steps=None):
    """J and d J / d rho of the cfg4-shaped problem through the reference's design
    chain (conic_filter, tanh_projection, MaterialGrid, DesignRegion, OptimizationProblem)
    and its autograd through run_tm(checkpoint_every=256) in float32; float64 checkpoints
    every 64 steps (the same gradient; 256-step float64 segments exceed this machine's
    memory)."""
    from meep_torch.adjoint.problem import DesignRegion, MaterialGrid, OptimizationProblem
    c = W.CFG4
    nx, ny, dx, npml = c["nx"], c["ny"], c["dx"], c["npml"]
    n = steps or c["steps"]
    dt_ = DT[prec]
    rng = np.random.default_rng(4)
    base = torch.full((nx, ny), c["eps_bg"], dtype=dt_)
    y0, y1 = ny // 2 - c["guide_w"] // 2, ny // 2 + c["guide_w"] // 2
    base[:, y0:y1] = c["eps_core"]
    d = c["design"]
    ix0, iy0 = nx // 2 - d // 2, ny // 2 - d // 2
    reg = DesignRegion(MaterialGrid((d, d), c["eps_bg"], c["eps_core"]),
                       ix0=ix0, ix1=ix0 + d, iy0=iy0, iy1=iy0 + d)
    grid = Grid(nx=nx, ny=ny, dx=dx, dtype=dt_, device="cpu")
    src = LineSource(grid, ix=npml + 10, j0=y0 - 10, j1=y1 + 10,
                     profile=GaussianPulse(0.645, 0.12))
    mon = FluxMonitorTM(grid, list(c["freqs"]), x_normal=True, idx=nx - npml - 10,
                        lo=y0 - 20, hi=y1 + 20)

    def run_fn(eps):
        m = build_tm_coeffs(grid, eps_inf=eps, npml=npml)
        _, (acc,) = run_tm(init_tm_state(grid), m, n, source=src, monitors=[mon],
                           checkpoint_every=256 if prec == "f32" else 64)
        return mon.flux(acc, dx).mean()

    rho0 = rng.uniform(0.4, 0.6, (d, d))
    opt = OptimizationProblem(run_fn, base, reg, filter_radius=c["radius"], dx=dx,
                              beta=c["beta"], eta=c["eta"], rho0=torch.tensor(rho0, dtype=dt_))
    J, g = opt()
    return dict(n_steps=n, rho0=rho0, J=float(J), grad=np.asarray(g, dtype=np.float64))


def cfg4_fd_case(n_pix=32, h=1e-4, steps=None):
    """Central differences of the float64 reference objective on n_pix random design
    pixels (np.random.default_rng(4): rho0 first, then the pixels), step h:
    (J(rho + h e_p) - J(rho - h e_p)) / 2h through OptimizationProblem.eval_at_delta
    (adjoint/problem.py:105-110), 8000 steps, checkpointing irrelevant (no_grad)."""
    from meep_torch.adjoint.problem import DesignRegion, MaterialGrid, OptimizationProblem
    c = W.CFG4
    nx, ny, dx, npml = c["nx"], c["ny"], c["dx"], c["npml"]
    n = steps or c["steps"]
    dt_ = torch.float64
    rng = np.random.default_rng(4)
    rho0 = rng.uniform(0.4, 0.6, (c["design"], c["design"]))
    pix = rng.choice(c["design"] * c["design"], n_pix, replace=False)
    base = torch.full((nx, ny), c["eps_bg"], dtype=dt_)
    y0, y1 = ny // 2 - c["guide_w"] // 2, ny // 2 + c["guide_w"] // 2
    base[:, y0:y1] = c["eps_core"]
    d = c["design"]
    ix0, iy0 = nx // 2 - d // 2, ny // 2 - d // 2
    reg = DesignRegion(MaterialGrid((d, d), c["eps_bg"], c["eps_core"]),
                       ix0=ix0, ix1=ix0 + d, iy0=iy0, iy1=iy0 + d)
    grid = Grid(nx=nx, ny=ny, dx=dx, dtype=dt_, device="cpu")
    src = LineSource(grid, ix=npml + 10, j0=y0 - 10, j1=y1 + 10,
                     profile=GaussianPulse(0.645, 0.12))
    mon = FluxMonitorTM(grid, list(c["freqs"]), x_normal=True, idx=nx - npml - 10,
                        lo=y0 - 20, hi=y1 + 20)

    def run_fn(eps):
        m = build_tm_coeffs(grid, eps_inf=eps, npml=npml)
        _, (acc,) = run_tm(init_tm_state(grid), m, n, source=src, monitors=[mon])
        return mon.flux(acc, dx).mean()

    opt = OptimizationProblem(run_fn, base, reg, filter_radius=c["radius"], dx=dx,
                              beta=c["beta"], eta=c["eta"], rho0=torch.tensor(rho0, dtype=dt_))
    fd = []
    for p in pix:
        i, j = int(p) // d, int(p) % d
        fd.append((opt.eval_at_delta(i, j, h) - opt.eval_at_delta(i, j, -h)) / (2 * h))
        print(f"  pixel {i},{j}: {fd[-1]:.6e}", flush=True)
    return dict(n_steps=n, h=h, pixels=np.asarray(pix), fd=np.asarray(fd))


def main(argv):
    torch.set_num_threads(os.cpu_count() or 1)
    which = argv or ["cfg1", "cfg2", "cfg3", "cfg4", "cfg4fd"]
    for arg in which:
        # "cfg4:f64" makes one precision; "cfg4:f64:4000" also shortens the run (the file
        # name then carries the step count)
        w, _, rest = arg.partition(":")
        only, _, nst = rest.partition(":")
        steps = int(nst) if nst else None
        if w == "cfg4fd":                       # float64 only
            t0 = time.time()
            np.savez_compressed(os.path.join(HERE, "config_cfg4_fd_f64.npz"), **cfg4_fd_case())
            print(f"cfg4fd f64: {time.time() - t0:.1f} s", flush=True)
            continue
        for prec in ("f32", "f64"):
            if only and prec != only:
                continue
            t0 = time.time()
            if w == "cfg1":
                np.savez_compressed(os.path.join(HERE, f"config_cfg1_{prec}.npz"),
                                    **cfg1_case(prec))
            elif w == "cfg2":
                specs = W.cfg2_specs()
                for b in cfg2_variants(specs):
                    np.savez_compressed(os.path.join(HERE, f"config_cfg2_b{b}_{prec}.npz"),
                                        index=b, **cfg2_case(prec, specs[b]))
            elif w == "cfg3":
                np.savez_compressed(os.path.join(HERE, f"config_cfg3_{prec}.npz"),
                                    **cfg3_case(prec))
            elif w == "cfg4":
                tag = f"_{steps}" if steps else ""
                np.savez_compressed(os.path.join(HERE, f"config_cfg4{tag}_{prec}.npz"),
                                    **cfg4_case(prec, steps))
            print(f"{w} {prec}: {time.time() - t0:.1f} s", flush=True)


if __name__ == "__main__":
    main(sys.argv[1:])
