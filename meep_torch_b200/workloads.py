"""Seeded synthetic inputs of the benchmark configurations.

cfg1  2D TM waveguide, 16 x 8 um at resolution 20 (320 x 160), 1 um PML,
      eps = 12 guide 1 um wide, Gaussian Ez point source (fcen 0.15,
      fwidth 0.1) at x = -6.5 um, one 50-frequency flux line at x = +6.5 um
      spanning 6 um, 4000 steps.
cfg2  256 independent 2D TE/TM bends (TM for even index, TE for odd), grid
      sides uniform in [256, 768] (numpy default_rng(2)), resolution 20,
      1 um PML: an eps = 12 input guide along +x and an output guide along +y
      meeting a 2 x 2 um design region of i.i.d. Bernoulli(0.5) pixels in
      {2.1, 12}; Gaussian line source (fcen 0.65, fwidth 0.2) across the input
      guide 1 um past the PML; DFT of Ez (TM) / Hz (TE) at 0.55, 0.65, 0.75
      over the full grid; an x-normal flux line on the input guide and a
      y-normal one on the output guide 1 um below the top PML; 5000 steps.
cfg3  3D 256^3 at resolution 16, 16-cell PML, 200 spheres (default_rng(3);
      centre U(1, 15) um, radius U(0.2, 0.6) um, eps U(2, 12), later spheres
      overwrite), Gaussian Ez dipole at the centre (fcen 0.5, fwidth 0.3), six
      20-frequency flux faces (linspace(0.35, 0.65, 20)) at cells 24 and 232
      on each axis with window [24, 232)^2, 2000 steps.

No public dataset is involved; these are the configurations' own shapes.
"""
from __future__ import annotations

import numpy as np
import torch

RES2D = 20
DX2D = 1.0 / RES2D
NPML2D = 20
CFG2_FREQS = (0.55, 0.65, 0.75)


def cfg2_specs(n: int = 256, seed: int = 2, lo: int = 256, hi: int = 768):
    """Per-structure geometry of cfg2 (eps as float32 numpy)."""
    rng = np.random.default_rng(seed)
    specs = []
    for b in range(n):
        nx, ny = (int(v) for v in rng.integers(lo, hi + 1, size=2))
        pol = "tm" if b % 2 == 0 else "te"
        eps = np.ones((nx, ny), dtype=np.float32)
        cx, cy = nx // 2, ny // 2
        half_w = RES2D // 2                        # 1 um guides
        eps[:cx - 20, cy - half_w:cy + half_w] = 12.0      # input guide along +x
        eps[cx - half_w:cx + half_w, cy + 20:] = 12.0      # output guide along +y
        pix = rng.random((40, 40)) < 0.5
        eps[cx - 20:cx + 20, cy - 20:cy + 20] = np.where(pix, 12.0, 2.1)
        specs.append(dict(nx=nx, ny=ny, pol=pol, eps=eps, src_ix=NPML2D + RES2D,
                          src_j=(cy - half_w, cy + half_w), flux_x=(NPML2D + RES2D + 10,
                                                                     cy - 15, cy + 15),
                          flux_y=(ny - NPML2D - RES2D, cx - 15, cx + 15)))
    return specs


def cfg2_item(spec, device, eps_t=None, freqs=CFG2_FREQS):
    """(state, coeffs, source, monitors) of one cfg2 structure via the public API."""
    from .core.coeffs import build_te_coeffs, build_tm_coeffs
    from .core.grid import Grid
    from .core.monitors import DFTFieldsMonitor, FluxMonitorTE, FluxMonitorTEY, FluxMonitorTM
    from .core.sources import GaussianPulse, LineSource, TESource
    from .core.stepper_te import init_te_state
    from .core.stepper_tm import init_tm_state
    nx, ny = spec["nx"], spec["ny"]
    g = Grid(nx=nx, ny=ny, dx=DX2D, device=device)
    eps = eps_t if eps_t is not None else torch.from_numpy(spec["eps"]).to(device)
    src = LineSource(g, ix=spec["src_ix"], j0=spec["src_j"][0], j1=spec["src_j"][1],
                     profile=GaussianPulse(0.65, 0.2))
    fx, fy = spec["flux_x"], spec["flux_y"]
    if spec["pol"] == "tm":
        m = build_tm_coeffs(g, eps_inf=eps, npml=NPML2D)
        mons = [DFTFieldsMonitor(g, freqs, "Ez"),
                FluxMonitorTM(g, freqs, x_normal=True, idx=fx[0], lo=fx[1], hi=fx[2]),
                FluxMonitorTM(g, freqs, x_normal=False, idx=fy[0], lo=fy[1], hi=fy[2])]
        return init_tm_state(g), m, src, mons
    m = build_te_coeffs(g, eps_inf=eps, npml=NPML2D)
    mons = [DFTFieldsMonitor(g, freqs, "Hz"),
            FluxMonitorTE(g, freqs, ix=fx[0], lo=fx[1], hi=fx[2]),
            FluxMonitorTEY(g, freqs, iy=fy[0], lo=fy[1], hi=fy[2])]
    return init_te_state(g), m, TESource(src), mons


def cfg2_bytes_per_step(specs, npml: int = NPML2D) -> float:
    """Algorithmic HBM bytes of one time step of the batch: read+write of the
    three stored fields (12 B read + 12 B write per cell), eps (4 B TM, 8 B TE:
    eps_x and eps_y), and read+write of the CPML memory inside the layers
    (8 B per psi cell: two psi arrays per axis band)."""
    total = 0.0
    for s in specs:
        nx, ny = s["nx"], s["ny"]
        cells = nx * ny
        base = 28 if s["pol"] == "tm" else 32
        band = 2 * npml * ny * 2 + 2 * npml * nx * 2       # x bands x 2 psi + y bands x 2 psi
        total += base * cells + 8 * band
    return total


# ------------------------------------------------------------------ cfg1

def cfg1_spec():
    nx, ny = 320, 160
    eps = np.ones((nx, ny), dtype=np.float32)
    eps[:, 70:90] = 12.0
    return dict(nx=nx, ny=ny, eps=eps, src=(30, 80), flux=(290, 20, 140),
                freqs=tuple(np.linspace(0.1, 0.2, 50).tolist()), steps=4000)


def cfg1_item(device, spec=None, eps_t=None):
    from .core.coeffs import build_tm_coeffs
    from .core.grid import Grid
    from .core.monitors import FluxMonitorTM
    from .core.sources import GaussianPulse, LineSource
    from .core.stepper_tm import init_tm_state
    spec = spec or cfg1_spec()
    g = Grid(nx=spec["nx"], ny=spec["ny"], dx=DX2D, device=device)
    eps = eps_t if eps_t is not None else torch.from_numpy(spec["eps"]).to(device)
    m = build_tm_coeffs(g, eps_inf=eps, npml=NPML2D)
    i, j = spec["src"]
    src = LineSource(g, ix=i, j0=j, j1=j + 1, profile=GaussianPulse(0.15, 0.1))
    ix, lo, hi = spec["flux"]
    mon = FluxMonitorTM(g, list(spec["freqs"]), x_normal=True, idx=ix, lo=lo, hi=hi)
    return init_tm_state(g), m, src, [mon]


# ------------------------------------------------------------------ cfg3

def cfg3_eps(n: int = 256, seed: int = 3, dx: float = 1.0 / 16, n_spheres: int = 200):
    rng = np.random.default_rng(seed)
    eps = np.ones((n, n, n), dtype=np.float32)
    ax = (np.arange(n) + 0.5) * dx
    for _ in range(n_spheres):
        c = rng.uniform(1.0, 15.0, 3)
        r = rng.uniform(0.2, 0.6)
        e = rng.uniform(2.0, 12.0)
        lo = np.maximum(((c - r) / dx).astype(int) - 1, 0)
        hi = np.minimum(((c + r) / dx).astype(int) + 2, n)
        X = ax[lo[0]:hi[0], None, None]
        Y = ax[None, lo[1]:hi[1], None]
        Z = ax[None, None, lo[2]:hi[2]]
        inside = (X - c[0]) ** 2 + (Y - c[1]) ** 2 + (Z - c[2]) ** 2 <= r * r
        sub = eps[lo[0]:hi[0], lo[1]:hi[1], lo[2]:hi[2]]
        sub[inside] = e
    return eps


CFG3_FACES = (("x", 24), ("x", 232), ("y", 24), ("y", 232), ("z", 24), ("z", 232))


def cfg3_setup(device, n: int = 256, npml: int = 16, eps=None):
    from .core.monitors_3d import FluxMonitor3D, PointSource3D
    from .core.sources import GaussianPulse
    from .core.stepper_3d import build_3d_coeffs, init_3d_state
    dx = 1.0 / 16
    e = eps if eps is not None else torch.from_numpy(cfg3_eps(n)).to(device)
    c = build_3d_coeffs(n, n, n, dx, eps=e, npml=npml, device=device)
    s = init_3d_state(n, n, n, npml=npml, device=device)
    src = PointSource3D(c.dt, "Ez", n // 2, n // 2, n // 2, GaussianPulse(0.5, 0.3))
    freqs = np.linspace(0.35, 0.65, 20).tolist()
    lo_, hi_ = 24 * n // 256, 232 * n // 256
    mons = [FluxMonitor3D(c.dt, freqs, normal=a, idx=(lo_ if i == 24 else hi_),
                          win=(lo_, hi_, lo_, hi_)) for a, i in CFG3_FACES]
    return s, c, src, mons


def cfg3_bytes_per_step(n: int = 256, npml: int = 16) -> float:
    """64 B per cell-step: 6 fields read+write (48 B), cell-centred eps (4 B)
    and the CPML memory (12 psi arrays, each read+written inside its layer:
    3 axes x 4 psi x 8 B x (2 npml / n))."""
    cells = n ** 3
    return cells * (48 + 4) + 3 * 4 * 8 * cells * (2 * npml / n)


# ------------------------------------------------------------------ cfg4

CFG4 = dict(nx=600, ny=400, dx=0.04, npml=25, eps_bg=2.1, eps_core=12.0, guide_w=20,
            design=160, steps=8000, radius=0.15, beta=8.0, eta=0.5,
            freqs=(1 / 1.60, 1 / 1.55, 1 / 1.50))


def cfg4_setup(device, seed: int = 4, steps: int = None):
    """cfg4-shaped gradient problem: 600 x 400 TM grid at res 25, 25-cell CPML,
    eps 2.1 background with an eps 12, 0.8 um wide input and output guide along x
    meeting a centred 160 x 160 design region (rho0 ~ U(0.4, 0.6), default_rng(4)),
    conic filter 0.15 um, tanh projection beta 8 / eta 0.5. A Gaussian line source
    across the input guide (fcen 0.645, fwidth 0.12: the 1.50-1.60 um band) stands in
    for the reference's mode source, and the objective is the mean transmitted flux
    through the output guide at the three wavelengths. Returns the
    OptimizationProblem (design.py) and the step count."""
    from .core.coeffs import build_tm_coeffs
    from .core.grid import Grid
    from .core.monitors import FluxMonitorTM
    from .core.run import run_tm
    from .core.sources import GaussianPulse, LineSource
    from .core.stepper_tm import init_tm_state
    from .design import DesignRegion, MaterialGrid, OptimizationProblem
    c = CFG4
    nx, ny, dx, npml = c["nx"], c["ny"], c["dx"], c["npml"]
    n = steps or c["steps"]
    rng = np.random.default_rng(seed)
    base = torch.full((nx, ny), c["eps_bg"], dtype=torch.float32)
    y0, y1 = ny // 2 - c["guide_w"] // 2, ny // 2 + c["guide_w"] // 2
    base[:, y0:y1] = c["eps_core"]
    d = c["design"]
    ix0, iy0 = nx // 2 - d // 2, ny // 2 - d // 2
    reg = DesignRegion(MaterialGrid((d, d), c["eps_bg"], c["eps_core"]), ix0=ix0, ix1=ix0 + d,
                       iy0=iy0, iy1=iy0 + d)
    grid = Grid(nx=nx, ny=ny, dx=dx, device=device)
    src = LineSource(grid, ix=npml + 10, j0=y0 - 10, j1=y1 + 10,
                     profile=GaussianPulse(0.645, 0.12))
    mon = FluxMonitorTM(grid, list(c["freqs"]), x_normal=True, idx=nx - npml - 10,
                        lo=y0 - 20, hi=y1 + 20)

    def run_fn(eps):
        m = build_tm_coeffs(grid, eps_inf=eps, npml=npml)
        _, (acc,) = run_tm(init_tm_state(grid), m, n, source=src, monitors=[mon],
                           checkpoint_every=256)
        return mon.flux(acc, dx).mean()

    rho0 = torch.tensor(rng.uniform(0.4, 0.6, (d, d)), dtype=torch.float32, device=device)
    opt = OptimizationProblem(run_fn, base.to(device), reg, filter_radius=c["radius"], dx=dx,
                              beta=c["beta"], eta=c["eta"], rho0=rho0)
    return opt, n
