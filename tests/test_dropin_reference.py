"""The drop-in through the reference's own public API, on the GPU.

With ``install("meep_torch")`` active, the reference's entry points route float32 CUDA
runs to this package's kernels. These tests build everything with the reference's own
objects (``mp.Simulation``; ``build_tm_coeffs``, ``Port``, ``ModeSourceTM``,
``FluxMonitorTM``, ``run_tm`` and ``decompose``) and compare the CUDA run against the
same calls on the CPU, where the reference's own torch code runs. The reference is found
through ``tests/golden/reference_path.py`` (MEEP_TORCH_REF or the reference arm's install
beside the repository); without it the tests skip.

Bar: relative L2 < 1e-4 (the parity tolerance) on fluxes, fields and mode amplitudes; the
design gradient through ModeSourceTM / decompose, accumulated over the reverse sweep in
float32 on both sides, is held to 1e-3.
"""
import importlib
import sys
import time

import numpy as np
import pytest
import torch

from tests.conftest import rel_l2
from tests.golden.reference_path import find_reference

pytestmark = pytest.mark.gpu
TOL = 1e-4


@pytest.fixture(scope="module")
def ref():
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    path = find_reference()
    if path is None:
        pytest.skip("reference not installed")
    if path not in sys.path:
        sys.path.insert(0, path)
    mt = importlib.import_module("meep_torch")
    for m in ("meep_torch.core.run", "meep_torch.core.monitors_3d", "meep_torch.solvers",
              "meep_torch.mp.cpp.core", "meep_torch.mp.simulation",
              "meep_torch.core.stepper_3d_lean", "meep_torch.core.adjoint3d",
              "meep_torch.ports.smatrix"):
        importlib.import_module(m)
    from meep_torch_b200 import build
    from meep_torch_b200.install import install, uninstall
    build.build()
    install("meep_torch")
    try:
        yield mt
    finally:
        uninstall()


def _launches():
    from meep_torch_b200 import _lib
    return _lib.load().mtb_launch_count()


def test_simulation_run_on_the_kernels_matches_the_reference_on_cpu(ref):
    """cfg1 through mp.Simulation.run (mp/simulation.py:1096 -> fields.step_n,
    mp/cpp/core.py:802 -> core.run._run_chunk): 320 x 160, eps 12 guide, Gaussian Ez
    point source, 50-frequency flux line, run(until=100) = 4000 steps."""
    mp = importlib.import_module("meep_torch.mp")

    def run(device):
        sim = mp.Simulation(
            cell_size=mp.Vector3(16, 8), resolution=20,
            geometry=[mp.Block(size=mp.Vector3(mp.inf, 1, mp.inf),
                               material=mp.Medium(epsilon=12))],
            sources=[mp.Source(mp.GaussianSource(0.15, fwidth=0.1), component=mp.Ez,
                               center=mp.Vector3(-6.5, 0))],
            boundary_layers=[mp.PML(1.0)], dtype=torch.float32, device=device)
        fl = sim.add_flux(0.15, 0.1, 50, mp.FluxRegion(center=mp.Vector3(6.5, 0),
                                                        size=mp.Vector3(0, 6)))
        n0 = _launches()
        sim.run(until=100)
        launched = _launches() - n0
        flux = np.asarray(mp.get_fluxes(fl), dtype=np.float64)
        ez = sim.get_array(component=mp.Ez)
        ez = ez.detach().cpu().double().numpy() if torch.is_tensor(ez) else np.asarray(ez)
        return flux, ez, launched

    f_cpu, ez_cpu, n_cpu = run("cpu")
    f_gpu, ez_gpu, n_gpu = run("cuda")
    assert n_cpu == 0 and n_gpu > 0, (n_cpu, n_gpu)      # the kernels ran the CUDA run
    e = {"flux": rel_l2(f_gpu, f_cpu), "Ez": rel_l2(ez_gpu, ez_cpu)}
    print(f"\n[Simulation cfg1] relL2 vs the reference on CPU: {e}; {n_gpu} library launches")
    assert max(e.values()) < TOL, e


def _mode_problem(device, dtype, eps_design=None):
    """A small two-mode converter on the reference's own objects: guide in, a design
    block, guide out; TE0-like input mode from ModeSourceTM, output decomposed into two
    modes (ports/mode_source.py:21, ports/mode_monitor.py:28)."""
    from meep_torch.core.coeffs import build_tm_coeffs
    from meep_torch.core.grid import Grid
    from meep_torch.core.monitors import FluxMonitorTM
    from meep_torch.core.run import run_tm
    from meep_torch.core.sources import GaussianPulse
    from meep_torch.core.stepper_tm import init_tm_state
    from meep_torch.ports.mode_monitor import decompose
    from meep_torch.ports.mode_source import ModeSourceTM
    from meep_torch.ports.port import Port
    nx, ny, dx, npml, n = 220, 120, 0.04, 20, 1800
    g = Grid(nx=nx, ny=ny, dx=dx, dtype=dtype, device=device)
    eps = torch.full((nx, ny), 2.1, dtype=dtype)
    eps[:, ny // 2 - 10:ny // 2 + 10] = 12.0
    rng = np.random.default_rng(8)
    design = torch.tensor(rng.uniform(2.1, 12.0, (40, 40)), dtype=dtype)
    if eps_design is not None:
        design = eps_design
    eps = eps.clone()
    eps[nx // 2 - 20:nx // 2 + 20, ny // 2 - 20:ny // 2 + 20] = design
    eps = eps.to(device)
    c = build_tm_coeffs(g, eps_inf=eps, npml=npml)
    freqs = [1 / 1.60, 1 / 1.55, 1 / 1.50]
    p_in = Port("x", npml + 12, ny // 2 - 30, ny // 2 + 30, +1)
    src = ModeSourceTM(g, c, p_in, GaussianPulse(0.645, 0.12), 0.645, mode=0)
    io = nx - npml - 12
    mon = FluxMonitorTM(g, freqs, x_normal=True, idx=io, lo=ny // 2 - 30, hi=ny // 2 + 30)
    _, (acc,) = run_tm(init_tm_state(g), c, n, source=src, monitors=[mon],
                       checkpoint_every=256)
    a_p, a_m = decompose(acc, c.eps_inf[io, ny // 2 - 30:ny // 2 + 30], dx, freqs, "tm",
                         n_modes=2)
    return acc, a_p, a_m, design


def test_mode_source_and_decompose_on_the_kernels(ref):
    """ModeSourceTM's J and M sheets (mask and h_masks) drive the kernels; the output
    monitor's accumulators and the reference's decompose() of them match the CPU run."""
    n0 = _launches()
    with torch.no_grad():
        acc_g, ap_g, am_g, _ = _mode_problem("cuda", torch.float32)
    assert _launches() > n0
    with torch.no_grad():
        acc_c, ap_c, am_c, _ = _mode_problem("cpu", torch.float32)
    e = {"acc": rel_l2(acc_g.cpu().numpy(), acc_c.numpy()),
         "a_plus": rel_l2(ap_g.cpu().numpy(), ap_c.numpy()),
         "a_minus": rel_l2(am_g.cpu().numpy(), am_c.numpy())}
    print(f"\n[ModeSourceTM + decompose] relL2 vs the reference on CPU: {e}")
    assert max(e.values()) < TOL, e


def test_mode_converter_gradient_on_the_kernels(ref):
    """d J / d eps_design of J = mean_f |a+_1|^2 (TE0 -> TE1 power) through ModeSourceTM,
    run_tm(checkpoint_every=256) and decompose: this package's adjoint kernels on the
    GPU against the reference's autograd on the CPU."""
    def grad(device):
        d0 = torch.tensor(np.random.default_rng(8).uniform(2.1, 12.0, (40, 40)),
                          dtype=torch.float32, requires_grad=True)
        _, a_p, _, _ = _mode_problem(device, torch.float32, eps_design=d0)
        J = (a_p[:, 1].abs() ** 2).mean()
        J.backward()
        return float(J), d0.grad.double().numpy()

    n0 = _launches()
    Jg, gg = grad("cuda")
    assert _launches() > n0
    Jc, gc = grad("cpu")
    eJ, eg = abs(Jg - Jc) / abs(Jc), rel_l2(gg, gc)
    print(f"\n[mode converter gradient] J rel err {eJ:.2e}, dJ/deps relL2 {eg:.2e}")
    assert eJ < TOL and eg < 1e-3, (eJ, eg)


def test_simulation_solve_cw_on_the_kernels_matches_the_reference(ref):
    """mp.Simulation(force_complex_fields=True).solve_cw (mp/simulation.py:2290 ->
    fields.solve_cw, mp/cpp/core.py:721) routed to the kernels' CW solve: an 80 x 80 cell
    with an eps 12 guide and a ContinuousSource(0.15) Ez point source, PML 1. The CUDA
    float32 solve (tol 1e-5) against the reference's own float64 solve on the CPU
    (tol 1e-8): the complex Ez map."""
    mp = importlib.import_module("meep_torch.mp")

    def solve(device, dtype, tol):
        sim = mp.Simulation(
            resolution=10, cell_size=mp.Vector3(8, 8),
            geometry=[mp.Block(size=mp.Vector3(mp.inf, 1, mp.inf),
                               material=mp.Medium(epsilon=12))],
            sources=[mp.Source(mp.ContinuousSource(0.15), component=mp.Ez,
                               center=mp.Vector3(-2, 0))],
            boundary_layers=[mp.PML(1.0)], force_complex_fields=True, dtype=dtype,
            device=device)
        sim.init_sim()
        n0 = _launches()
        t0 = time.perf_counter()
        ok = sim.solve_cw(tol, 10000, 2)
        if device == "cuda":
            torch.cuda.synchronize()
        times[device] = time.perf_counter() - t0
        launched = _launches() - n0
        ez = sim.get_array(component=mp.Ez)
        ez = ez.detach().cpu().numpy() if torch.is_tensor(ez) else np.asarray(ez)
        return ok, np.asarray(ez, dtype=np.complex128), launched

    times = {}
    ok_c, ez_c, n_c = solve("cpu", torch.float64, 1e-8)
    ok_g, ez_g, n_g = solve("cuda", torch.float32, 1e-5)
    assert ok_g and n_c == 0 and n_g > 0, (ok_c, ok_g, n_c, n_g)
    e = float(np.linalg.norm(ez_g - ez_c) / np.linalg.norm(ez_c))
    print(f"\n[Simulation solve_cw] Ez relL2 vs the reference (CPU, float64; converged "
          f"{ok_c}): {e:.2e}; {n_g} library launches; solve {times['cuda']:.3f} s on the "
          f"kernels, {times['cpu']:.3f} s for the reference on the CPU")
    assert e < 1e-3, e
