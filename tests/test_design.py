"""The design chain (meep_torch_b200.design) against the reference's own outputs
(tests/golden/golden_design.npz: adjoint/filters.py, adjoint/problem.py run in float64)."""
import numpy as np
import pytest
import torch

from tests.conftest import load_golden, rel_l2


def test_filter_projection_paint_match_reference():
    from meep_torch_b200.design import DesignRegion, MaterialGrid, conic_filter, tanh_projection
    g = load_golden("design")
    r = torch.tensor(g["rho"], dtype=torch.float64)
    filt = conic_filter(r, 0.15, 0.04)
    proj = tanh_projection(filt, 8.0, 0.5)
    assert np.allclose(filt.numpy(), g["filt"], rtol=0, atol=1e-14)
    assert np.allclose(proj.numpy(), g["proj"], rtol=0, atol=1e-13)
    ix0, ix1, iy0, iy1 = (int(v) for v in g["box"])
    reg = DesignRegion(MaterialGrid(g["rho"].shape, 2.1, 12.0), ix0=ix0, ix1=ix1, iy0=iy0,
                       iy1=iy1)
    painted = reg.paint(torch.tensor(g["base"]), proj)
    assert np.allclose(painted.numpy(), g["painted"], rtol=0, atol=1e-12)


def test_filter_keeps_constants_and_projection_limits():
    from meep_torch_b200.design import conic_filter, tanh_projection
    c = torch.full((13, 9), 0.37, dtype=torch.float64)
    assert torch.allclose(conic_filter(c, 0.3, 0.05), c, atol=1e-15)
    x = torch.tensor([0.0, 0.5, 1.0], dtype=torch.float64)
    y = tanh_projection(x, 30.0, 0.5)
    assert abs(float(y[0])) < 1e-12 and abs(float(y[2]) - 1) < 1e-12 and abs(float(y[1]) - 0.5) < 1e-12


@pytest.mark.gpu
def test_optimization_problem_gradient_matches_reference():
    """OptimizationProblem with a TM run_fn on the B200 kernels: J and dJ/drho against
    the reference's float64 autograd (golden_design.npz)."""
    from meep_torch_b200.core.coeffs import build_tm_coeffs
    from meep_torch_b200.core.grid import Grid
    from meep_torch_b200.core.monitors import FluxMonitorTM
    from meep_torch_b200.core.run import run_tm
    from meep_torch_b200.core.sources import GaussianPulse, LineSource
    from meep_torch_b200.core.stepper_tm import init_tm_state
    from meep_torch_b200.design import DesignRegion, MaterialGrid, OptimizationProblem
    g = load_golden("design")
    nx, ny, dx, npml = 48, 36, 0.05, 8
    grid = Grid(nx=nx, ny=ny, dx=dx, device="cuda")
    src = LineSource(grid, ix=12, j0=12, j1=24, profile=GaussianPulse(0.65, 0.4))
    mon = FluxMonitorTM(grid, [0.6, 0.7], x_normal=True, idx=38, lo=9, hi=27)

    def run_fn(eps):
        m = build_tm_coeffs(grid, eps_inf=eps, npml=npml)
        _, (acc,) = run_tm(init_tm_state(grid), m, 200, source=src, monitors=[mon],
                           checkpoint_every=50)
        return mon.flux(acc, dx).mean() * 1e9

    ix0, ix1, iy0, iy1 = (int(v) for v in g["box"])
    reg = DesignRegion(MaterialGrid((20, 16), 2.1, 12.0), ix0=ix0, ix1=ix1, iy0=iy0, iy1=iy1)
    base = torch.tensor(g["base"], dtype=torch.float32, device="cuda")
    rho0 = torch.tensor(g["rho0"], dtype=torch.float32, device="cuda")
    opt = OptimizationProblem(run_fn, base, reg, filter_radius=0.1, dx=dx, beta=4.0, eta=0.5,
                              rho0=rho0)
    f0, grad = opt()
    e = rel_l2(grad, g["grad"])
    print(f"design gradient rel L2 vs reference float64: {e:.3e}; J {f0:.8e} vs "
          f"{float(g['f0']):.8e}")
    assert abs(f0 - float(g["f0"])) <= 1e-4 * abs(float(g["f0"]))
    assert e < 1e-4
