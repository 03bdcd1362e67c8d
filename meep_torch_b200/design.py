"""Design chain in front of the differentiable TM run (reference: adjoint/filters.py,
adjoint/problem.py): design density rho -> conic blur -> tanh projection -> eps between
two materials -> bilinear paint into a base eps map -> run_fn(eps) -> objective J, with
dJ/drho by reverse mode. The chain is a few small torch operations; the FDTD inside
run_fn (``core.run.run_tm`` with eps requiring grad) is where the time goes, and its
gradient comes from the library's adjoint kernels.

Same names, arguments and conventions as the reference, so an optimisation script runs
unchanged against either.
"""
from __future__ import annotations

import math

import torch
import torch.nn.functional as F


def _cone(radius: float, dx: float, dtype, device) -> torch.Tensor:
    """Cone weights max(0, 1 - r / radius) on the (2n+1)^2 grid of offsets, n = ceil(radius/dx)."""
    n = max(1, int(math.ceil(radius / dx)))
    off = torch.arange(-n, n + 1, dtype=dtype, device=device) * dx
    r = torch.sqrt(off[:, None] ** 2 + off[None, :] ** 2)
    return (1.0 - r / radius).clamp_min(0.0)


def conic_filter(rho: torch.Tensor, radius: float, dx: float) -> torch.Tensor:
    """Conic blur of physical radius ``radius`` (adjoint/filters.py:27-33): each cell is the
    cone-weighted mean of its in-bounds neighbours, so a constant density is unchanged up to
    the edges."""
    w = _cone(radius, dx, rho.dtype, rho.device)
    half = (w.shape[0] // 2, w.shape[1] // 2)
    x = rho.reshape(1, 1, *rho.shape)
    weighted = F.conv2d(x, w.reshape(1, 1, *w.shape), padding=half)
    mass = F.conv2d(torch.ones_like(x), w.reshape(1, 1, *w.shape), padding=half)
    return (weighted / mass).reshape(rho.shape)


def tanh_projection(rho: torch.Tensor, beta: float, eta: float = 0.5) -> torch.Tensor:
    """Smoothed threshold at eta with sharpness beta (adjoint/filters.py:45-52):
    (tanh(beta eta) + tanh(beta (rho - eta))) / (tanh(beta eta) + tanh(beta (1 - eta)))."""
    t0 = math.tanh(beta * eta)
    return (t0 + torch.tanh(beta * (rho - eta))) / (t0 + math.tanh(beta * (1.0 - eta)))


class MaterialGrid:
    """Design density grid: rho in [0, 1] maps linearly onto [eps_min, eps_max]
    (adjoint/problem.py:19-29)."""

    def __init__(self, shape, eps_min: float = 1.0, eps_max: float = 12.0):
        self.shape = tuple(shape)
        self.eps_min, self.eps_max = float(eps_min), float(eps_max)

    def eps(self, rho_projected: torch.Tensor) -> torch.Tensor:
        return self.eps_min + (self.eps_max - self.eps_min) * rho_projected


class DesignRegion:
    """An index box [ix0, ix1) x [iy0, iy1) of the eps map painted from a MaterialGrid by
    bilinear upsampling, cell centres aligned (adjoint/problem.py:46-59)."""

    def __init__(self, material_grid: MaterialGrid, *, ix0, ix1, iy0, iy1):
        self.mg = material_grid
        self.box = (ix0, ix1, iy0, iy1)

    def paint(self, base_eps: torch.Tensor, rho_projected: torch.Tensor) -> torch.Tensor:
        ix0, ix1, iy0, iy1 = self.box
        up = F.interpolate(rho_projected.reshape(1, 1, *rho_projected.shape),
                           size=(ix1 - ix0, iy1 - iy0), mode="bilinear",
                           align_corners=False).reshape(ix1 - ix0, iy1 - iy0)
        out = base_eps.clone()
        out[ix0:ix1, iy0:iy1] = self.mg.eps(up)
        return out


class OptimizationProblem:
    """``opt()`` -> (J, dJ/drho) for the density ``opt.rho`` (adjoint/problem.py:62-110).
    ``beta`` / ``eta`` default to the grid's own values when it carries them, else 1 / 0.5."""

    def __init__(self, run_fn, base_eps: torch.Tensor, design_region: DesignRegion, *,
                 filter_radius: float = 0.0, dx: float = 1.0, beta: float = None,
                 eta: float = None, rho0=None):
        self.run_fn, self.base_eps, self.region = run_fn, base_eps, design_region
        self.filter_radius, self.dx = filter_radius, dx
        mg = design_region.mg
        self.beta = beta if beta is not None else (getattr(mg, "beta", 0) or 1.0)
        self.eta = eta if eta is not None else (getattr(mg, "eta", None) or 0.5)
        self.rho = (rho0.clone() if rho0 is not None
                    else torch.full(mg.shape, 0.5, dtype=base_eps.dtype))

    def _objective(self, rho: torch.Tensor):
        r = conic_filter(rho, self.filter_radius, self.dx) if self.filter_radius > 0 else rho
        r = tanh_projection(r, self.beta, self.eta)
        return self.run_fn(self.region.paint(self.base_eps, r))

    def __call__(self, need_gradient: bool = True):
        rho = self.rho.detach().clone().requires_grad_(need_gradient)
        J = self._objective(rho)
        if not need_gradient:
            return float(J), None
        J.backward()
        return float(J.detach()), rho.grad.detach().cpu().numpy().copy()

    def eval_at_delta(self, i: int, j: int, h: float) -> float:
        """Objective with rho[i, j] perturbed by h (finite-difference checks)."""
        rho = self.rho.detach().clone()
        rho[i, j] += h
        with torch.no_grad():
            return float(self._objective(rho))
