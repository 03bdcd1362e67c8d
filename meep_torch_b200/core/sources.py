"""Soft-source time profiles and spatial masks (reference: core/sources.py:26-159).

Host-side: profiles are evaluated in FP64 per step, masks are built once;
the kernels read the mask's nonzero cells and a per-step coefficient table.
"""
import math

import torch

from .grid import Grid


class GaussianPulse:
    """cos(2 pi f (t - t0)) exp(-(t - t0)^2 / (2 w^2)), w = 1/fwidth, t0 = cutoff*w."""

    def __init__(self, fcen: float, fwidth: float, cutoff: float = 5.0):
        self.fcen = fcen
        self.w = 1.0 / fwidth
        self.t0 = cutoff * self.w
        self.t_end = 2.0 * self.t0

    def amplitude(self, t: float) -> float:
        return math.cos(2 * math.pi * self.fcen * (t - self.t0)) * math.exp(
            -((t - self.t0) ** 2) / (2 * self.w ** 2))


class CWRamp:
    """sin(2 pi f t) with a linear turn-on over t_ramp."""

    def __init__(self, fcen: float, t_ramp: float):
        self.fcen = fcen
        self.t_ramp = t_ramp

    def amplitude(self, t: float) -> float:
        return math.sin(2 * math.pi * self.fcen * t) * min(1.0, t / self.t_ramp)


class ContinuousSource:
    """sin(2 pi f t) with a raised-cosine turn-on of slowness*width."""

    def __init__(self, frequency: float, width: float | None = None, slowness: float = 3.0,
                 cutoff: float = 5.0, fcen: float | None = None):
        self.fcen = float(fcen if fcen is not None else frequency)
        self.t_ramp = (slowness * width) if width is not None else max(1.0, slowness / self.fcen)
        self.cutoff = cutoff

    def amplitude(self, t: float) -> float:
        ramp = 1.0 if self.t_ramp <= 0 else 0.5 - 0.5 * math.cos(
            math.pi * min(1.0, t / self.t_ramp))
        return math.sin(2 * math.pi * self.fcen * t) * ramp


class CustomSource:
    """User profile; complex values contribute their real part."""

    def __init__(self, fn):
        self.fn = fn

    def amplitude(self, t: float) -> float:
        v = self.fn(t)
        return float(v.real) if isinstance(v, complex) else float(v)


class LineSource:
    """Soft current on x = ix, y in [j0, j1): mask 1/dx per cell for a line,
    1/dx^2 for a single cell (the source measure over the cell area)."""

    def __init__(self, grid: Grid, ix: int, j0: int, j1: int, profile, amp_func=None, amps=None):
        if not 0 <= ix < grid.nx:
            raise ValueError(f"source ix={ix} outside grid nx={grid.nx}")
        if not 0 <= j0 < j1 <= grid.ny:
            raise ValueError(f"source segment j0={j0}, j1={j1} invalid for ny={grid.ny}")
        self.profile = profile
        self.dt = grid.dt
        mask = grid.zeros(grid.nx, grid.ny)
        if amps is not None:
            mask[ix, j0:j1] = torch.as_tensor(amps, dtype=grid.dtype, device=grid.device)
        elif amp_func is None:
            mask[ix, j0:j1] = 1.0
        else:
            for j in range(j0, j1):
                mask[ix, j] = float(amp_func((j + 0.5) * grid.dx))
        per_cell = grid.dx if (j1 - j0) > 1 else 1.0
        self.mask = mask * (per_cell / grid.dx ** 2)

    def amplitude(self, t_idx: int) -> float:
        return self.profile.amplitude((t_idx + 0.5) * self.dt)


class SoftSource:
    """Jz(x, y, t) = profile(t) * mask(x, y) for an arbitrary (nx, ny) mask."""

    def __init__(self, grid: Grid, mask, profile):
        self.mask = mask
        self.profile = profile
        self.dt = grid.dt

    def amplitude(self, t_idx: int) -> float:
        return self.profile.amplitude((t_idx + 0.5) * self.dt)


class TESource:
    """A 2D source bound to a TE run: the Dy mask is the (nx, ny) mask minus
    its last column (the reference Simulation's TE binding,
    mp/simulation.py:867-869)."""

    def __init__(self, source):
        self.source = source
        self.mask = source.mask[:, :-1]
        self.profile = getattr(source, "profile", None)
        self.dt = getattr(source, "dt", None)

    def amplitude(self, t_idx: int) -> float:
        return self.source.amplitude(t_idx)
