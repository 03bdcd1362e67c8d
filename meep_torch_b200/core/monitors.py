"""2D point probes, DFT and flux monitors (reference: core/monitors.py:11-155).

On the B200 path the monitors are descriptors: the kernels sample the
fields into a ring and a contraction kernel folds dt*[cos(wt) F, -sin(wt) F]
into accumulators of the reference's shapes -- (nfreq, 2, *comp_shape) for
DFTFieldsMonitor and (nfreq, 4, L) for the flux lines. ``flux`` reduces an
accumulator exactly as the reference does.
"""
from typing import Sequence

import torch

from .grid import Grid


class PointProbe:
    """Ez at node (ix, iy) after every step; a run returns the k values of its steps as
    one (k,) tensor (stack-reduced; reference interface core/monitors.py:11-21). The
    kernels copy the node into the sample ring each step and the engine gathers the
    ring after every flush."""
    reduce = "stack"

    def __init__(self, ix: int, iy: int):
        self.ix, self.iy = int(ix), int(iy)


class DFTFieldsMonitor:
    """Full-grid running DFT of one component. Time of a sample: (t+1)dt for
    E components, (t+1/2)dt for H components (the reference's convention)."""
    reduce = "sum"

    def __init__(self, grid: Grid, freqs: Sequence[float], component: str = "Ez"):
        self.component = component
        self.dt = grid.dt
        self.freqs = torch.tensor(freqs, dtype=grid.dtype, device=grid.device)


class FluxMonitorTM:
    """Ez and the 2-point-averaged Hy (x-normal) / Hx (y-normal) on a line;
    flux = -1/2 sum(ReE ReH + ImE ImH) dx for x-normal, +1/2 for y-normal."""
    reduce = "sum"

    def __init__(self, grid: Grid, freqs: Sequence[float], *, x_normal: bool, idx: int,
                 lo: int, hi: int):
        self.x_normal = x_normal
        self.idx, self.lo, self.hi = idx, lo, hi
        self.dt = grid.dt
        self.freqs = torch.tensor(freqs, dtype=grid.dtype, device=grid.device)
        if x_normal and not (1 <= idx < grid.nx - 1):
            raise ValueError(f"x-normal monitor ix={idx} must be interior")
        if not x_normal and not (1 <= idx < grid.ny - 1):
            raise ValueError(f"y-normal monitor iy={idx} must be interior")

    def flux(self, acc: torch.Tensor, dx: float) -> torch.Tensor:
        ReE, ImE, ReH, ImH = acc.unbind(1)
        s = (ReE * ReH + ImE * ImH).sum(-1) * dx
        return -0.5 * s if self.x_normal else 0.5 * s


class FluxMonitorTE:
    """x-normal TE line: Ey and Hz averaged across x; E at (t+1/2)dt, Hz at (t+1)dt."""
    reduce = "sum"

    def __init__(self, grid: Grid, freqs, *, ix: int, lo: int, hi: int):
        if not (1 <= ix < grid.nx - 1):
            raise ValueError(f"ix={ix} must be interior")
        self.ix, self.lo, self.hi = ix, lo, hi
        self.dt = grid.dt
        self.freqs = torch.tensor(freqs, dtype=grid.dtype, device=grid.device)

    def flux(self, acc: torch.Tensor, dx: float) -> torch.Tensor:
        ReE, ImE, ReH, ImH = acc.unbind(1)
        return 0.5 * (ReE * ReH + ImE * ImH).sum(-1) * dx


class FluxMonitorTEY:
    """y-normal TE line: Ex and Hz averaged across y."""
    reduce = "sum"

    def __init__(self, grid: Grid, freqs, *, iy: int, lo: int, hi: int):
        if not (1 <= iy < grid.ny - 1):
            raise ValueError(f"iy={iy} must be interior")
        self.iy, self.lo, self.hi = iy, lo, hi
        self.dt = grid.dt
        self.freqs = torch.tensor(freqs, dtype=grid.dtype, device=grid.device)

    def flux(self, acc: torch.Tensor, dx: float) -> torch.Tensor:
        ReE, ImE, ReH, ImH = acc.unbind(1)
        return -0.5 * (ReE * ReH + ImE * ImH).sum(-1) * dx
