"""Soft sources for the B200 engines (reference interface: core/sources.py:26-159).

The engines read four things from a source: ``amplitude(t_idx)`` -- the time profile at
the half step (t_idx + 1/2) dt --, ``mask`` -- a weight per grid node, whose nonzero
cells become the kernels' sparse cell list --, and ``profile`` / ``dt``, which let them
tabulate the amplitudes of a whole run at once. The reference's own source objects have
the same members and can be handed to the engines directly; the classes below serve
callers without the reference. The time profiles are the published ones the reference
uses (a Gaussian-modulated cosine, and sinusoids switched on by a linear or a
raised-cosine ramp); amplitudes are evaluated in float64 on the host.
"""
import math

import torch

TWO_PI = 2.0 * math.pi


class _Profile:
    """A scalar time profile f(t); ``amplitude`` is its float value."""

    def value(self, t: float) -> float:
        raise NotImplementedError

    def amplitude(self, t: float) -> float:
        return float(self.value(t))


class GaussianPulse(_Profile):
    """Gaussian-enveloped carrier at fcen: width w = 1 / fwidth, centred t0 = cutoff w
    after the start, negligible after t_end = 2 t0."""

    def __init__(self, fcen: float, fwidth: float, cutoff: float = 5.0):
        self.fcen = fcen
        self.w = 1.0 / fwidth
        self.t0 = cutoff * self.w
        self.t_end = 2.0 * self.t0

    def value(self, t: float) -> float:
        s = t - self.t0
        envelope = math.exp(-(s * s) / (2.0 * self.w * self.w))
        return math.cos(TWO_PI * self.fcen * s) * envelope


class CWRamp(_Profile):
    """A sine at fcen whose amplitude rises linearly to 1 over t_ramp."""

    def __init__(self, fcen: float, t_ramp: float):
        self.fcen = fcen
        self.t_ramp = t_ramp

    def value(self, t: float) -> float:
        return math.sin(TWO_PI * self.fcen * t) * min(1.0, t / self.t_ramp)


class ContinuousSource(_Profile):
    """A sine at the frequency, switched on by a raised cosine over t_ramp =
    slowness * width (or max(1, slowness / f) without a width)."""

    def __init__(self, frequency: float, width: float | None = None, slowness: float = 3.0,
                 cutoff: float = 5.0, fcen: float | None = None):
        self.fcen = float(frequency if fcen is None else fcen)
        self.t_ramp = slowness * width if width is not None else max(1.0, slowness / self.fcen)
        self.cutoff = cutoff

    def value(self, t: float) -> float:
        if self.t_ramp > 0:
            on = 0.5 * (1.0 - math.cos(math.pi * min(1.0, t / self.t_ramp)))
        else:
            on = 1.0
        return math.sin(TWO_PI * self.fcen * t) * on


class CustomSource(_Profile):
    """A user function of time; complex values drive the field with their real part."""

    def __init__(self, fn):
        self.fn = fn

    def value(self, t: float) -> float:
        v = self.fn(t)
        return v.real if isinstance(v, complex) else v


class _Sampled:
    """Shared by the spatial sources: the profile sampled at half steps."""

    def amplitude(self, t_idx: int) -> float:
        return self.profile.amplitude((t_idx + 0.5) * self.dt)


class LineSource(_Sampled):
    """A soft current on the node column x = ix, y in [j0, j1). The weights (1, or
    ``amps``, or ``amp_func`` of the cell-centre y) are scaled to a density: by 1 / dx
    along a segment of several cells, by 1 / dx^2 for a single cell."""

    def __init__(self, grid, ix: int, j0: int, j1: int, profile, amp_func=None, amps=None):
        if ix < 0 or ix >= grid.nx or j0 < 0 or j1 > grid.ny or j0 >= j1:
            raise ValueError(f"LineSource: column ix={ix}, rows [{j0}, {j1}) do not fit a "
                             f"{grid.nx} x {grid.ny} grid")
        count = j1 - j0
        if amps is not None:
            weights = torch.as_tensor(amps, dtype=grid.dtype, device=grid.device)
        elif amp_func is not None:
            weights = torch.tensor([float(amp_func((j + 0.5) * grid.dx)) for j in range(j0, j1)],
                                   dtype=grid.dtype, device=grid.device)
        else:
            weights = torch.ones(count, dtype=grid.dtype, device=grid.device)
        density = 1.0 / grid.dx if count > 1 else 1.0 / (grid.dx * grid.dx)
        self.mask = grid.zeros(grid.nx, grid.ny)
        self.mask[ix, j0:j1] = weights * density
        self.profile = profile
        self.dt = grid.dt


class SoftSource(_Sampled):
    """A soft current with an arbitrary (nx, ny) weight map."""

    def __init__(self, grid, mask, profile):
        self.mask = mask
        self.profile = profile
        self.dt = grid.dt


class TESource:
    """A 2D source bound to a TE run, which drives Dy: its mask is the source's
    (nx, ny) mask without the last column (the reference Simulation's TE binding,
    mp/simulation.py:867-869)."""

    def __init__(self, source):
        self.source = source
        self.mask = source.mask[:, :-1]
        self.profile = getattr(source, "profile", None)
        self.dt = getattr(source, "dt", None)

    def amplitude(self, t_idx: int) -> float:
        return self.source.amplitude(t_idx)
