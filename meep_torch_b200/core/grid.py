"""The 2D grid descriptor the B200 engines read (reference interface: core/grid.py:33-59).

The engines take only ``nx``, ``ny``, ``dx``, ``dt``, ``dtype`` and ``device`` from a grid,
so the reference's own ``Grid`` objects work unchanged; this class is for callers without
the reference. Time step and stability rule are the reference's: ``dt = courant * dx``
with ``0 < courant <= 1/sqrt(2)`` for the 2D Yee scheme.
"""
import os

import torch

_COURANT_2D_MAX = 0.5 ** 0.5


def default_device() -> str:
    """Device for new grids: ``MEEP_TORCH_DEVICE`` if set, else ``cuda`` (this package
    computes on the GPU only)."""
    return os.environ.get("MEEP_TORCH_DEVICE") or "cuda"


class Grid:
    """nx x ny Yee nodes at spacing dx. Defaults to float32, the precision of the
    kernels (the reference's grid defaults to float64)."""

    __slots__ = ("nx", "ny", "dx", "courant", "dtype", "device")

    def __init__(self, nx: int, ny: int, dx: float, courant: float = 0.5,
                 dtype: torch.dtype = torch.float32, device=None):
        problems = [what for what, ok in (("nx >= 3", nx >= 3), ("ny >= 3", ny >= 3),
                                          ("dx > 0", dx > 0),
                                          ("0 < courant <= 1/sqrt(2)",
                                           0 < courant <= _COURANT_2D_MAX)) if not ok]
        if problems:
            raise ValueError(f"Grid(nx={nx}, ny={ny}, dx={dx}, courant={courant}) needs "
                             + ", ".join(problems))
        object.__setattr__(self, "nx", int(nx))
        object.__setattr__(self, "ny", int(ny))
        object.__setattr__(self, "dx", float(dx))
        object.__setattr__(self, "courant", float(courant))
        object.__setattr__(self, "dtype", dtype)
        object.__setattr__(self, "device", device if device is not None else default_device())

    def __setattr__(self, name, value):
        raise AttributeError("Grid is immutable")

    def __repr__(self):
        return (f"Grid(nx={self.nx}, ny={self.ny}, dx={self.dx}, courant={self.courant}, "
                f"dtype={self.dtype}, device={self.device!r})")

    def __eq__(self, other):
        return isinstance(other, Grid) and all(
            getattr(self, k) == getattr(other, k) for k in self.__slots__)

    def __hash__(self):
        return hash(tuple(getattr(self, k) for k in self.__slots__))

    @property
    def dt(self) -> float:
        return self.courant * self.dx

    def zeros(self, *shape) -> torch.Tensor:
        """A zero tensor of the grid's dtype on its device."""
        return torch.zeros(*shape, dtype=self.dtype, device=self.device)
