"""2D grid descriptor (reference: core/grid.py:33-59)."""
import math
import os
from dataclasses import dataclass, field

import torch


def default_device() -> str:
    """Device for new grids: ``MEEP_TORCH_DEVICE`` or ``cuda`` (the B200 path
    has no CPU mode, unlike core/grid.py:10-30 which defaults to CPU)."""
    return os.environ.get("MEEP_TORCH_DEVICE", "cuda")


@dataclass(frozen=True)
class Grid:
    """nx x ny nodes at spacing dx; dt = courant * dx. Defaults to float32,
    the dtype the kernels compute in (the reference defaults to float64)."""
    nx: int
    ny: int
    dx: float
    courant: float = 0.5
    dtype: torch.dtype = torch.float32
    device: str = field(default_factory=default_device)

    def __post_init__(self):
        if self.nx < 3:
            raise ValueError(f"nx must be >= 3, got {self.nx}")
        if self.ny < 3:
            raise ValueError(f"ny must be >= 3, got {self.ny}")
        if self.dx <= 0:
            raise ValueError(f"dx must be > 0, got {self.dx}")
        if not 0 < self.courant <= 1 / math.sqrt(2):
            raise ValueError(
                f"courant must be in (0, 1/sqrt(2)] for 2D stability, got {self.courant}")

    @property
    def dt(self) -> float:
        return self.courant * self.dx

    def zeros(self, *shape) -> torch.Tensor:
        return torch.zeros(*shape, dtype=self.dtype, device=self.device)
