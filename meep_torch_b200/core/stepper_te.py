"""TE state (reference: core/stepper_te.py:11-49) and a one-step driver."""
from typing import NamedTuple

import torch

from .grid import Grid
from .stepper_tm import _OneStepSource


class TEState(NamedTuple):
    Hz: torch.Tensor       # (nx-1, ny-1) at n
    Ex: torch.Tensor       # (nx-1, ny)   at n-1/2
    Ey: torch.Tensor       # (nx, ny-1)   at n-1/2
    Dx: torch.Tensor       # (nx-1, ny)
    Dy: torch.Tensor       # (nx, ny-1)
    Px_cur: torch.Tensor   # (n_poles, nx-1, ny) ADE polarisation on Ex
    Px_prev: torch.Tensor
    Py_cur: torch.Tensor   # (n_poles_y, nx, ny-1) on Ey
    Py_prev: torch.Tensor
    psi_Eyx: torch.Tensor  # (nx-1, ny-1)
    psi_Exy: torch.Tensor  # (nx-1, ny-1)
    psi_Hzy: torch.Tensor  # (nx-1, ny-2)
    psi_Hzx: torch.Tensor  # (nx-2, ny-1)


def init_te_state(grid: Grid, n_poles: int = 0, n_poles_y: int | None = None) -> TEState:
    """Zero TE state (core/stepper_te.py:27-49); n_poles sizes the Ex pole stack and
    n_poles_y (default n_poles: shared poles) the Ey one."""
    nx, ny = grid.nx, grid.ny
    npy = n_poles if n_poles_y is None else n_poles_y
    z = grid.zeros
    return TEState(Hz=z(nx - 1, ny - 1), Ex=z(nx - 1, ny), Ey=z(nx, ny - 1), Dx=z(nx - 1, ny),
                   Dy=z(nx, ny - 1), Px_cur=z(n_poles, nx - 1, ny),
                   Px_prev=z(n_poles, nx - 1, ny), Py_cur=z(npy, nx, ny - 1),
                   Py_prev=z(npy, nx, ny - 1),
                   psi_Eyx=z(nx - 1, ny - 1), psi_Exy=z(nx - 1, ny - 1),
                   psi_Hzy=z(nx - 1, ny - 2), psi_Hzx=z(nx - 2, ny - 1))


def step_te(state, m, src_amp=0.0, src_mask_ey=None, src_h_amp: float = 0.0,
            src_hz_mask=None):
    """One TE step (core/stepper_te.py:178-190: D half first, then Hz)."""
    from ..engine2d import Engine2D
    hm = {"src_hz_mask": src_hz_mask} if src_hz_mask is not None else {}
    src = _OneStepSource(src_amp, src_mask_ey, src_h_amp, hm)
    eng = Engine2D([(state, m, src if (src_mask_ey is not None or hm) else None, [])])
    eng.run(0, 1)
    out = eng.state(0)
    eng.close()
    return out
