"""TM state (reference: core/stepper_tm.py:12-71) and a one-step driver."""
from typing import NamedTuple

import torch

from .grid import Grid


class TMState(NamedTuple):
    Ez: torch.Tensor       # (nx, ny)        at n
    Hx: torch.Tensor       # (nx, ny-1)      at n-1/2
    Hy: torch.Tensor       # (nx-1, ny)      at n-1/2
    Dz: torch.Tensor       # (nx, ny)
    P_cur: torch.Tensor    # (n_poles, nx, ny) ADE polarisation of each pole
    P_prev: torch.Tensor
    psi_Ezy: torch.Tensor  # (nx, ny-1)      CPML memory of dEz/dy (Hx update)
    psi_Ezx: torch.Tensor  # (nx-1, ny)      dEz/dx (Hy update)
    psi_Hyx: torch.Tensor  # (nx_e, ny_e)    dHy/dx (Dz update, live Ez region)
    psi_Hxy: torch.Tensor  # (nx_e, ny_e)    dHx/dy
    Bx: torch.Tensor | None = None
    By: torch.Tensor | None = None
    Mx_cur: torch.Tensor | None = None
    Mx_prev: torch.Tensor | None = None
    My_cur: torch.Tensor | None = None
    My_prev: torch.Tensor | None = None
    Hx0: torch.Tensor | None = None   # (nx,) on-plane Hx row at a live low-y cut
    Hy0: torch.Tensor | None = None   # (ny,) on-plane Hy column at a live low-x cut


def init_tm_state(grid: Grid, n_poles: int = 0, y_pmc: bool = False, y_mirror: int = 0,
                  x_mirror: int = 0, y_rot2: int = 0, rot4: int = 0, n_mpoles: int = 0,
                  **kw) -> TMState:
    """Zero TM state, as core/stepper_tm.py:41-71: psi_Hyx / psi_Hxy cover the live
    Ez region -- the interior, every column under y_pmc, or from the cut row / column
    of a low-edge symmetry cut; P_cur / P_prev hold one (nx, ny) plane per dispersive
    pole; Hx0 / Hy0 are the on-plane H lines that an odd mirror, Rotate2 or Rotate4
    keeps live; ``n_mpoles`` magnetic poles add B and the M histories on Hx / Hy."""
    for k, v in kw.items():
        if v:
            raise NotImplementedError(f"{k}: not implemented on the B200 path")
    nx, ny = grid.nx, grid.ny
    y_cut, x_cut = bool(y_mirror or y_rot2 or rot4), bool(x_mirror or rot4)
    ny_e = ny if y_pmc else (ny - 1 if y_cut else ny - 2)
    nx_e = nx - 1 if x_cut else nx - 2
    z = grid.zeros
    return TMState(Ez=z(nx, ny), Hx=z(nx, ny - 1), Hy=z(nx - 1, ny), Dz=z(nx, ny),
                   P_cur=z(n_poles, nx, ny), P_prev=z(n_poles, nx, ny), psi_Ezy=z(nx, ny - 1),
                   psi_Ezx=z(nx - 1, ny), psi_Hyx=z(nx_e, ny_e), psi_Hxy=z(nx_e, ny_e),
                   Hx0=z(nx) if (y_mirror == -1 or y_rot2 or rot4) else None,
                   Hy0=z(ny) if (x_mirror == -1 or rot4) else None,
                   **(dict(Bx=z(nx, ny - 1), By=z(nx - 1, ny),
                           Mx_cur=z(n_mpoles, nx, ny - 1), Mx_prev=z(n_mpoles, nx, ny - 1),
                           My_cur=z(n_mpoles, nx - 1, ny), My_prev=z(n_mpoles, nx - 1, ny))
                      if n_mpoles else {}))


def step_tm(state, m, src_amp=0.0, src_mask=None, src_h_amp: float = 0.0,
            src_hy_mask=None, src_hx_mask=None):
    """One TM step (core/stepper_tm.py:234-254 phase order) on the GPU.
    Convenience wrapper: a run of k steps should use run_tm / _run_chunk."""
    from ..engine2d import Engine2D
    src = _OneStepSource(src_amp, src_mask, src_h_amp,
                         {k: v for k, v in (("src_hy_mask", src_hy_mask),
                                            ("src_hx_mask", src_hx_mask)) if v is not None})
    eng = Engine2D([(state, m, src if (src_mask is not None or src.h_masks) else None, [])])
    eng.run(0, 1)
    out = eng.state(0)
    eng.close()
    return out


class _OneStepSource:
    """Adapter: a fixed amplitude for the single step of step_tm / step_te."""

    def __init__(self, amp, mask, h_amp, h_masks):
        self._a, self.mask, self._h, self.h_masks = float(amp), mask, float(h_amp), h_masks

    def amplitude(self, t_idx):
        return self._a

    def h_amplitude(self, t_idx):
        return self._h
