"""Forward-only 3D entry point with the lean stepper's conventions
(reference: core/stepper_3d_lean.py:90-349).

The B200 kernel already updates in place-of-ping-pong with psi touched only in
the layers, so ``build_lean`` returns the same coefficient/state pair as the
functional path; ``run_3d_lean`` differs in the point-source sign (the lean
stepper subtracts dt*amp/eps) and returns a view with the fields as attributes.
"""
from dataclasses import dataclass, field

import torch

from ..engine3d import Engine3D
from .stepper_3d import build_3d_coeffs, init_3d_state


@dataclass
class Lean3D:
    dt: float
    dx: float
    nx: int
    ny: int
    nz: int
    npml: int
    coeffs: object
    F: dict = field(default_factory=dict)


class _StateView:
    def __init__(self, F):
        self.__dict__.update(F)


def build_lean(nx, ny, nz, dx, eps, npml, poles=(), pole_masks=None, dtype=torch.float32,
               device="cuda") -> Lean3D:
    """With ``poles`` / ``pole_masks`` the lean stepper's ADE poles
    (core/stepper_3d_lean.py:143-150): the same folded-D update as the functional
    stepper, which the split kernels' pole variant runs."""
    c = build_3d_coeffs(nx, ny, nz, dx, eps=eps, npml=npml, dtype=dtype, device=device,
                        poles=poles, pole_masks=pole_masks)
    st = init_3d_state(nx, ny, nz, npml=npml, dtype=dtype, device=device,
                       n_poles=len(poles))
    return Lean3D(dt=c.dt, dx=dx, nx=nx, ny=ny, nz=nz, npml=npml, coeffs=c, F=st._asdict())


def run_3d_lean(c: Lean3D, n_steps: int, *, source=None, monitors=(), compile: bool = False,
                phase_mode="exact", variant: int = 0):
    """``compile`` is accepted for signature parity; the kernels are already fused.
    ``variant`` selects the 3D kernel (0 default, 1 fused x-march, 2 split H / E)."""
    monitors = list(monitors)
    eng = Engine3D(dict(c.F), c.coeffs, source, monitors, point_sign=-1, phase_mode=phase_mode,
                   variant=variant)
    try:
        eng.run(0, n_steps)
        c.F = eng.state()
        return _StateView(c.F), list(eng.accs)
    finally:
        eng.close()
