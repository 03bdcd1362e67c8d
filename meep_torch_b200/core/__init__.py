"""Host-side mirror of meep_torch.core for the FDTD hot path.

Same names, argument meanings and error behaviour as the reference modules
(core/grid.py, core/pml.py, core/coeffs.py, core/stepper_tm.py,
core/stepper_te.py, core/sources.py, core/monitors.py, core/run.py,
core/stepper_3d.py, core/monitors_3d.py, core/stepper_3d_lean.py), restricted
to the feature set the B200 kernels implement. Setup (coefficients, masks) is
host code; every time step runs in the CUDA library.
"""
