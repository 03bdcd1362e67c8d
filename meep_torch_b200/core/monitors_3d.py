"""3D sources, monitors and the forward runner (reference: core/monitors_3d.py:18-210)."""
import torch

from ..engine3d import Engine3D


class _Sampled3D:
    """Shared by the 3D sources: the profile sampled at half steps (t_idx + 1/2) dt."""

    def amplitude(self, t_idx: int) -> float:
        return self.profile.amplitude((t_idx + 0.5) * self.dt)


# array shape of each E component (its staggered axis is one node shorter)
_E_AXIS = {"Ex": 0, "Ey": 1, "Ez": 2}


class PlaneSource(_Sampled3D):
    """A soft area current with unit weight on the plane idx normal to ``axis`` of one E
    component, optionally limited to [lo, hi) along the two in-plane axes; run_3d
    subtracts dt amp mask / eps (core/stepper_3d.py:452-461)."""

    def __init__(self, nx, ny, nz, dt, comp, axis, idx, profile, lo=None, hi=None, device=None):
        shape = [nx, ny, nz]
        shape[_E_AXIS[comp]] -= 1
        region = [slice(None)] * 3
        region[axis] = idx
        if lo is not None and hi is not None:
            for other in {0, 1, 2} - {axis}:
                region[other] = slice(lo, hi)
        mask = torch.zeros(shape, dtype=torch.float32, device=device)
        mask[tuple(region)] = 1.0
        self.src = (comp, mask)
        self.profile = profile
        self.dt = dt


class PointSource3D(_Sampled3D):
    """A soft current at one node (i, j, k) of an E component. The functional stepper
    adds dt amp / eps there (core/stepper_3d.py:474-480); the lean stepper subtracts it
    (core/stepper_3d_lean.py:293-296)."""

    def __init__(self, dt, comp, i, j, k, profile):
        if comp not in _E_AXIS:
            raise ValueError(f"PointSource3D drives Ex, Ey or Ez, not {comp!r}")
        self.src = (comp, int(i), int(j), int(k))
        self.profile = profile
        self.dt = dt


class DFTFieldsMonitor3D:
    """Running DFT of one component on a plane (axis, idx); accumulator
    (nfreq, 2, *plane shape)."""
    reduce = "sum"

    def __init__(self, dt, freqs, component="Ez", plane=None, dtype=torch.float64):
        self.component = component
        self.dt = dt
        self.freqs = torch.tensor(freqs, dtype=dtype)
        self.plane = plane


class FluxMonitor3D:
    """Poynting flux through an axis-normal plane: 8 accumulators (Re/Im of
    Ea, Ha, Eb, Hb) on the window ``win`` = (l0, h0, l1, h1) or the centred
    ``ap`` margin; flux = 1/2 sum(sa - sb) dx^2 (core/monitors_3d.py:97-189)."""
    reduce = "sum"

    def __init__(self, dt, freqs, *, normal, idx, ap=0, win=None, dtype=torch.float64):
        if normal not in ("x", "y", "z"):
            raise ValueError(f"normal must be x/y/z, got {normal!r}")
        self.normal = normal
        self.idx = idx
        self.ap = ap
        self.win = win
        self.dt = dt
        self.freqs = torch.tensor(freqs, dtype=dtype)

    def flux(self, acc: torch.Tensor, dx: float) -> torch.Tensor:
        ReaE, ImaE, ReaH, ImaH, RebE, ImbE, RebH, ImbH = acc.unbind(1)
        sa = ReaE * ReaH + ImaE * ImaH
        sb = RebE * RebH + ImbE * ImbH
        return 0.5 * (sa - sb).sum(tuple(range(1, sa.ndim))) * dx * dx


def run_3d(state, coeffs, n_steps: int, *, source=None, monitors=(), phase_mode="exact",
           rows_per_seg: int = 0, ring_slots: int = 0, variant: int = 0, geometry: int = 0):
    """Forward 3D run (core/monitors_3d.py:192-210) on the B200 kernels. ``variant`` and
    ``geometry`` are the plan's tuning knobs (``mtb_tuning``)."""
    monitors = list(monitors)
    if n_steps <= 0:
        return state, [None] * len(monitors)
    eng = Engine3D(state, coeffs, source, monitors, point_sign=+1, phase_mode=phase_mode,
                   rows_per_seg=rows_per_seg, ring_slots=ring_slots, variant=variant,
                   geometry=geometry)
    try:
        eng.run(0, n_steps)
        return eng.state(), list(eng.accs)
    finally:
        eng.close()
