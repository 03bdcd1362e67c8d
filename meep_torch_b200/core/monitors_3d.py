"""3D sources, monitors and the forward runner (reference: core/monitors_3d.py:18-210)."""
import torch

from ..engine3d import Engine3D


class PlaneSource:
    """Soft area current on the plane idx normal to ``axis`` on an E component
    (mask subtracted, core/stepper_3d.py:452-461)."""

    def __init__(self, nx, ny, nz, dt, comp, axis, idx, profile, lo=None, hi=None, device=None):
        shape = {"Ex": (nx - 1, ny, nz), "Ey": (nx, ny - 1, nz), "Ez": (nx, ny, nz - 1)}[comp]
        mask = torch.zeros(shape, dtype=torch.float32, device=device)
        sl = [slice(None)] * 3
        sl[axis] = idx
        mask[tuple(sl)] = 1.0
        if lo is not None and hi is not None:
            sel = [slice(None)] * 3
            for a in range(3):
                if a != axis:
                    sel[a] = slice(lo, hi)
            window = mask[tuple(sel)].clone()
            mask = torch.zeros_like(mask)
            mask[tuple(sel)] = window
        self.profile = profile
        self.dt = dt
        self.src = (comp, mask)

    def amplitude(self, t_idx: int) -> float:
        return self.profile.amplitude((t_idx + 0.5) * self.dt)


class PointSource3D:
    """Soft point current; run_3d ADDS dt*amp/eps (core/stepper_3d.py:474-480),
    run_3d_lean subtracts (core/stepper_3d_lean.py:293-296)."""
    _COMP = {"Ex", "Ey", "Ez"}

    def __init__(self, dt, comp, i, j, k, profile):
        if comp not in self._COMP:
            raise ValueError(f"PointSource3D comp must be Ex/Ey/Ez, got {comp!r}")
        self.dt = dt
        self.profile = profile
        self.src = (comp, int(i), int(j), int(k))

    def amplitude(self, t_idx: int) -> float:
        return self.profile.amplitude((t_idx + 0.5) * self.dt)


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
           rows_per_seg: int = 0, ring_slots: int = 0, variant: int = 0):
    """Forward 3D run (core/monitors_3d.py:192-210) on the B200 kernels."""
    monitors = list(monitors)
    if n_steps <= 0:
        return state, [None] * len(monitors)
    eng = Engine3D(state, coeffs, source, monitors, point_sign=+1, phase_mode=phase_mode,
                   rows_per_seg=rows_per_seg, ring_slots=ring_slots, variant=variant)
    try:
        eng.run(0, n_steps)
        return eng.state(), list(eng.accs)
    finally:
        eng.close()
