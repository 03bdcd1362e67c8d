"""CFS-PML recursion coefficients (reference interface: core/pml.py:8-59).

For a node at position p = i + offset, d(p) in [0, 1] is its normalised depth into the
low layer (n_lo cells, from p = 0 inward) or the high layer (n_hi cells, whose outer wall
sits at n - 1 + 2 offset, so the half-offset and integer profiles share one wall).
With grading order m and target reflection R0 (the published CFS-CPML choices):

    sigma(p) = sigma_max d^m,  sigma_max = (m + 1) ln(1 / R0) / (2 n_side dx)
    alpha(p) = alpha_max (1 - d) inside a layer, 0 outside;  kappa = 1
    b = exp(-(sigma / kappa + alpha) dt)
    a = sigma (b - 1) / (kappa (sigma + kappa alpha))  where sigma > 0, else 0

and the memory recursion psi' = b psi + a d_field. Each profile is evaluated in float64
and rounded once to the requested dtype.
"""
import math

import numpy as np
import torch


def side_counts(n_or_pair) -> tuple[int, int]:
    """(n_low, n_high) layer cells from one count or a (low, high) pair."""
    if isinstance(n_or_pair, (tuple, list)):
        return int(n_or_pair[0]), int(n_or_pair[1])
    return int(n_or_pair), int(n_or_pair)


def _depth(pos: np.ndarray, n: int, offset: float, n_lo: int, n_hi: int):
    """Per-layer normalised depths (low, high), zero outside each layer."""
    zero = np.zeros_like(pos)
    lo = np.clip((n_lo - pos) / n_lo, 0.0, None) if n_lo > 0 else zero
    hi = np.clip((pos - (n - 1 + 2.0 * offset - n_hi)) / n_hi, 0.0, None) if n_hi > 0 else zero
    return lo, hi


def cpml_profiles(n, npml, offset, dt, dx, m=3, R0=1e-6, alpha_max=0.05,
                  dtype=torch.float32, device="cpu"):
    """(b, a, kappa), each of length n, for nodes at positions i + offset."""
    n_lo, n_hi = side_counts(npml)
    pos = np.arange(n, dtype=np.float64) + offset
    d_lo, d_hi = _depth(pos, n, offset, n_lo, n_hi)
    grade = lambda count: (m + 1) * math.log(1.0 / R0) / (2.0 * count * dx)  # noqa: E731
    sigma = np.zeros(n)
    if n_lo > 0:
        sigma += grade(n_lo) * d_lo ** m
    if n_hi > 0:
        sigma += grade(n_hi) * d_hi ** m
    depth = np.minimum(d_lo + d_hi, 1.0)
    alpha = np.where(depth > 0, alpha_max * (1.0 - depth), 0.0)
    b = np.exp(-(sigma + alpha) * dt)
    a = np.zeros(n)
    active = sigma > 0
    a[active] = sigma[active] * (b[active] - 1.0) / (sigma[active] + alpha[active])
    out = lambda v: torch.tensor(v, dtype=dtype, device=device)  # noqa: E731
    return out(b), out(a), torch.ones(n, dtype=dtype, device=device)


def absorber_sigma(n: int, nabs, dx: float, *, R0: float = 1e-15, m: int = 2,
                   dtype=torch.float32, device="cpu") -> torch.Tensor:
    """Conductivity of a matched absorber (meep's Absorber; reference interface
    core/pml.py:62-80) along an axis of n cells: zero inside, and over the n_side cells
    of each layer a ramp sigma_max u^m of the cell-centre depth u = (n_side - i - 1/2) /
    n_side counted from the outer edge, with sigma_max = (m + 1) ln(1 / R0) / (2 n_side
    dx). The same curve damps D and B (sigma_d = sigma_b)."""
    n_lo, n_hi = side_counts(nabs)
    sig = np.zeros(n)
    for count, edge in ((n_lo, "lo"), (n_hi, "hi")):
        if count <= 0:
            continue
        peak = (m + 1) * math.log(1.0 / R0) / (2.0 * count * dx)
        ramp = peak * ((count - np.arange(count) - 0.5) / count) ** m
        if edge == "lo":
            sig[:count] = ramp
        else:
            sig[n - count:] = ramp[::-1]
    return torch.tensor(sig, dtype=dtype, device=device)
