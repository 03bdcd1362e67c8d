"""CFS-PML profiles (reference: core/pml.py:8-59)."""
import math

import torch


def side_counts(n_or_pair) -> tuple[int, int]:
    """(n_low, n_high) cells from an int or a (lo, hi) pair."""
    if isinstance(n_or_pair, (tuple, list)):
        lo, hi = n_or_pair
        return int(lo), int(hi)
    return int(n_or_pair), int(n_or_pair)


def cpml_profiles(n, npml, offset, dt, dx, m=3, R0=1e-6, alpha_max=0.05,
                  dtype=torch.float32, device="cpu"):
    """(b, a, kappa) of length n at positions i + offset, evaluated in ``dtype``.

    sigma grows as u^m with sigma_max = -(m+1) ln(R0) / (2 n_side dx) over each
    layer, alpha = alpha_max (1 - u) inside it, kappa = 1, and
    b = exp(-(sigma/kappa + alpha) dt), a = sigma (b - 1) / (kappa (sigma + kappa alpha))
    where sigma > 0. The high-side ramp is anchored at n - 1 + 2 offset so the
    half-offset (H) and integer (E) profiles stretch together."""
    n_lo, n_hi = side_counts(npml)
    x = torch.arange(n, dtype=dtype, device=device) + offset
    u = torch.zeros(n, dtype=dtype, device=device)
    sigma = torch.zeros_like(u)
    if n_lo > 0:
        u_lo = torch.clamp((n_lo - x) / n_lo, min=0.0)
        u = u + u_lo
        sigma = sigma + (-(m + 1) * math.log(R0) / (2.0 * n_lo * dx)) * u_lo ** m
    if n_hi > 0:
        wall = n - 1 + 2.0 * offset
        u_hi = torch.clamp((x - (wall - n_hi)) / n_hi, min=0.0)
        u = u + u_hi
        sigma = sigma + (-(m + 1) * math.log(R0) / (2.0 * n_hi * dx)) * u_hi ** m
    u = torch.clamp(u, max=1.0)
    alpha = torch.where(u > 0, alpha_max * (1.0 - u), torch.zeros_like(u))
    kappa = torch.ones_like(u)
    b = torch.exp(-(sigma / kappa + alpha) * dt)
    denom = kappa * (sigma + kappa * alpha)
    a = torch.where(sigma > 0, sigma * (b - 1.0) / denom.clamp(min=torch.finfo(dtype).tiny),
                    torch.zeros_like(b))
    return b, a, kappa
