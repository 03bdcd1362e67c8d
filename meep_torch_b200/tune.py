"""Autotuning of the 2D batch plan: time the library's launch shapes on the batch itself.

The best launch shape depends on the batch. Rows per warp trade register blocking against
parallelism (a small batch needs one row per warp to fill 148 SMs). The row march and
the tile kernels differ per structure size. The ring depth trades the contraction's
accumulator traffic against ring memory. ``autotune_2d`` builds one plan per candidate
on the batch (each plan imports its own copy of the state, so the caller's tensors are
not touched), times ``steps`` steps of each with CUDA events after ``warmup`` steps, and
returns the fastest candidate as keyword arguments for ``Engine2D``. The steps include
the DFT ring folds the candidate's ring depth implies.
"""
from __future__ import annotations

import torch

from .engine2d import Engine2D

__all__ = ["DEFAULT_CANDIDATES", "autotune_2d"]

DEFAULT_CANDIDATES = (
    {"variant": 3, "rows_per_warp": 0, "ring_slots": 32},     # library default: TB tiles
    {"variant": 3, "rows_per_warp": 0, "ring_slots": 16},
    {"variant": 2, "rows_per_warp": 0, "ring_slots": 32},     # one-step tiles
    {"variant": 2, "rows_per_warp": 1, "ring_slots": 32},     # tiles, one row per warp
    {"variant": 2, "rows_per_warp": 4, "ring_slots": 32},     # tiles, register-blocked rows
    {"variant": 1, "rows_per_warp": 0, "ring_slots": 32},     # row march
    {"variant": 2, "rows_per_warp": 0, "ring_slots": 16},
)


def autotune_2d(items, *, candidates=DEFAULT_CANDIDATES, steps: int = 64, warmup: int = 16,
                phase_mode: str = "exact", stream=None):
    """Returns (best keyword arguments, [(candidate, ms per step), ...]) for the batch
    ``items`` (the list Engine2D takes). ``steps`` should span at least one ring fold of
    the deepest candidate so that the contraction is in the timing."""
    items = list(items)
    if steps < 1 or warmup < 0:
        raise ValueError("steps must be >= 1 and warmup >= 0")
    results = []
    for cand in candidates:
        eng = Engine2D(items, phase_mode=phase_mode, stream=stream, **cand)
        try:
            st = stream if stream is not None else torch.cuda.current_stream(eng.device)
            if warmup:
                eng.run(0, warmup)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize(eng.device)
            e0.record(st)
            eng.run(warmup, steps)
            e1.record(st)
            torch.cuda.synchronize(eng.device)
            results.append((dict(cand), e0.elapsed_time(e1) / steps))
        finally:
            eng.close()
    best = min(results, key=lambda r: r[1])[0]
    return best, results
