"""Run drivers on the B200 kernels (reference: core/run.py:10-126).

``_run_chunk`` keeps the reference's signature and return value -- the
advanced state in the input's own type and one accumulator per monitor -- but
the k steps run inside the CUDA library: one fused launch per step plus one
DFT contraction per ring of steps, instead of ~30 torch ops per step.
"""
import torch

from ..engine2d import Engine2D


def _run_chunk(step_fn, state, coeffs, step0: int, k: int, source, monitors,
               *, phase_mode: str = "exact"):
    """Advance ``state`` k steps from step index step0 (core/run.py:10-40).
    ``step_fn`` only names the polarisation (step_tm / step_te); the state's
    type decides it here. Monitors are sum-reduced."""
    monitors = list(monitors)
    eng = Engine2D([(state, coeffs, source, monitors)], phase_mode=phase_mode)
    try:
        eng.run(step0, k)
        return eng.state(0), eng.accumulators(0)
    finally:
        eng.close()


def _make_runner(kind):
    def run(state, coeffs, n_steps: int, *, source=None, monitors=(), checkpoint_every: int = 0,
            phase_mode: str = "exact"):
        """core/run.py:44-122. When the eps the kernels read requires grad (TM
        coeffs.eps_inf; TE coeffs.eps_x / eps_y, e.g. built from an eps_inf that
        requires grad) and grad mode is on, the run is differentiable through the
        library's adjoint kernels, checkpointed every ``checkpoint_every`` steps
        (the default 32); otherwise checkpoint_every has no effect."""
        monitors = list(monitors)
        if n_steps <= 0:
            return state, [None] * len(monitors)
        eps = [getattr(coeffs, f, None) for f in (("eps_x", "eps_y") if kind == "te"
                                                 else ("eps_inf",))]
        if torch.is_grad_enabled() and any(torch.is_tensor(e) and e.requires_grad for e in eps):
            from ..adjoint2d import run_grad
            return run_grad(state, coeffs, n_steps, source=source, monitors=monitors,
                            checkpoint_every=checkpoint_every, phase_mode=phase_mode)
        state, acc = _run_chunk(None, state, coeffs, 0, n_steps, source, monitors,
                                phase_mode=phase_mode)
        return state, acc
    run.__name__ = f"run_{kind}"
    return run


run_tm = _make_runner("tm")
run_te = _make_runner("te")
