"""cfg5 surrogate: design maps, FNO, the trust-region design loop and plan reuse.

CPU tests cover the host logic (maps, the FNO on CPU, the loop's accept / reject
rules on an analytic problem). GPU tests cover Engine2D.set_eps against a freshly
built plan, batched vs single-design data generation, the BF16 FNO's forward and
gradients against an FP64 CPU copy with the same weights, and a short end-to-end run.
"""
import copy

import pytest
import torch

from meep_torch_b200 import surrogate as S


def test_grf_designs_seeded_and_bounded():
    a = S.grf_designs(6, seed=11)
    b = S.grf_designs(6, seed=11)
    assert a.shape == (6, 64, 64)
    assert torch.equal(a, b)
    assert float(a.min()) >= 0.0 and float(a.max()) <= 1.0
    m = S.grf_designs(64, seed=3).mean()
    assert 0.3 < float(m) < 0.7
    assert not torch.equal(S.grf_designs(2, seed=1), S.grf_designs(2, seed=2))


def test_grf_soft_half_is_grey():
    """With soft = 0.5 the second half of the maps is soft-thresholded: far more grey
    pixels (0.2 < rho < 0.8) than the thresholded half, whose grey pixels are only the
    filtered edges; the first half equals the all-binary maps of the same seed."""
    hard = S.grf_designs(16, seed=4)
    mixed = S.grf_designs(16, seed=4, soft=0.5)
    assert torch.equal(mixed[:8], hard[:8])
    grey = lambda r: float(((r > 0.2) & (r < 0.8)).float().mean())  # noqa: E731
    assert grey(mixed[8:]) > 2.0 * grey(mixed[:8])
    assert float(mixed.min()) >= 0.0 and float(mixed.max()) <= 1.0


def test_problem_geometry_cpu():
    p = S.Cfg5Problem("cpu")
    rho = torch.zeros(2, 64, 64)
    rho[1] = 1.0
    eps = p.eps_map(rho)
    assert eps.shape == (2, 256, 256)
    assert float(eps[0].max()) == 1.0
    assert float(eps[1, 96:160, 96:160].min()) == 4.0
    assert float(eps[1, :96].max()) == 1.0
    x = p.fno_input(rho)
    assert x.shape == (2, 1, 128, 128)
    assert float(x[1, 0, 32:96, 32:96].min()) == 1.0 and float(x[1, 0, :32].max()) == 0.0
    f = torch.zeros(1, 6, 128, 128)
    i0, i1, j0, j1 = p.c["target"]
    f[:, 0, i0 - 64:i1 - 64, j0 - 64:j1 - 64] = 2.0          # Re of frequency 0
    assert torch.allclose(p.fom(f), torch.tensor([4.0 / 3.0]))


def test_fno_shapes_cpu():
    m = S.FNO2d(width=8, modes=4, layers=2)
    y = m(torch.rand(3, 1, 32, 32))
    assert y.shape == (3, 6, 32, 32)
    y.square().mean().backward()
    assert all(p.grad is not None for p in m.parameters())


def test_fno_fp64_restatement_matches_fno_cpu():
    """The FP64 restatement used as the GPU FNO's oracle agrees with FNO2d run in
    FP32 on the CPU (no autocast there)."""
    torch.manual_seed(2)
    m = S.FNO2d(width=16, modes=6, layers=3)
    ref = copy.deepcopy(m).double()
    x = torch.rand(2, 1, 32, 32)
    y = m(x)
    yr = _fno_fp64(ref, x.double())
    assert float((y.double() - yr).detach().norm() / yr.detach().norm()) < 1e-5
    (y.square().sum()).backward()
    (yr.square().sum()).backward()
    for (n, pa), pb in zip(m.named_parameters(), ref.parameters()):
        g = pb.grad.to(pa.grad.dtype)
        assert float((pa.grad - g).norm() / g.norm()) < 1e-4, n


class _Quadratic:
    """An analytic stand-in for Cfg5Problem: FOM = 10 - |rho - rho*|^2 / 64 with a
    smooth optimum rho*, 'FDTD' gradients exact; the surrogate is a biased model."""

    def __init__(self):
        self.device = torch.device("cpu")
        g = torch.Generator().manual_seed(0)
        self.opt = 0.2 + 0.6 * torch.rand(8, 8, generator=g)
        self.runs = 0

    def _f(self, rho):
        return 10.0 - (rho - self.opt).square().sum(dim=(-2, -1)) / 64

    def fdtd_fom_and_grad(self, rho, fields=False):
        self.runs += 1
        f = float(self._f(rho))
        g = -2.0 * (rho - self.opt) / 64
        return (f, g, torch.full((1, 1, 1, 1), f)) if fields else (f, g)

    def simulate(self, rhos, batch=0):
        self.runs += 1
        return self._f(rhos)[:, None, None, None]

    def fno_input(self, rho):
        return rho[:, None]

    def fom(self, fields):
        return fields.flatten(1).mean(1)


class _BiasedModel(torch.nn.Module):
    """Surrogate of _Quadratic with a wrong optimum and a wrong offset."""

    def __init__(self, opt):
        super().__init__()
        self.w = torch.nn.Parameter(torch.ones(()))
        self.opt = (opt + 0.1).clamp(0, 1)

    def forward(self, x):
        d = x[:, 0] - self.opt
        return (3.0 - 1.5 * d.square().sum(dim=(1, 2)) / 64 * self.w)[:, None, None, None] \
            .expand(x.shape[0], 1, 1, 1)


def test_trust_region_loop_monotone_and_reaches_target_cpu():
    prob = _Quadratic()
    rho0 = torch.full((8, 8), 0.5)
    plain = S.design_loop(prob, rho0, 40, lr=0.05)
    assert plain["fom"][-1] > plain["fom"][0]
    model = _BiasedModel(prob.opt)
    target = 0.99999 * 10.0
    sur = S.design_loop(prob, rho0, 40, model=model, target=target, inner=10, inner_lr=0.2,
                        probes=(2, 5, 10))
    best = sur["fom"][0]
    for f, ok in zip(sur["fom"][1:], sur["accepted"][1:]):
        assert ok == (f > best)
        if ok:
            best = f
    assert sur["fdtd_runs"] == prob.runs - 1 - len(plain["fom"]) + 1
    assert sur["adjoint_runs"] == 1 + sum(sur["accepted"][1:])
    assert sur["surrogate_steps"] == 10 * (len(sur["fom"]) - 1)
    # model parameters are left as they were (trainable, no gradient)
    assert model.w.requires_grad and model.w.grad is None
    assert max(sur["fom"]) > plain["fom"][-1]


def test_trust_region_rejects_bad_proposals_cpu():
    """A surrogate pointing the wrong way: the first-order correction still makes the
    corrected model ascend, and rejected proposals leave the anchor unchanged."""
    prob = _Quadratic()

    class Wrong(torch.nn.Module):
        def __init__(self):
            super().__init__()
            self.k = torch.nn.Parameter(torch.tensor(50.0))

        def forward(self, x):
            return (self.k * (x[:, 0] - 0.5).square().mean(dim=(1, 2)))[:, None, None, None]

    out = S.design_loop(prob, torch.full((8, 8), 0.5), 12, model=Wrong(), inner=5,
                        probes=(1, 5))
    accepted = [f for f, ok in zip(out["fom"], out["accepted"]) if ok]
    assert accepted == sorted(accepted)
    assert float(prob._f(out["rho"])) == pytest.approx(accepted[-1], abs=1e-5)


def test_trust_region_finetunes_the_model_cpu():
    """With finetune > 0 the surrogate learns from the verified probes (here the
    'fields' are the FOM itself): its parameters move toward the FDTD values and are
    left trainable afterwards."""
    prob = _Quadratic()
    model = _BiasedModel(prob.opt)
    w0 = float(model.w.detach())
    rx = torch.rand(32, 1, 8, 8)
    ry = prob._f(rx[:, 0])[:, None, None, None]
    out = S.design_loop(prob, torch.full((8, 8), 0.5), 6, model=model, inner=8,
                        probes=(4, 8), finetune=5, ft_lr=0.05, replay=(rx, ry))
    assert float(model.w.detach()) != w0
    assert model.w.requires_grad
    accepted = [f for f, ok in zip(out["fom"], out["accepted"]) if ok]
    assert accepted == sorted(accepted) and len(accepted) >= 2


# ------------------------------------------------------------------------ GPU

@pytest.mark.gpu
def test_set_eps_matches_fresh_plan():
    from meep_torch_b200.engine2d import Engine2D
    dev = torch.device("cuda", 0)
    p = S.Cfg5Problem(dev, steps=300)
    rho = S.grf_designs(6, seed=7).to(dev)
    eps = p.eps_map(rho)
    eng = Engine2D([p._item(e) for e in eps[:3]])
    eng.run(0, 300)
    for b in range(3):
        eng.set_eps(b, eps[3 + b])
    eng.reset()
    eng.run(0, 300)
    got = [eng.accumulators(b)[0].clone() for b in range(3)]
    eng.close()
    fresh = Engine2D([p._item(e) for e in eps[3:]])
    fresh.run(0, 300)
    for b in range(3):
        assert torch.equal(got[b], fresh.accumulators(b)[0])
    fresh.close()


@pytest.mark.gpu
def test_set_eps_refuses_conductive_structures():
    from meep_torch_b200 import _lib as L
    from meep_torch_b200.core.coeffs import build_tm_coeffs
    from meep_torch_b200.engine2d import Engine2D
    dev = torch.device("cuda", 0)
    p = S.Cfg5Problem(dev, steps=10)
    st, _, src, mons = p._item(torch.ones(256, 256, device=dev))
    m = build_tm_coeffs(p.grid, eps_inf=torch.ones(256, 256, device=dev), npml=20, sigma_d=0.1)
    eng = Engine2D([(st, m, src, mons)])
    with pytest.raises(L.MtbUnsupported):
        eng.set_eps(0, torch.ones(256, 256, device=dev))
    eng.close()


@pytest.mark.gpu
def test_simulate_batched_equals_single():
    dev = torch.device("cuda", 0)
    p = S.Cfg5Problem(dev, steps=400)
    rho = S.grf_designs(5, seed=9).to(dev)
    both = p.simulate(rho, batch=3)                  # plans of 3, then 2
    again = p.simulate(rho[1:2], batch=1)
    p.close()
    assert both.shape == (5, 6, 128, 128)
    assert torch.allclose(both[1], again[0], rtol=1e-6, atol=1e-6 * float(both.abs().max()))


@pytest.mark.gpu
def test_fno_bf16_forward_and_gradients_vs_cpu_fp64():
    """The GPU FNO (BF16 autocast, FP32 accumulation, FP32 FFTs) against an FP64 CPU
    copy with the same weights: outputs and every parameter gradient within BF16
    tolerance (relative L2 3e-2)."""
    torch.manual_seed(0)
    dev = torch.device("cuda", 0)
    m = S.FNO2d().to(dev)
    ref = copy.deepcopy(m).cpu().double()
    x = torch.rand(4, 1, 128, 128, device=dev)
    t = torch.randn(4, 6, 128, 128, device=dev)
    y = m(x)
    (y * t).sum().backward()
    xr = x.cpu().double()
    b, _, h, w = xr.shape
    yr = _fno_fp64(ref, xr)
    (yr * t.cpu().double()).sum().backward()

    def rel(a, b):
        wide = torch.complex128 if a.is_complex() else torch.float64
        a, b = a.detach().cpu().to(wide), b.detach().to(wide)
        return float((a - b).norm() / b.norm())
    assert rel(y, yr) < 3e-2
    for (n, pa), pb in zip(m.named_parameters(), ref.parameters()):
        assert rel(pa.grad, pb.grad) < 3e-2, n


def _fno_fp64(m, x):
    """FNO2d.forward without autocast (FP64 on CPU)."""
    import torch.nn.functional as F
    b, _, h, w = x.shape
    gy, gx = torch.meshgrid(torch.linspace(0, 1, h, dtype=x.dtype),
                            torch.linspace(0, 1, w, dtype=x.dtype), indexing="ij")
    x = torch.cat([x, gy.expand(b, 1, h, w), gx.expand(b, 1, h, w)], dim=1)
    x = m.lift(x)
    for k, (s, mix) in enumerate(zip(m.spec, m.mix)):
        xf = torch.fft.rfft2(x)
        md = s.modes
        out = torch.zeros(b, x.shape[1], h, w // 2 + 1, dtype=xf.dtype)
        wc = s.w.to(torch.complex128)
        out[:, :, :md, :md] = torch.einsum("bixy,ioxy->boxy", xf[:, :, :md, :md], wc[0])
        out[:, :, -md:, :md] = torch.einsum("bixy,ioxy->boxy", xf[:, :, -md:, :md], wc[1])
        y = torch.fft.irfft2(out, s=(h, w)) + mix(x)
        x = F.gelu(y) if k < len(m.spec) - 1 else y
    return m.proj2(F.gelu(m.proj1(x)))


@pytest.mark.gpu
def test_short_end_to_end_loop():
    """Short runs (400 steps): data, a few epochs of training, and both loops. The
    adjoint's forward FOM equals the batched forward's; the trained FNO beats the
    untrained one on held-out designs; the surrogate loop's accepted FOMs rise."""
    dev = torch.device("cuda", 0)
    p = S.Cfg5Problem(dev, steps=400)
    rho = S.grf_designs(544, seed=5).to(dev)
    y = p.simulate(rho, batch=272)
    x = p.fno_input(rho)
    torch.manual_seed(1)
    m = S.FNO2d().to(dev)
    scale = float(y[:512].pow(2).mean().sqrt())
    e0 = S.rel_error(m, x[512:], y[512:], scale)
    scale, _ = S.train_fno(m, x[:512], y[:512], epochs=4, scale=scale)
    e1 = S.rel_error(m, x[512:], y[512:], scale)
    assert e1 < 0.7 * e0
    f, g = p.fdtd_fom_and_grad(rho[0])
    assert f == pytest.approx(float(p.fom(y[:1])[0]), rel=1e-5)
    assert g.shape == (64, 64) and torch.isfinite(g).all()
    out = S.design_loop(p, torch.full((64, 64), 0.5), 4, model=m, scale=scale, finetune=2,
                        replay=(x[:512], y[:512] / scale))
    acc = [v for v, ok in zip(out["fom"], out["accepted"]) if ok]
    assert acc == sorted(acc) and len(out["fom"]) == 4
    assert out["adjoint_runs"] == sum(out["accepted"]) and out["fdtd_runs"] == 3 + acc.__len__()
    plain = S.design_loop(p, torch.full((64, 64), 0.5), 3)
    assert plain["fom"][0] == pytest.approx(out["fom"][0], rel=1e-5)
    p.close()


def test_trust_region_grad_every_cpu():
    """grad_every = 2: every second accepted anchor gets an adjoint run; the loop
    still only accepts verified improvements."""
    prob = _Quadratic()
    model = _BiasedModel(prob.opt)
    out = S.design_loop(prob, torch.full((8, 8), 0.5), 10, model=model, inner=6,
                        probes=(2, 4, 6), grad_every=2)
    n_acc = sum(out["accepted"][1:])
    assert out["adjoint_runs"] == 1 + n_acc // 2
    accepted = [f for f, ok in zip(out["fom"], out["accepted"]) if ok]
    assert accepted == sorted(accepted) and n_acc >= 2


def _bf(t):
    return t.detach().to(torch.bfloat16).float()


@pytest.mark.gpu
@pytest.mark.parametrize("cout,act,hw", [(64, True, (24, 24)), (64, False, (16, 16)),
                                         (128, True, (32, 20))])
def test_channel_mix_kernels_vs_fp32(cout, act, hw):
    """The tcgen05 channel mix (forward, dx, dW) against FP32 torch on the same
    BF16-rounded operands: only the accumulation order differs. 576 pixels exercise
    a partial 128-pixel tile."""
    import torch.nn.functional as F

    from meep_torch_b200 import _lib as L
    dev = torch.device("cuda", 0)
    g = torch.Generator(device="cpu").manual_seed(3)
    bsz, cin = 3, 64
    h, w = hw
    x = torch.randn(bsz, cin, h, w, generator=g).to(dev).requires_grad_(True)
    W = (torch.randn(cout, cin, 1, 1, generator=g) / 8).to(dev).requires_grad_(True)
    b = torch.randn(cout, generator=g).to(dev).requires_grad_(True)
    s = torch.randn(bsz, cout, h, w, generator=g).to(dev).requires_grad_(True)
    y = S.channel_mix(x, W, b, s, act)
    zr = (torch.einsum("oi,bihw->bohw", _bf(W[:, :, 0, 0]), _bf(x)) + b.detach()[None, :, None, None]
          + s.detach()).requires_grad_(True)
    yr = F.gelu(zr) if act else zr

    def rel(a, r):
        return float((a.detach() - r.detach()).norm() / r.detach().norm())
    assert rel(y, yr) < 1e-5
    dy = torch.randn(y.shape, generator=g).to(dev)
    y.backward(dy)
    yr.backward(dy)
    dzr = zr.grad
    dxr = torch.einsum("oi,bohw->bihw", _bf(W[:, :, 0, 0]), _bf(dzr))
    dwr = torch.einsum("bohw,bihw->oi", _bf(dzr), _bf(x))
    assert rel(x.grad, dxr) < 1e-4
    assert rel(W.grad[:, :, 0, 0], dwr) < 1e-4
    assert rel(b.grad, dzr.sum(dim=(0, 2, 3))) < 1e-5
    assert rel(s.grad, dzr) < 1e-5
    L.check(L.load().mtb_fno_status(torch.cuda.current_stream().cuda_stream), "mtb_fno_status")


@pytest.mark.gpu
def test_channel_mix_rejects_unbuilt_shapes():
    from meep_torch_b200 import _lib as L
    dev = torch.device("cuda", 0)
    x = torch.randn(1, 32, 8, 8, device=dev)
    with pytest.raises(L.MtbUnsupported):
        S.channel_mix(x, torch.randn(64, 32, 1, 1, device=dev))
    x = torch.randn(1, 64, 3, 3, device=dev)                      # 9 pixels: not a multiple of 8
    with pytest.raises(ValueError):
        S.channel_mix(x, torch.randn(64, 64, 1, 1, device=dev))
