"""Surrogate-assisted inverse design on the FDTD engine (the cfg5 workload).

The FDTD data and every verification run through the library's batched 2D TM kernels.
The surrogate is a Fourier neural operator (FNO) trained on those runs. Its pointwise
channel mixes (fused with the spectral branch's sum, the bias and GELU) and its
64 -> 128 projection run forward and backward on the library's tcgen05 kernels (BF16
operands, FP32 accumulation in TMEM). The spectral transforms are cuFFT (torch.fft),
and the per-mode complex mixes are FP32 cuBLAS: library calls.

Pieces:

* ``grf_designs``: seeded design maps. A Gaussian random field (correlation length in
  pixels) is thresholded at 0, then conic-filtered (``design.conic_filter``).
* ``Cfg5Problem``: the 256 x 256 TM cell at resolution 20. It has a 20-cell CPML, a 64 x 64
  design painted at the centre (eps between ``eps_min`` and ``eps_max``) and a Gaussian
  line source across the grid 10 cells inside the left absorber. The DFT of Ez at three
  frequencies is read on the 128 x 128 region around the design.
  ``simulate(rho)`` runs a batch of designs in one plan and returns the six real target
  channels (Re, Im per frequency). ``fom(fields)`` is the objective: the mean |Ez|^2 over
  a target patch behind the design, averaged over the frequencies.
* ``FNO2d``: lift (eps, x, y) to ``width`` channels, ``layers`` Fourier layers (rfft2,
  ``modes`` x ``modes`` low modes in each corner mixed by complex weights, plus a 1x1
  channel mix, GELU), then a projection to the six channels.
* ``train_fno``: Adam with a cosine schedule on the relative L2 error.
* ``design_loop``: gradient ascent on the design latent. Without a model each
  iteration is one FDTD run with the library's adjoint (``run_tm`` with eps requiring
  grad): the plain loop. With one, blocks of surrogate steps on a first-order-corrected
  FNO propose designs inside a trust region, and an FDTD adjoint run verifies each
  proposal and re-anchors the correction.
"""
from __future__ import annotations

import math
import time

import torch
import torch.nn as nn
import torch.nn.functional as F

from .design import conic_filter

__all__ = ["CFG5", "grf_designs", "Cfg5Problem", "FNO2d", "channel_mix", "train_fno",
           "rel_error", "design_loop", "shard_range"]

CFG5 = dict(n=256, dx=0.05, npml=20, design=64, region=128, eps_min=1.0, eps_max=4.0,
            freqs=(0.6, 0.65, 0.7), fcen=0.65, fwidth=0.25, steps=3000, corr_px=4.0,
            filter_radius=0.1, target=(176, 184, 124, 132))


def grf_designs(n: int, size: int = 64, corr_px: float = 4.0, radius: float = 0.1,
                dx: float = 0.05, seed: int = 5, device="cpu", soft: float = 0.0,
                beta=(0.5, 4.0)) -> torch.Tensor:
    """``n`` Gaussian-random-field maps (size x size, correlation length ``corr_px``
    pixels), conic-filtered with ``radius``: values in [0, 1]. The first
    ``n - round(soft * n)`` maps are thresholded at 0 (binary); the rest are
    soft-thresholded, sigmoid(beta * g / std(g)) with beta uniform in ``beta``, which
    gives the grey densities a gradient-based design passes through."""
    g = torch.Generator(device="cpu").manual_seed(seed)
    noise = torch.randn(n, size, size, generator=g)
    k = torch.fft.fftfreq(size)
    k2 = k[:, None] ** 2 + k[None, :] ** 2
    kernel = torch.exp(-2.0 * (math.pi * corr_px) ** 2 * k2)
    field = torch.fft.ifft2(torch.fft.fft2(noise) * kernel).real
    rho = (field > 0).to(torch.float32)
    n_soft = int(round(soft * n))
    if n_soft:
        b = beta[0] + (beta[1] - beta[0]) * torch.rand(n_soft, 1, 1, generator=g)
        f = field[n - n_soft:]
        rho[n - n_soft:] = torch.sigmoid(b * f / f.std(dim=(1, 2), keepdim=True))
    out = torch.stack([conic_filter(r, radius, dx) for r in rho])
    return out.to(device)


class Cfg5Problem:
    """The cfg5 TM cell; ``simulate`` batches designs through one Engine2D plan."""

    def __init__(self, device, steps: int | None = None, **over):
        self.c = dict(CFG5, **over)
        if steps is not None:
            self.c["steps"] = int(steps)
        c = self.c
        self.device = torch.device(device)
        n, d, r = c["n"], c["design"], c["region"]
        self.d0 = (n - d) // 2
        self.r0 = (n - r) // 2
        from .core.grid import Grid
        from .core.sources import GaussianPulse, LineSource
        self.grid = Grid(nx=n, ny=n, dx=c["dx"], device=self.device)
        self.source = LineSource(self.grid, ix=c["npml"] + 10, j0=c["npml"], j1=n - c["npml"],
                                 profile=GaussianPulse(c["fcen"], c["fwidth"]))

    # -------------------------------------------------------------- geometry
    def eps_map(self, rho: torch.Tensor) -> torch.Tensor:
        """(B, d, d) design densities -> (B, n, n) eps."""
        c, d0, d = self.c, self.d0, self.c["design"]
        eps = torch.full((rho.shape[0], c["n"], c["n"]), c["eps_min"], dtype=torch.float32,
                         device=rho.device)
        eps[:, d0:d0 + d, d0:d0 + d] = c["eps_min"] + (c["eps_max"] - c["eps_min"]) * rho
        return eps

    def region(self, full: torch.Tensor) -> torch.Tensor:
        r0, r = self.r0, self.c["region"]
        return full[..., r0:r0 + r, r0:r0 + r]

    def fno_input(self, rho: torch.Tensor) -> torch.Tensor:
        """(B, d, d) -> (B, 1, region, region) normalised eps of the region."""
        c = self.c
        e = self.region(self.eps_map(rho))
        return ((e - c["eps_min"]) / (c["eps_max"] - c["eps_min"]))[:, None]

    # ------------------------------------------------------------------ FDTD
    def _item(self, eps):
        from .core.coeffs import build_tm_coeffs
        from .core.monitors import DFTFieldsMonitor
        from .core.stepper_tm import init_tm_state
        m = build_tm_coeffs(self.grid, eps_inf=eps, npml=self.c["npml"])
        mon = DFTFieldsMonitor(self.grid, list(self.c["freqs"]), "Ez")
        return (init_tm_state(self.grid), m, self.source, [mon])

    def simulate(self, rho: torch.Tensor, batch: int = 1024) -> torch.Tensor:
        """FDTD of each design: (B, d, d) -> (B, 6, region, region) = (Re, Im) of the Ez
        DFT at each frequency on the region. One plan per batch size is built once and
        kept; later batches only repack eps (Engine2D.set_eps) and reset."""
        nf, r = len(self.c["freqs"]), self.c["region"]
        outs = []
        with torch.no_grad():
            for b0 in range(0, rho.shape[0], batch):
                eps = self.eps_map(rho[b0:b0 + batch].to(self.device))
                eng = self._engine(eps)
                eng.run(0, self.c["steps"])
                acc = torch.stack([eng.accumulators(b)[0] for b in range(eps.shape[0])])
                outs.append(self.region(acc).reshape(acc.shape[0], 2 * nf, r, r))
        return torch.cat(outs)

    def _engine(self, eps):
        from .engine2d import Engine2D
        if not hasattr(self, "_engines"):
            self._engines = {}
        n = eps.shape[0]
        eng = self._engines.get(n)
        if eng is None:
            eng = self._engines[n] = Engine2D([self._item(e) for e in eps])
        else:
            for b in range(n):
                eng.set_eps(b, eps[b])
            eng.reset()
        return eng

    def plan(self, n: int):
        """The Engine2D kept for batches of ``n`` designs (None before the first)."""
        return getattr(self, "_engines", {}).get(n)

    def close(self):
        for eng in getattr(self, "_engines", {}).values():
            eng.close()
        self._engines = {}

    def fdtd_fom_and_grad(self, rho: torch.Tensor, fields: bool = False):
        """(FOM, dFOM/drho) of one design by the library's adjoint (run_tm with eps
        requiring grad); with ``fields`` also its (1, 6, region, region) DFT fields."""
        from .core.run import run_tm
        rho = rho.detach().clone().requires_grad_(True)
        eps = self.eps_map(rho[None])[0]
        st, m, src, mons = self._item(eps)
        _, (acc,) = run_tm(st, m, self.c["steps"], source=src, monitors=mons,
                           checkpoint_every=64)
        nf = len(self.c["freqs"])
        y = self.region(acc).reshape(1, 2 * nf, self.c["region"], self.c["region"])
        f = self.fom(y)[0]
        f.backward()
        if fields:
            return float(f.detach()), rho.grad.detach(), y.detach()
        return float(f.detach()), rho.grad.detach()

    def fom(self, fields: torch.Tensor) -> torch.Tensor:
        """Mean |Ez|^2 over the target patch and the frequencies: (B, 6, r, r) -> (B,)."""
        i0, i1, j0, j1 = self.c["target"]
        r0 = self.r0
        patch = fields[:, :, i0 - r0:i1 - r0, j0 - r0:j1 - r0]
        re, im = patch[:, 0::2], patch[:, 1::2]
        return (re * re + im * im).mean(dim=(1, 2, 3))


class _SpectralConv(nn.Module):
    """Complex channel mix of the ``modes`` x ``modes`` lowest modes in the two
    positive-frequency corners of rfft2."""

    def __init__(self, width: int, modes: int):
        super().__init__()
        self.modes = modes
        scale = 1.0 / (width * width)
        self.w = nn.Parameter(scale * torch.randn(2, width, width, modes, modes,
                                                  dtype=torch.cfloat))

    def forward(self, x):
        b, c, h, w = x.shape
        m = self.modes
        xf = torch.fft.rfft2(x.float())
        out = torch.zeros(b, c, h, w // 2 + 1, dtype=torch.cfloat, device=x.device)
        out[:, :, :m, :m] = torch.einsum("bixy,ioxy->boxy", xf[:, :, :m, :m], self.w[0])
        out[:, :, -m:, :m] = torch.einsum("bixy,ioxy->boxy", xf[:, :, -m:, :m], self.w[1])
        return torch.fft.irfft2(out, s=(h, w))


class _ChannelMix(torch.autograd.Function):
    """y = act(W x + b + s) over NCHW pixels on the library's tcgen05 kernels (BF16
    operands, FP32 accumulation): mtb_fno_mix forward; mtb_fno_mix_dx (dz = dy *
    GELU'(z), dx = W^T dz) and mtb_fno_mix_dw (dW = dz x^T) backward; db and ds are
    sums / copies of dz."""

    @staticmethod
    def forward(ctx, x, weight, bias, s, act):
        from . import _lib as L
        lib = L.load()
        bsz, cin, h, w = x.shape
        cout = weight.shape[0]
        x = x.contiguous().float()
        w2 = weight.reshape(cout, cin).contiguous().float()
        b = bias.contiguous().float() if bias is not None else None
        sv = s.contiguous().float() if s is not None else None
        y = torch.empty(bsz, cout, h, w, device=x.device, dtype=torch.float32)
        z = torch.empty_like(y) if act else None
        st = torch.cuda.current_stream(x.device).cuda_stream
        L.check(lib.mtb_fno_mix(L.ptr(x), L.ptr(w2), L.ptr(b) if b is not None else None,
                                L.ptr(sv) if sv is not None else None, L.ptr(y),
                                L.ptr(z) if z is not None else None, bsz, cin, cout, h * w,
                                1 if act else 0, st), "mtb_fno_mix")
        ctx.save_for_backward(x, w2, z)
        ctx.act, ctx.has_b, ctx.has_s = bool(act), bias is not None, s is not None
        ctx.wshape = weight.shape
        return y

    @staticmethod
    def backward(ctx, dy):
        from . import _lib as L
        lib = L.load()
        x, w2, z = ctx.saved_tensors
        bsz, cin, h, w = x.shape
        cout = w2.shape[0]
        dy = dy.contiguous().float()
        dz = torch.empty(bsz, cout, h, w, device=x.device, dtype=torch.float32)
        dx = torch.empty_like(x)
        dw = torch.zeros(cout, cin, device=x.device, dtype=torch.float32)
        st = torch.cuda.current_stream(x.device).cuda_stream
        L.check(lib.mtb_fno_mix_dx(L.ptr(dy), L.ptr(z) if z is not None else None, L.ptr(w2),
                                   L.ptr(dz), L.ptr(dx), bsz, cin, cout, h * w,
                                   1 if ctx.act else 0, st), "mtb_fno_mix_dx")
        L.check(lib.mtb_fno_mix_dw(L.ptr(dz), L.ptr(x), L.ptr(dw), bsz, cin, cout, h * w, st),
                "mtb_fno_mix_dw")
        db = dz.sum(dim=(0, 2, 3)) if ctx.has_b else None
        return dx, dw.reshape(ctx.wshape), db, (dz if ctx.has_s else None), None


def channel_mix(x, weight, bias=None, s=None, act=False):
    """act(W x + b + s) for NCHW x on the tcgen05 channel-mix kernels (CUDA only)."""
    return _ChannelMix.apply(x, weight, bias, s, act)


class FNO2d(nn.Module):
    """Fourier neural operator: (B, 1, r, r) normalised eps -> (B, 6, r, r) fields.

    On CUDA (``native``, the default) the four channel mixes (each fused with the
    spectral branch's sum, the bias and GELU) and the 64 -> 128 projection run on the
    library's tcgen05 kernels; the FFTs and per-mode complex mixes are cuFFT / cuBLAS
    in FP32, the 3 -> 64 lift and 128 -> 6 head plain convolutions. ``native=False``
    runs every layer through torch with BF16 autocast."""

    def __init__(self, width: int = 64, modes: int = 24, layers: int = 4, out_ch: int = 6,
                 native: bool = True):
        super().__init__()
        self.native = native
        self.lift = nn.Conv2d(3, width, 1)
        self.spec = nn.ModuleList([_SpectralConv(width, modes) for _ in range(layers)])
        self.mix = nn.ModuleList([nn.Conv2d(width, width, 1) for _ in range(layers)])
        self.proj1 = nn.Conv2d(width, 128, 1)
        self.proj2 = nn.Conv2d(128, out_ch, 1)

    def forward(self, x):
        b, _, h, w = x.shape
        gy, gx = torch.meshgrid(torch.linspace(0, 1, h, device=x.device),
                                torch.linspace(0, 1, w, device=x.device), indexing="ij")
        x = torch.cat([x, gy.expand(b, 1, h, w), gx.expand(b, 1, h, w)], dim=1)
        if self.native and x.is_cuda:
            x = self.lift(x)
            n = len(self.spec)
            for k, (s, m) in enumerate(zip(self.spec, self.mix)):
                x = channel_mix(x, m.weight, m.bias, s(x), act=k < n - 1)
            x = channel_mix(x, self.proj1.weight, self.proj1.bias, None, act=True)
            return self.proj2(x)
        with torch.autocast("cuda", dtype=torch.bfloat16, enabled=x.is_cuda):
            x = self.lift(x)
            for k, (s, m) in enumerate(zip(self.spec, self.mix)):
                y = s(x) + m(x)
                x = F.gelu(y) if k < len(self.spec) - 1 else y
            x = self.proj2(F.gelu(self.proj1(x)))
        return x.float()


def shard_range(n: int, rank: int, world: int) -> tuple:
    """Contiguous [start, stop) of n designs owned by ``rank`` of ``world``; shard sizes
    differ by at most one. Data generation runs each shard on its own rank with no
    collective (the designs are independent)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} of world {world}")
    base, extra = divmod(n, world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def _dist(group):
    """(torch.distributed, world size) when a process group is up, else (None, 1)."""
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return None, 1
    return dist, dist.get_world_size(group)


def _real_views(ts):
    return [torch.view_as_real(t) if t.is_complex() else t for t in ts]


def _allreduce_mean_grads(params, dist, group, world):
    """Mean of every parameter gradient over the ranks, through one flat buffer
    (complex gradients travel as their real and imaginary parts)."""
    for p in params:
        if p.grad is None:
            p.grad = torch.zeros_like(p)
    views = _real_views([p.grad for p in params])
    flat = torch.cat([v.reshape(-1) for v in views])
    dist.all_reduce(flat, group=group)
    flat /= world
    off = 0
    for v in views:
        v.copy_(flat[off:off + v.numel()].view_as(v))
        off += v.numel()


def train_fno(model: FNO2d, x: torch.Tensor, y: torch.Tensor, *, epochs: int = 30,
              batch: int = 32, lr: float = 2e-3, scale: float | None = None, log=None,
              group=None):
    """Adam + cosine schedule on the relative L2 error of the (scaled) fields. Returns
    (scale, seconds): targets are divided by ``scale`` (their RMS unless given).

    Under torch.distributed (a process group is initialised) the training is data-parallel:
    x, y are this rank's shard, ``batch`` is per rank, rank 0's parameters are broadcast
    first, every step all-reduces the mean gradient (one flat buffer), the RMS scale is
    global, and every rank takes the smallest shard's number of steps per epoch."""
    dist, world = _dist(group)
    params = list(model.parameters())
    if world > 1:
        for v in _real_views([p.data for p in params]):
            dist.broadcast(v, 0, group=group)
    if scale is None:
        ss = torch.tensor([float(y.pow(2).sum(dtype=torch.float64)), float(y.numel())],
                          dtype=torch.float64, device=y.device)
        if world > 1:
            dist.all_reduce(ss, group=group)
        scale = float((ss[0] / ss[1]).sqrt())
    spe = max(1, x.shape[0] // batch)
    if world > 1:
        n = torch.tensor([spe], dtype=torch.int64, device=y.device)
        dist.all_reduce(n, op=dist.ReduceOp.MIN, group=group)
        spe = int(n.item())
    yn = y / scale
    opt = torch.optim.Adam(params, lr=lr)
    sched = torch.optim.lr_scheduler.CosineAnnealingLR(opt, epochs * spe)
    g = torch.Generator(device="cpu").manual_seed(0)
    t0 = time.perf_counter()
    for ep in range(epochs):
        perm = torch.randperm(x.shape[0], generator=g)
        tot = 0.0
        for k in range(spe):
            idx = perm[k * batch:(k + 1) * batch].to(x.device)
            pred = model(x[idx])
            t = yn[idx]
            loss = ((pred - t).flatten(1).norm(dim=1) / t.flatten(1).norm(dim=1)).mean()
            opt.zero_grad(set_to_none=True)
            loss.backward()
            if world > 1:
                _allreduce_mean_grads(params, dist, group, world)
            opt.step()
            sched.step()
            tot += float(loss.detach())
        if log is not None:
            log(ep, tot / spe)
    if x.is_cuda:
        torch.cuda.synchronize(x.device)
    return scale, time.perf_counter() - t0


def rel_error(model: FNO2d, x: torch.Tensor, y: torch.Tensor, scale: float) -> float:
    with torch.no_grad():
        p = torch.cat([model(x[i:i + 64]) for i in range(0, x.shape[0], 64)]) * scale
    return float(((p - y).flatten(1).norm(dim=1) / y.flatten(1).norm(dim=1)).mean())


def design_loop(prob: Cfg5Problem, rho0: torch.Tensor, iters: int, *, model=None,
                scale: float = 1.0, lr: float = 0.05, inner: int = 40, inner_lr: float = 0.1,
                radius: float = 1.0, probes=(5, 10, 20, 40), finetune: int = 0,
                ft_lr: float = 2e-4, replay=None, grad_every: int = 1,
                target: float | None = None):
    """Gradient ascent on the design latent z (rho = sigmoid(z)) from ``rho0``.

    Without ``model`` (the plain loop): ``iters`` Adam steps (``lr``), each on the FOM
    and gradient of one FDTD run with its adjoint.

    With ``model``: a first-order-corrected trust-region loop (surrogate management
    after Alexandrov, Dennis, Lewis and Torczon, 1998) of at most ``iters`` blocks. At
    an anchor z_k the FDTD adjoint gives f_k and g_k = dFOM/drho. The surrogate s(rho)
    is shifted to agree with FDTD in value and gradient there, m(rho) = s(rho) +
    (f_k - s_k) + (g_k - grad s_k) . (rho - rho_k). ``inner`` surrogate Adam steps
    (``inner_lr``) maximise m with z kept within ``radius`` of z_k (max norm); the
    designs after each count in ``probes`` are verified together by one batched
    forward FDTD run. The best verified probe becomes the next anchor if it beats f_k;
    every ``grad_every``-th new anchor gets an adjoint run, the others keep the last
    adjoint anchor's gradient correction g - grad s with the value correction taken
    from the verified FOM. The radius doubles when the accepted probe is the last one
    and halves when no probe beats f_k. With ``finetune`` > 0 the model then takes that
    many Adam steps (``ft_lr``) on the verified fields of this loop, mixed with
    samples of ``replay`` = (inputs, targets / scale) when given. The loop stops
    once a verified FOM reaches ``target``. Only FDTD FOMs are reported.

    Returns dict(fom=[verified FOM of each anchor / best probe], t=[seconds at each],
    accepted=[bool], seconds, surrogate_steps, fdtd_runs (adjoint runs plus batched
    forward runs), adjoint_runs, rho)."""
    dev = prob.device
    z = torch.logit(rho0.clamp(0.02, 0.98)).detach().clone().to(dev)
    hist, times, acc = [], [], []
    t0 = time.perf_counter()
    n_adj = n_fwd = n_sur = 0

    def mark(f, ok):
        hist.append(f)
        times.append(time.perf_counter() - t0)
        acc.append(ok)

    if model is None:
        z.requires_grad_(True)
        opt = torch.optim.Adam([z], lr=lr)
        for _ in range(iters):
            rho = torch.sigmoid(z).detach()
            f, g = prob.fdtd_fom_and_grad(rho)
            n_adj += 1
            mark(f, True)
            if target is not None and f >= target:
                break
            opt.zero_grad(set_to_none=True)
            z.grad = -(g * rho * (1 - rho))          # d(-FOM)/dz
            opt.step()
    else:
        probes = sorted(set(int(p) for p in probes if 0 < int(p) <= inner)) or [inner]
        params = list(model.parameters())
        trainable = [p.requires_grad for p in params]
        ft_opt = torch.optim.Adam([p for p, t in zip(params, trainable) if t], lr=ft_lr) \
            if finetune else None
        mem_x, mem_y = [], []
        gen = torch.Generator(device="cpu").manual_seed(0)

        def freeze(on):
            for p, t in zip(params, trainable):
                p.requires_grad_(t and not on)

        freeze(True)
        f_k, g_k, y_k = prob.fdtd_fom_and_grad(torch.sigmoid(z), fields=True)
        n_adj += 1
        mark(f_k, True)
        mem_x.append(prob.fno_input(torch.sigmoid(z)[None]))
        mem_y.append(y_k / scale)
        n_acc = 0
        cg = None
        for _ in range(iters - 1):
            if target is not None and f_k >= target:
                break
            rho_k = torch.sigmoid(z).detach()
            r = rho_k.clone().requires_grad_(True)
            s_k = prob.fom(model(prob.fno_input(r[None])) * scale)[0]
            if g_k is not None or cg is None:
                (gs_k,) = torch.autograd.grad(s_k, r)
                cg = g_k - gs_k
            c0 = f_k - float(s_k.detach())
            zc = z.clone().requires_grad_(True)
            opt = torch.optim.Adam([zc], lr=inner_lr)
            cand = []
            for j in range(1, probes[-1] + 1):
                rho = torch.sigmoid(zc)
                m = prob.fom(model(prob.fno_input(rho[None])) * scale)[0] + c0 + \
                    (cg * (rho - rho_k)).sum()
                opt.zero_grad(set_to_none=True)
                (-m).backward()
                opt.step()
                with torch.no_grad():
                    zc.copy_(torch.minimum(torch.maximum(zc, z - radius), z + radius))
                n_sur += 1
                if j in probes:
                    cand.append(zc.detach().clone())
            rhos = torch.sigmoid(torch.stack(cand))
            y = prob.simulate(rhos, batch=len(cand))
            n_fwd += 1
            fc = prob.fom(y)
            best = int(torch.argmax(fc))
            ok = float(fc[best]) > f_k
            if finetune:
                mem_x.append(prob.fno_input(rhos))
                mem_y.append(y / scale)
            if ok:
                if best == len(cand) - 1:
                    radius = min(2.0 * radius, 8.0)
                z = cand[best]
                n_acc += 1
                if n_acc % max(1, grad_every) == 0:
                    f_k, g_k = prob.fdtd_fom_and_grad(torch.sigmoid(z))
                    n_adj += 1
                else:
                    f_k, g_k = float(fc[best]), None
            else:
                radius *= 0.5
            mark(f_k if ok else float(fc[best]), ok)
            if finetune:
                freeze(False)
                xs, ys = torch.cat(mem_x), torch.cat(mem_y)
                for _ in range(finetune):
                    bx, by = xs, ys
                    if replay is not None:
                        idx = torch.randint(0, replay[0].shape[0], (16,), generator=gen)
                        idx = idx.to(replay[0].device)
                        bx = torch.cat([xs[-16:], replay[0][idx]])
                        by = torch.cat([ys[-16:], replay[1][idx]])
                    pred = model(bx)
                    loss = ((pred - by).flatten(1).norm(dim=1) /
                            by.flatten(1).norm(dim=1)).mean()
                    ft_opt.zero_grad(set_to_none=True)
                    loss.backward()
                    ft_opt.step()
                freeze(True)
        freeze(False)
    if dev.type == "cuda":
        torch.cuda.synchronize(dev)
    return dict(fom=hist, t=times, accepted=acc, seconds=time.perf_counter() - t0,
                surrogate_steps=n_sur, fdtd_runs=n_adj + n_fwd, adjoint_runs=n_adj,
                rho=torch.sigmoid(z).detach())
