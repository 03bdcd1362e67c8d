#!/usr/bin/env python
"""Benchmark of the B200 FDTD hot path (one JSON line on rank 0).

Workload (default ``cfg2``): 256 batched 2D TE/TM bend variants, grids
uniform in 256^2..768^2, resolution 20, 1 um CPML, Gaussian line source,
full-grid DFT of Ez/Hz at 3 frequencies plus 2 flux lines, 5000 time steps.
One bench step = one whole run of that batch (reset to t = 0, 5000 steps,
every DFT contribution folded). Metric: Gcell-updates/s = sum(nx*ny) *
5000 / s over all ranks.

* ``value``: inputs resident in HBM (engine built once, reset per step).
* ``e2e``: the public API from host buffers: pinned eps maps copied in,
  coefficients / sources / monitors / states built on the GPU, the run, and
  the DFT + flux accumulators copied back -- all inside the timed region.
* ``roofline``: the step kernels of one time step (cfg2: k_tile_tm + k_tile_te),
  CUDA-event time per step on the plan's stream over the timed region, against
  algorithmic bytes per step (fields + eps + CPML layers; the DFT ring and
  contraction are reported separately); ``achieved_raw`` / ``frac_raw`` use the
  measured DRAM bytes (``traffic``) instead.
* ``--workload cfg1 | cfg3 | cfg4``: the single-structure TM run, the 256^3 3D
  run and the 600 x 400 gradient problem, on the same line format.
* ``--workload cfg5``: the surrogate-assisted design loop. FDTD data generation and
  FNO training come first (untimed). Then the plain adjoint loop and the surrogate
  loop run from the same start. ``value`` is the plain loop's iteration count over
  the surrogate loop's wall time to reach 99 % of the plain loop's final FOM, with
  both FOMs verified by FDTD. Each bench step is one pair of loops.
* ``cpu_baseline``: the oracle (numpy restatement of the reference's TM/TE
  step and monitors) on a bounded sample of the same batch, on the host cores.
* ``--impl reference``: the same sample through the oracle only (the
  reference is a Python/torch package that cannot be installed on the GPU
  box; the oracle is its restatement, pinned against it by the golden tests).
Multi-GPU (torchrun): every rank advances its own 256-structure batch
(seed 2 + 1009*rank), no collective in the data path: weak scaling.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

STEPS_PER_RUN = {"cfg2": 5000, "cfg3": 2000, "cfg1": 4000}
S_CFG5_STEPS = 3000
CFG5_METRIC = ("design-iterations/s (plain-loop iterations matched per second of the surrogate "
               "loop, at <= 1% FOM error)")


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class Clocks:
    """nvidia-smi sampler running during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={self.index}",
                                       f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                       "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None
        return self

    def __exit__(self, *a):
        if self.p is not None:
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.p.kill()

    def summary(self):
        try:
            rows = [r.split(",") for r in open(self.f.name).read().strip().splitlines()]
        except OSError:
            rows = []
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            r = [x.strip() for x in r]
            if len(r) < 9:
                continue
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
            except ValueError:
                continue
            for n, v in zip(names, r[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        os.unlink(self.f.name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ------------------------------------------------------------------ CPU sample

def cpu_sample(specs, steps, threads):
    """Oracle run of `steps` steps on every spec (threads over structures).
    Returns (cell-updates, seconds)."""
    import numpy as np

    from meep_torch_b200 import workloads as W
    from oracle import fdtd as O

    def one(spec):
        nx, ny, eps = spec["nx"], spec["ny"], spec["eps"]
        f32 = np.float32
        prof = O.gaussian_pulse(0.65, 0.2)
        mask = O.line_source_mask(nx, ny, W.DX2D, spec["src_ix"], *spec["src_j"], dtype=f32)
        freqs = W.CFG2_FREQS
        fx, fy = spec["flux_x"], spec["flux_y"]
        if spec["pol"] == "tm":
            c = O.tm_coeffs(nx, ny, W.DX2D, eps=eps, npml=W.NPML2D, dtype=f32)
            dt = c["dt"]
            mons = [lambda s, t: O.dft_sample(s["Ez"], t, dt, freqs, "Ez", f32),
                    lambda s, t: O.flux_tm_sample(s, t, dt, freqs, True, *fx, f32),
                    lambda s, t: O.flux_tm_sample(s, t, dt, freqs, False, *fy, f32)]
            step, s0 = O.tm_step, O.tm_state(c)
        else:
            c = O.te_coeffs(nx, ny, W.DX2D, eps=eps, npml=W.NPML2D, dtype=f32)
            dt = c["dt"]
            mask = mask[:, :-1]
            mons = [lambda s, t: O.dft_sample(s["Hz"], t, dt, freqs, "Hz", f32),
                    lambda s, t: O.flux_te_sample(s, t, dt, freqs, *fx, f32),
                    lambda s, t: O.flux_tey_sample(s, t, dt, freqs, *fy, f32)]
            step, s0 = O.te_step, O.te_state(c)
        O.run_2d(step, s0, c, steps, amp_fn=lambda t: prof(O.src_time(t, dt)), mask=mask,
                 monitors=mons)
        return nx * ny * steps

    t0 = time.perf_counter()
    with cf.ThreadPoolExecutor(max_workers=threads) as ex:
        cells = sum(ex.map(one, specs))
    return cells, time.perf_counter() - t0


def cpu_baseline_line(n_struct, steps, threads):
    from meep_torch_b200 import workloads as W
    specs = W.cfg2_specs()[:n_struct]
    cells, sec = cpu_sample(specs, steps, threads)
    return {"value": cells / sec / 1e9, "unit": "Gcell-updates/s", "cores": threads,
            "kind": "port",
            "sample": f"oracle (numpy float32) on cfg2 structures 0..{n_struct - 1} x {steps} "
                      f"steps, {threads} threads over structures, {sec:.1f} s"}


def cpu_sample_cfg1(steps):
    """Oracle run of `steps` steps of cfg1 (one thread). Returns (cell-updates, seconds)."""
    import numpy as np

    from meep_torch_b200 import workloads as W
    from oracle import fdtd as O
    spec = W.cfg1_spec()
    nx, ny, f32 = spec["nx"], spec["ny"], np.float32
    c = O.tm_coeffs(nx, ny, W.DX2D, eps=spec["eps"], npml=W.NPML2D, dtype=f32)
    dt = c["dt"]
    i, j = spec["src"]
    mask = O.line_source_mask(nx, ny, W.DX2D, i, j, j + 1, dtype=f32)
    prof = O.gaussian_pulse(0.15, 0.1)
    ix, lo, hi = spec["flux"]
    mons = [lambda s, t: O.flux_tm_sample(s, t, dt, spec["freqs"], True, ix, lo, hi, f32)]
    t0 = time.perf_counter()
    O.run_2d(O.tm_step, O.tm_state(c), c, steps, amp_fn=lambda t: prof(O.src_time(t, dt)),
             mask=mask, monitors=mons)
    return nx * ny * steps, time.perf_counter() - t0


def cpu_sample_cfg3(steps, n=256):
    """Oracle run of `steps` steps of the cfg3 grid (n^3, spheres, point source, six flux
    faces), one thread. Returns (cell-updates, seconds)."""
    import numpy as np

    from meep_torch_b200 import workloads as W
    from oracle import fdtd as O
    f32 = np.float32
    c = O.coeffs_3d(n, n, n, 1.0 / 16, eps=W.cfg3_eps(n), npml=16, dtype=f32)
    dt = c["dt"]
    prof = O.gaussian_pulse(0.5, 0.3)
    freqs = np.linspace(0.35, 0.65, 20)
    lo_, hi_ = 24 * n // 256, 232 * n // 256
    mons = [(lambda a, i: (lambda st, t: O.flux3d_sample(st, t, dt, freqs, a, i,
                                                         win=(lo_, hi_, lo_, hi_))))(
        a, lo_ if i == 24 else hi_) for a, i in W.CFG3_FACES]
    t0 = time.perf_counter()
    O.run_3d(O.state_3d(c), c, steps, amp_fn=lambda t: prof(O.src_time(t, dt)),
             src=("Ez", n // 2, n // 2, n // 2), monitors=mons)
    return n ** 3 * steps, time.perf_counter() - t0


# ------------------------------------------------------------------ GPU bench

def run_cfg4(args, rank, world, dev):
    """cfg4: gradient evaluations (design chain + 8000-step TM run + adjoint sweep)."""
    import torch

    from meep_torch_b200 import _lib
    from meep_torch_b200 import workloads as W

    lib = _lib.load()
    steps = args.run_steps if args.run_steps != 5000 else W.CFG4["steps"]
    opt, n = W.cfg4_setup(dev, seed=4 + 1009 * rank, steps=steps)
    stream = torch.cuda.current_stream(dev)
    for _ in range(args.warmup):
        opt()
    torch.cuda.synchronize(dev)
    barrier(world)
    n0 = lib.mtb_launch_count()
    with Clocks(dev.index if dev.index is not None else 0) as clk:
        torch.cuda.synchronize(dev)
        barrier(world)
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        for _ in range(args.steps):
            opt()
        ev1.record(stream)
        torch.cuda.synchronize(dev)
        barrier(world)
    launches = lib.mtb_launch_count() - n0
    ms = ev0.elapsed_time(ev1)
    c = W.CFG4
    res = dict(cells=c["nx"] * c["ny"], nsteps=n, ms=allreduce_max(ms, world, dev),
               launches=launches, clocks=clk.summary(), grad_evals=args.steps * world)
    if args.no_e2e:
        res.update(e2e_s=float("nan"), h2d=0, d2h=0)
        return res
    host_rho = opt.rho.detach().cpu().pin_memory()
    torch.cuda.synchronize(dev)
    barrier(world)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        opt.rho = host_rho.to(dev, non_blocking=True)
        _, grad = opt()                              # dJ/drho comes back as numpy
    torch.cuda.synchronize(dev)
    res.update(e2e_s=allreduce_max(time.perf_counter() - t0, world, dev),
               h2d=host_rho.numel() * 4, d2h=grad.size * 4)
    return res


def cpu_sample_cfg4(steps):
    """Oracle forward of `steps` steps on the cfg4 grid (one thread)."""
    import numpy as np

    from meep_torch_b200 import workloads as W
    from oracle import fdtd as O
    c = W.CFG4
    nx, ny, dx = c["nx"], c["ny"], c["dx"]
    eps = np.full((nx, ny), c["eps_bg"], dtype=np.float32)
    eps[:, ny // 2 - 10: ny // 2 + 10] = c["eps_core"]
    oc = O.tm_coeffs(nx, ny, dx, eps=eps, npml=c["npml"], dtype=np.float32)
    dt = oc["dt"]
    mask = O.line_source_mask(nx, ny, dx, c["npml"] + 10, ny // 2 - 20, ny // 2 + 20,
                              dtype=np.float32)
    prof = O.gaussian_pulse(0.645, 0.12)
    t0 = time.perf_counter()
    O.run_2d(O.tm_step, O.tm_state(oc), oc, steps, amp_fn=lambda t: prof(O.src_time(t, dt)),
             mask=mask)
    return time.perf_counter() - t0


def run_cfg5(args, rank, world, dev):
    """cfg5: FDTD data generation, FNO training, then the plain adjoint design loop and
    the surrogate-assisted loop from the same start; the surrogate loop stops once its
    FDTD-verified FOM reaches 99 % of the plain loop's final FOM."""
    import torch

    from meep_torch_b200 import _lib
    from meep_torch_b200 import surrogate as S
    from meep_torch_b200 import workloads as W

    lib = _lib.load()
    torch.manual_seed(5 + 1009 * rank)
    prob = S.Cfg5Problem(dev)
    c = prob.c
    n_train, n_test = args.maps, 256
    rho = S.grf_designs(n_train + n_test, seed=5 + 1009 * rank, soft=0.5).to(dev)
    batch = min(1024, n_train)
    # data generation: one plan of `batch` designs, eps repacked per chunk
    prob.simulate(rho[:batch], batch=batch)                       # plan build + warm-up
    eng = prob.plan(batch)
    eng.set_timing(True)
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    y = prob.simulate(rho, batch=batch)
    torch.cuda.synchronize(dev)
    gen_s = time.perf_counter() - t0
    step_ms, step_n, dft_ms, dft_n = eng.timing()
    eng.set_timing(False)
    prob.close()
    x = prob.fno_input(rho)
    model = S.FNO2d().to(dev)
    scale, train_s = S.train_fno(model, x[:n_train], y[:n_train], epochs=args.epochs)
    model.eval()
    test_err = S.rel_error(model, x[n_train:], y[n_train:], scale)
    with torch.no_grad():
        fp = torch.cat([model(x[n_train + i:n_train + i + 64]) for i in range(0, n_test, 64)])
        ft = prob.fom(y[n_train:])
        fom_err = float(((prob.fom(fp * scale) - ft).abs() / ft).median())
    replay = (x[:n_train], y[:n_train] / scale)
    del y
    rho0 = torch.full((c["design"], c["design"]), 0.5)
    import copy
    for _ in range(args.warmup):                                   # plans, cuFFT, autotune
        S.design_loop(prob, rho0.to(dev), 2)
        S.design_loop(prob, rho0.to(dev), 2, model=copy.deepcopy(model), scale=scale,
                      **CFG5_LOOP, replay=replay)
    torch.cuda.synchronize(dev)
    n0 = lib.mtb_launch_count()
    runs = []
    with Clocks(dev.index if dev.index is not None else 0) as clk:
        for _ in range(args.steps):
            plain = S.design_loop(prob, rho0.to(dev), args.iters)
            target = 0.99 * plain["fom"][-1]
            sur = S.design_loop(prob, rho0.to(dev), 2 * args.iters,
                                model=copy.deepcopy(model), scale=scale, **CFG5_LOOP,
                                replay=replay, target=target)
            runs.append((plain, sur, target))
    launches = lib.mtb_launch_count() - n0
    plain, sur, target = runs[len(runs) // 2]
    # e2e: the surrogate loop from a pinned host design to the final design on the host
    host = rho0.pin_memory()
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    out = S.design_loop(prob, host.to(dev, non_blocking=True), 2 * args.iters,
                        model=copy.deepcopy(model), scale=scale, **CFG5_LOOP, replay=replay,
                        target=target)
    final = out["rho"].cpu()
    e2e_s = time.perf_counter() - t0
    spec = [{"nx": c["n"], "ny": c["n"], "pol": "tm"}] * batch
    return dict(plain=plain, sur=sur, target=target, e2e_s=e2e_s, e2e_reached=
                out["fom"][-1] >= target, h2d=host.numel() * 4, d2h=final.numel() * 4,
                gen_s=gen_s, gen_updates=(n_train + n_test) * c["n"] ** 2 * c["steps"],
                step_ms=step_ms, step_n=step_n, dft_ms=dft_ms,
                bytes_launch=W.cfg2_bytes_per_step(spec, c["npml"]), train_s=train_s,
                test_err=test_err, fom_err=fom_err, launches=launches,
                clocks=clk.summary(), n_train=n_train)


# surrogate-loop settings (chosen by a sweep of inner steps, probe sets, fine-tuning and
# adjoint frequency on this problem)
CFG5_LOOP = dict(inner=20, inner_lr=0.2, radius=2.0, probes=(2, 5, 10, 15, 20), finetune=2,
                 grad_every=1)


def cpu_sample_cfg5(steps):
    """Oracle TM forward of `steps` steps on the cfg5 grid (one thread): seconds."""
    import numpy as np

    from meep_torch_b200 import surrogate as S
    from oracle import fdtd as O
    c = S.CFG5
    n = c["n"]
    rho = S.grf_designs(1, seed=5)[0].numpy()
    eps = np.full((n, n), c["eps_min"], dtype=np.float32)
    d0 = (n - c["design"]) // 2
    eps[d0:d0 + c["design"], d0:d0 + c["design"]] = c["eps_min"] + \
        (c["eps_max"] - c["eps_min"]) * rho
    oc = O.tm_coeffs(n, n, c["dx"], eps=eps, npml=c["npml"], dtype=np.float32)
    dt = oc["dt"]
    mask = O.line_source_mask(n, n, c["dx"], c["npml"] + 10, c["npml"], n - c["npml"],
                              dtype=np.float32)
    prof = O.gaussian_pulse(c["fcen"], c["fwidth"])
    freqs = list(c["freqs"])
    mons = [lambda s, t: O.dft_sample(s["Ez"], t, dt, freqs, "Ez", np.float32)]
    t0 = time.perf_counter()
    O.run_2d(O.tm_step, O.tm_state(oc), oc, steps, amp_fn=lambda t: prof(O.src_time(t, dt)),
             mask=mask, monitors=mons)
    return time.perf_counter() - t0


def run_cfg1(args, rank, world, dev):
    """cfg1: one 320 x 160 TM structure per rank, 4000 steps per run. The working
    set is L2-resident and the step is launch/latency-bound: whole ring flushes
    are replayed as CUDA graphs (per-launch timing stays off)."""
    import torch

    from meep_torch_b200 import _lib
    from meep_torch_b200 import workloads as W
    from meep_torch_b200.core.run import run_tm
    from meep_torch_b200.engine2d import Engine2D

    lib = _lib.load()
    spec = W.cfg1_spec()
    nsteps = args.run_steps if args.run_steps != 5000 else spec["steps"]
    eng = Engine2D([W.cfg1_item(dev, spec)], rows_per_warp=args.rows, ring_slots=args.ring,
                   variant=args.variant)
    stream = torch.cuda.current_stream(dev)

    def bench_step():
        eng.reset()
        eng.run(0, nsteps)

    for _ in range(args.warmup):
        bench_step()
    torch.cuda.synchronize(dev)
    barrier(world)
    n0 = lib.mtb_launch_count()
    with Clocks(dev.index if dev.index is not None else 0) as clk:
        torch.cuda.synchronize(dev)
        barrier(world)
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        for _ in range(args.steps):
            bench_step()
        ev1.record(stream)
        torch.cuda.synchronize(dev)
        barrier(world)
    launches = lib.mtb_launch_count() - n0
    ms = ev0.elapsed_time(ev1)
    eng.close()
    cells = spec["nx"] * spec["ny"]
    spec2 = dict(spec, pol="tm")
    per_step_ms = ms / (args.steps * nsteps)
    res = dict(cells=cells, nsteps=nsteps, ms=allreduce_max(ms, world, dev), launches=launches,
               clocks=clk.summary(), step_ms=per_step_ms * args.steps * nsteps,
               step_n=args.steps * nsteps, dft_ms=0.0, dft_n=0,
               bytes_launch=W.cfg2_bytes_per_step([spec2]), e2e_s=float("nan"), h2d=0, d2h=0)
    if args.no_e2e:
        return res
    # ---- e2e: host eps through run_tm, flux accumulator back
    host_eps = torch.from_numpy(spec["eps"]).pin_memory()

    def e2e_step():
        e = host_eps.to(dev, non_blocking=True)
        st, m, src, mons = W.cfg1_item(dev, spec, eps_t=e)
        _, accs = run_tm(st, m, nsteps, source=src, monitors=mons)
        out = [a.to("cpu", non_blocking=True) for a in accs]
        torch.cuda.synchronize(dev)
        return out, sum(a.numel() * 4 for a in accs)

    e2e_step()
    torch.cuda.synchronize(dev)
    barrier(world)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        _, d2h = e2e_step()
    torch.cuda.synchronize(dev)
    res.update(e2e_s=allreduce_max(time.perf_counter() - t0, world, dev),
               h2d=host_eps.numel() * 4, d2h=d2h)
    return res


def run_cfg2(args, rank, world, dev):
    import numpy as np
    import torch

    from meep_torch_b200 import _lib
    from meep_torch_b200 import workloads as W
    from meep_torch_b200.engine2d import Engine2D

    lib = _lib.load()
    nsteps = args.run_steps
    fixed = args.shard == "fixed"
    if fixed:       # one batch split across the ranks (LPT on cells): strong scaling
        from meep_torch_b200.shard import lpt_partition
        all_specs = W.cfg2_specs(n=args.structs, seed=2)
        costs = [s["nx"] * s["ny"] for s in all_specs]
        parts = lpt_partition(costs, world)
        specs = [all_specs[i] for i in parts[rank]]
    else:           # every rank its own batch: weak scaling
        specs = W.cfg2_specs(n=args.structs, seed=2 + 1009 * rank)
    cells = sum(s["nx"] * s["ny"] for s in specs)
    items = [W.cfg2_item(s, dev) for s in specs]
    eng = Engine2D(items, rows_per_warp=args.rows, ring_slots=args.ring, variant=args.variant)
    stream = torch.cuda.current_stream(dev)

    def bench_step():
        eng.reset()
        eng.run(0, nsteps)

    for _ in range(args.warmup):
        bench_step()
    torch.cuda.synchronize(dev)
    eng.set_timing(True)
    barrier(world)
    n0 = lib.mtb_launch_count()
    with Clocks(dev.index if dev.index is not None else 0) as clk:
        torch.cuda.synchronize(dev)
        barrier(world)
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        for _ in range(args.steps):
            bench_step()
        ev1.record(stream)
        torch.cuda.synchronize(dev)
        barrier(world)
    launches = lib.mtb_launch_count() - n0
    ms = ev0.elapsed_time(ev1)
    step_ms, step_n, dft_ms, dft_n = eng.timing()
    eng.set_timing(False)
    ms_max = allreduce_max(ms, world, dev)
    clocks = clk.summary()
    bytes_launch = W.cfg2_bytes_per_step(specs)
    res = dict(cells=cells, nsteps=nsteps, ms=ms_max, launches=launches, clocks=clocks,
               step_ms=step_ms, step_n=step_n, dft_ms=dft_ms, dft_n=dft_n,
               timed_steps=nsteps * args.steps, bytes_launch=bytes_launch,
               ring_elems=eng.ring_elems)
    eng.close()
    del eng, items
    torch.cuda.empty_cache()

    if args.no_e2e:
        res.update(e2e_s=float("nan"), h2d=0, d2h=0)
        return res
    # ---- e2e: host buffers through the public API
    host_eps = [torch.from_numpy(s["eps"]).pin_memory() for s in specs]
    h2d = sum(t.numel() * 4 for t in host_eps)
    d2h = 0

    def run_share(idx):
        """Structures idx of this rank's specs: eps in, run, accumulators out."""
        nonlocal d2h
        dev_eps = [host_eps[i].to(dev, non_blocking=True) for i in idx]
        its = [W.cfg2_item(specs[i], dev, eps_t=e) for i, e in zip(idx, dev_eps)]
        e = Engine2D(its, rows_per_warp=args.rows, ring_slots=args.ring, variant=args.variant)
        e.run(0, nsteps)
        outs = []
        nb = 0
        for b in range(len(its)):
            outs.append([a.to("cpu", non_blocking=True) for a in e.accumulators(b)])
            nb += sum(a.numel() * 4 for a in e.accumulators(b))
        torch.cuda.synchronize(dev)
        e.close()
        d2h = nb
        return outs

    def e2e_step():
        if fixed:   # every structure's accumulators end on rank 0, in batch order
            from meep_torch_b200.shard import run_sharded
            local = iter(range(len(specs)))
            return run_sharded(costs, lambda idx: run_share([next(local) for _ in idx]),
                               rank=rank, world=world)
        return run_share(list(range(len(specs))))

    e2e_step()                                   # warm
    torch.cuda.synchronize(dev)
    barrier(world)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        e2e_step()
    torch.cuda.synchronize(dev)
    e2e_s = allreduce_max(time.perf_counter() - t0, world, dev)
    barrier(world)
    res.update(e2e_s=e2e_s, h2d=h2d, d2h=d2h)
    return res


def run_cfg3(args, rank, world, dev):
    """cfg3: one 256^3 structure per rank, 2000 steps per run."""
    import torch

    from meep_torch_b200 import _lib
    from meep_torch_b200 import workloads as W
    from meep_torch_b200.engine3d import Engine3D

    lib = _lib.load()
    n = args.n3
    nsteps = args.run_steps if args.run_steps != 5000 else 2000
    s, c, src, mons = W.cfg3_setup(dev, n=n)
    eng = Engine3D(s, c, src, mons, rows_per_seg=args.rows, ring_slots=args.ring,
                   variant=args.variant, geometry=args.geometry)
    stream = torch.cuda.current_stream(dev)

    def bench_step():
        eng.reset()
        eng.run(0, nsteps)

    for _ in range(args.warmup):
        bench_step()
    torch.cuda.synchronize(dev)
    eng.set_timing(True)
    barrier(world)
    n0 = lib.mtb_launch_count()
    with Clocks(dev.index if dev.index is not None else 0) as clk:
        torch.cuda.synchronize(dev)
        barrier(world)
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        for _ in range(args.steps):
            bench_step()
        ev1.record(stream)
        torch.cuda.synchronize(dev)
        barrier(world)
    launches = lib.mtb_launch_count() - n0
    ms = ev0.elapsed_time(ev1)
    step_ms, step_n, dft_ms, dft_n = eng.timing()
    eng.close()
    res = dict(cells=n ** 3, nsteps=nsteps, ms=allreduce_max(ms, world, dev), launches=launches,
               clocks=clk.summary(), step_ms=step_ms, step_n=step_n, dft_ms=dft_ms,
               dft_n=dft_n, bytes_launch=W.cfg3_bytes_per_step(n), e2e_s=float("nan"), h2d=0,
               d2h=0)
    del eng, s, c, src, mons
    torch.cuda.empty_cache()
    if args.no_e2e:
        return res
    # ---- e2e: host eps through the public API (run_3d), flux accumulators back
    from meep_torch_b200.core.monitors_3d import run_3d
    host_eps = torch.from_numpy(W.cfg3_eps(n)).pin_memory()
    d2h = 0

    def e2e_step():
        nonlocal d2h
        e = host_eps.to(dev, non_blocking=True)
        s_, c_, src_, mons_ = W.cfg3_setup(dev, n=n, eps=e)
        _, accs = run_3d(s_, c_, nsteps, source=src_, monitors=mons_, rows_per_seg=args.rows,
                         ring_slots=args.ring, variant=args.variant)
        outs = [a.to("cpu", non_blocking=True) for a in accs]
        torch.cuda.synchronize(dev)
        d2h = sum(a.numel() * 4 for a in accs)
        return outs

    e2e_step()                                   # warm
    torch.cuda.synchronize(dev)
    barrier(world)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        e2e_step()
    torch.cuda.synchronize(dev)
    res.update(e2e_s=allreduce_max(time.perf_counter() - t0, world, dev),
               h2d=host_eps.numel() * 4, d2h=d2h)
    return res


def run_cfg3_slabs(args, rank, world, dev):
    """cfg3 as one 256^3 grid split along x into ``world`` slabs, one per rank: halo
    planes (Ey, Ez after each E update, Hy, Hz after each H update) travel between
    neighbours over torch.distributed point-to-point (NCCL), flux accumulators are
    summed onto rank 0 at the end. Strong scaling."""
    import torch

    from meep_torch_b200 import _lib
    from meep_torch_b200 import slab3d as SL
    from meep_torch_b200 import workloads as W
    from meep_torch_b200.engine3d import Engine3D

    lib = _lib.load()
    n = args.n3
    nsteps = args.run_steps if args.run_steps != 5000 else 2000
    s, c, src, mons = W.cfg3_setup(dev, n=n)
    sl = SL.slab_bounds(n, world)[rank]
    parts = SL.slice_monitors(mons, sl, n, n)
    eng = Engine3D(SL.slice_state(s, sl), SL.slice_coeffs(c, sl), SL.slice_source(src, sl),
                   [p.monitor for p in parts if p is not None], own=sl.own_local,
                   ring_slots=args.ring)
    del s, c, src
    torch.cuda.empty_cache()
    halo = SL.DistHalo(eng, sl) if world > 1 else SL.LocalHalo([eng], [sl])
    drv = SL.SlabDriver([eng], halo)
    stream = torch.cuda.current_stream(dev)

    def bench_step():
        eng.reset()
        drv.run(0, nsteps)

    for _ in range(args.warmup):
        bench_step()
    torch.cuda.synchronize(dev)
    eng.set_timing(True)
    barrier(world)
    n0 = lib.mtb_launch_count()
    with Clocks(dev.index if dev.index is not None else 0) as clk:
        torch.cuda.synchronize(dev)
        barrier(world)
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        for _ in range(args.steps):
            bench_step()
        ev1.record(stream)
        torch.cuda.synchronize(dev)
        barrier(world)
    launches = lib.mtb_launch_count() - n0
    ms = ev0.elapsed_time(ev1)
    step_ms, step_n, dft_ms, dft_n = eng.timing()
    eng.close()
    own = (sl.x1 - sl.x0) * n * n
    res = dict(cells=own, nsteps=nsteps, ms=allreduce_max(ms, world, dev), launches=launches,
               clocks=clk.summary(), step_ms=step_ms, step_n=step_n, dft_ms=dft_ms,
               dft_n=dft_n, bytes_launch=W.cfg3_bytes_per_step(n) * (sl.x1 - sl.x0) / n,
               e2e_s=float("nan"), h2d=0, d2h=0)
    del eng
    torch.cuda.empty_cache()
    if args.no_e2e:
        return res
    # ---- e2e: host eps through the public API (run_3d_distributed), flux
    # accumulators summed onto rank 0 and read back there
    host_eps = torch.from_numpy(W.cfg3_eps(n)).pin_memory()
    d2h = 0

    def e2e_step():
        nonlocal d2h
        e = host_eps.to(dev, non_blocking=True)
        s_, c_, src_, mons_ = W.cfg3_setup(dev, n=n, eps=e)
        if world > 1:
            _, accs = SL.run_3d_distributed(s_, c_, nsteps, source=src_, monitors=mons_,
                                            rank=rank, world=world, ring_slots=args.ring)
        else:
            _, accs = SL.run_3d_slabs(s_, c_, nsteps, source=src_, monitors=mons_, n_slabs=1,
                                      ring_slots=args.ring)
        outs = [a.to("cpu", non_blocking=True) for a in accs] if accs is not None else []
        torch.cuda.synchronize(dev)
        d2h = sum(a.numel() * 4 for a in outs)
        return outs

    e2e_step()                                   # warm
    torch.cuda.synchronize(dev)
    barrier(world)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        e2e_step()
    torch.cuda.synchronize(dev)
    res.update(e2e_s=allreduce_max(time.perf_counter() - t0, world, dev),
               h2d=host_eps.numel() * 4, d2h=d2h)
    return res


# ------------------------------------------------------------------ reference arm
REF_DIR = os.path.join(ROOT, "baseline", "_ref")


def reference_module():
    """The reference (meep_torch) installed beside the repository by
    baseline/install_reference.py, or None when it is not there."""
    if not os.path.isdir(os.path.join(REF_DIR, "meep_torch")):
        return None
    if REF_DIR not in sys.path:
        sys.path.insert(0, REF_DIR)
    import meep_torch
    return meep_torch


def ref_cfg2(specs, steps):
    """The reference's own run_tm / run_te (core/run.py:125-126) on cfg2 structures:
    its Grid, build_tm_coeffs / build_te_coeffs, LineSource, DFTFieldsMonitor and flux
    monitors, float32, no_grad, all host threads (torch intra-op). Returns
    (cell-updates, seconds); set-up is outside the timed region."""
    import torch
    from meep_torch.core.coeffs import build_te_coeffs, build_tm_coeffs
    from meep_torch.core.grid import Grid
    from meep_torch.core.monitors import (DFTFieldsMonitor, FluxMonitorTE, FluxMonitorTEY,
                                          FluxMonitorTM)
    from meep_torch.core.run import run_te, run_tm
    from meep_torch.core.sources import GaussianPulse, LineSource
    from meep_torch.core.stepper_te import init_te_state
    from meep_torch.core.stepper_tm import init_tm_state

    from meep_torch_b200 import workloads as W
    cells, sec = 0, 0.0
    for spec in specs:
        nx, ny = spec["nx"], spec["ny"]
        g = Grid(nx=nx, ny=ny, dx=W.DX2D, dtype=torch.float32, device="cpu")
        eps = torch.from_numpy(spec["eps"])
        line = LineSource(g, ix=spec["src_ix"], j0=spec["src_j"][0], j1=spec["src_j"][1],
                          profile=GaussianPulse(0.65, 0.2))
        fx, fy = spec["flux_x"], spec["flux_y"]
        freqs = list(W.CFG2_FREQS)
        if spec["pol"] == "tm":
            m = build_tm_coeffs(g, eps_inf=eps, npml=W.NPML2D)
            mons = [DFTFieldsMonitor(g, freqs, "Ez"),
                    FluxMonitorTM(g, freqs, x_normal=True, idx=fx[0], lo=fx[1], hi=fx[2]),
                    FluxMonitorTM(g, freqs, x_normal=False, idx=fy[0], lo=fy[1], hi=fy[2])]
            run, st0, src = run_tm, init_tm_state(g), line
        else:
            m = build_te_coeffs(g, eps_inf=eps, npml=W.NPML2D)

            class _TESrc:                   # Simulation's TE binding: mask[:, :-1] -> Dy
                mask = line.mask[:, :-1]
                amplitude = staticmethod(line.amplitude)

            mons = [DFTFieldsMonitor(g, freqs, "Hz"),
                    FluxMonitorTE(g, freqs, ix=fx[0], lo=fx[1], hi=fx[2]),
                    FluxMonitorTEY(g, freqs, iy=fy[0], lo=fy[1], hi=fy[2])]
            run, st0, src = run_te, init_te_state(g), _TESrc()
        with torch.no_grad():
            t0 = time.perf_counter()
            run(st0, m, steps, source=src, monitors=mons)
            sec += time.perf_counter() - t0
        cells += nx * ny * steps
    return cells, sec


def ref_cfg1(steps=4000):
    """The reference's run_tm on cfg1 (the full run by default). (cell-updates, s)."""
    import torch
    from meep_torch.core.coeffs import build_tm_coeffs
    from meep_torch.core.grid import Grid
    from meep_torch.core.monitors import FluxMonitorTM
    from meep_torch.core.run import run_tm
    from meep_torch.core.sources import GaussianPulse, LineSource
    from meep_torch.core.stepper_tm import init_tm_state

    from meep_torch_b200 import workloads as W
    sp = W.cfg1_spec()
    g = Grid(nx=sp["nx"], ny=sp["ny"], dx=W.DX2D, dtype=torch.float32, device="cpu")
    m = build_tm_coeffs(g, eps_inf=torch.from_numpy(sp["eps"]), npml=W.NPML2D)
    i, j = sp["src"]
    src = LineSource(g, ix=i, j0=j, j1=j + 1, profile=GaussianPulse(0.15, 0.1))
    ix, lo, hi = sp["flux"]
    mon = FluxMonitorTM(g, list(sp["freqs"]), x_normal=True, idx=ix, lo=lo, hi=hi)
    with torch.no_grad():
        t0 = time.perf_counter()
        run_tm(init_tm_state(g), m, steps, source=src, monitors=[mon])
        sec = time.perf_counter() - t0
    return sp["nx"] * sp["ny"] * steps, sec


def ref_cfg3(steps, n=256):
    """The reference's run_3d (core/monitors_3d.py:192) on the cfg3 grid with its point
    source and six flux faces, `steps` steps. (cell-updates, s)."""
    import numpy as np
    import torch
    from meep_torch.core.monitors_3d import FluxMonitor3D, PointSource3D, run_3d
    from meep_torch.core.sources import GaussianPulse
    from meep_torch.core.stepper_3d import build_3d_coeffs, init_3d_state

    from meep_torch_b200 import workloads as W
    dx, npml = 1.0 / 16, 16
    c = build_3d_coeffs(n, n, n, dx, eps=torch.from_numpy(W.cfg3_eps(n)), npml=npml,
                        dtype=torch.float32)
    s0 = init_3d_state(n, n, n, npml=npml, dtype=torch.float32)
    src = PointSource3D(c.dt, "Ez", n // 2, n // 2, n // 2, GaussianPulse(0.5, 0.3))
    lo_, hi_ = 24 * n // 256, 232 * n // 256
    freqs = np.linspace(0.35, 0.65, 20).tolist()
    mons = [FluxMonitor3D(c.dt, freqs, normal=a, idx=(lo_ if i == 24 else hi_),
                          win=(lo_, hi_, lo_, hi_), dtype=torch.float32)
            for a, i in W.CFG3_FACES]
    with torch.no_grad():
        t0 = time.perf_counter()
        run_3d(s0, c, steps, source=src, monitors=mons)
        sec = time.perf_counter() - t0
    return n ** 3 * steps, sec


def ref_cfg4(steps):
    """One gradient of the cfg4-shaped problem through the reference's design chain and
    autograd of run_tm(checkpoint_every=256), `steps` time steps. Returns seconds."""
    import numpy as np
    import torch
    from meep_torch.adjoint.problem import DesignRegion, MaterialGrid, OptimizationProblem
    from meep_torch.core.coeffs import build_tm_coeffs
    from meep_torch.core.grid import Grid
    from meep_torch.core.monitors import FluxMonitorTM
    from meep_torch.core.run import run_tm
    from meep_torch.core.sources import GaussianPulse, LineSource
    from meep_torch.core.stepper_tm import init_tm_state

    from meep_torch_b200 import workloads as W
    c = W.CFG4
    nx, ny, dx, npml = c["nx"], c["ny"], c["dx"], c["npml"]
    base = torch.full((nx, ny), c["eps_bg"], dtype=torch.float32)
    y0, y1 = ny // 2 - c["guide_w"] // 2, ny // 2 + c["guide_w"] // 2
    base[:, y0:y1] = c["eps_core"]
    d = c["design"]
    ix0, iy0 = nx // 2 - d // 2, ny // 2 - d // 2
    reg = DesignRegion(MaterialGrid((d, d), c["eps_bg"], c["eps_core"]), ix0=ix0, ix1=ix0 + d,
                       iy0=iy0, iy1=iy0 + d)
    grid = Grid(nx=nx, ny=ny, dx=dx, dtype=torch.float32, device="cpu")
    src = LineSource(grid, ix=npml + 10, j0=y0 - 10, j1=y1 + 10,
                     profile=GaussianPulse(0.645, 0.12))
    mon = FluxMonitorTM(grid, list(c["freqs"]), x_normal=True, idx=nx - npml - 10,
                        lo=y0 - 20, hi=y1 + 20)

    def run_fn(eps):
        m = build_tm_coeffs(grid, eps_inf=eps, npml=npml)
        _, (acc,) = run_tm(init_tm_state(grid), m, steps, source=src, monitors=[mon],
                           checkpoint_every=256)
        return mon.flux(acc, dx).mean()

    rho0 = torch.tensor(np.random.default_rng(4).uniform(0.4, 0.6, (d, d)), dtype=torch.float32)
    opt = OptimizationProblem(run_fn, base, reg, filter_radius=c["radius"], dx=dx,
                              beta=c["beta"], eta=c["eta"], rho0=rho0)
    t0 = time.perf_counter()
    opt()
    return time.perf_counter() - t0


def reference_cpu(wl, args, threads):
    """(value, unit, cores, sample, kind) of the reference's own CPU path on a bounded
    sample of workload `wl`, or None when the reference is not installed (cfg5: the
    reference has no surrogate, so None). The reference runs on every host thread; the
    process's own torch thread count is put back afterwards. It runs after every GPU
    measurement of the line."""
    import torch
    prev = torch.get_num_threads()
    try:
        return _reference_cpu(wl, args, threads)
    finally:
        torch.set_num_threads(prev)


def _reference_cpu(wl, args, threads):
    if wl == "cfg5" or reference_module() is None:
        return None
    import torch
    torch.set_num_threads(os.cpu_count() or 1)
    cores = torch.get_num_threads()
    from meep_torch_b200 import workloads as W
    if wl == "cfg2":
        n_s, steps = args.ref_structs, args.ref_steps or 500
        cells, sec = ref_cfg2(W.cfg2_specs()[:n_s], steps)
        return (cells / sec / 1e9, "Gcell-updates/s", cores,
                f"reference meep_torch run_tm / run_te (float32, no_grad, {cores} torch "
                f"threads) on cfg2 structures 0..{n_s - 1} x {steps} steps with the cfg2 DFT and "
                f"flux monitors, {sec:.1f} s", "reference")
    if wl == "cfg1":
        cells, sec = ref_cfg1(4000)
        return (cells / sec / 1e9, "Gcell-updates/s", cores,
                f"reference meep_torch run_tm (float32, no_grad, {cores} torch threads), the "
                f"full 4000-step cfg1 run, {sec:.1f} s", "reference")
    if wl == "cfg3":
        steps = 6
        cells, sec = ref_cfg3(steps, n=args.n3)
        return (cells / sec / 1e9, "Gcell-updates/s", cores,
                f"reference meep_torch run_3d (float32, no_grad, {cores} torch threads) on the "
                f"cfg3 {args.n3}^3 grid with its source and six flux faces, {steps} steps, "
                f"{sec:.1f} s", "reference")
    if wl == "cfg4":
        steps = args.ref_steps or 256
        n = args.run_steps if args.run_steps != 5000 else W.CFG4["steps"]
        sec = ref_cfg4(steps)
        return (1.0 / (sec * n / steps), "gradient-evaluations/s", cores,
                f"reference meep_torch OptimizationProblem gradient (design chain + autograd "
                f"of run_tm, checkpoint_every=256, float32, {cores} torch threads) over {steps} "
                f"steps in {sec:.1f} s, scaled to the {n}-step run", "reference")
    return None


def config_suite(args, rank, world, dev):
    """The other single-GPU configurations measured in the same run as the default line
    (cfg1 4000-step TM run, cfg3 256^3 2000-step run, cfg4 gradient), each with its own
    value and, for the HBM-bound cfg3, its roofline; two warm-up and two timed steps."""
    out = {}
    peak, _ = peaks()
    for wl in ("cfg1", "cfg3", "cfg4"):
        a = argparse.Namespace(**dict(vars(args)))
        a.workload, a.steps, a.warmup, a.no_e2e, a.run_steps = wl, 2, 2, True, 5000
        a.rows = a.ring = 0
        a.variant = 0
        if wl == "cfg4":
            r = run_cfg4(a, rank, world, dev)
            out[wl] = {"metric": "gradient-evaluations/s",
                       "value": r["grad_evals"] / (r["ms"] / 1e3),
                       "ms_per_step": r["ms"] / a.steps, "steps": a.steps,
                       "time_steps": r["nsteps"], "checkpoint_every": 256}
            continue
        r = (run_cfg1 if wl == "cfg1" else run_cfg3)(a, rank, world, dev)
        total = r["cells"] * r["nsteps"] * a.steps
        ent = {"metric": "Gcell-updates/s", "value": total / (r["ms"] / 1e3) / 1e9,
               "ms_per_step": r["ms"] / a.steps, "steps": a.steps, "time_steps": r["nsteps"],
               "cells": r["cells"]}
        if wl == "cfg3":
            avg = r["step_ms"] / max(r["step_n"], 1)
            ach = r["bytes_launch"] / (avg / 1e3) / 1e9
            ent["roofline"] = {"bound": "hbm", "kernel": "k_yee3d_xm (one pass per step)",
                               "achieved": ach, "peak": peak, "unit": "GB/s",
                               "frac": ach / peak, "alg_bytes_per_step": r["bytes_launch"],
                               "launch_ms": avg}
        out[wl] = ent
    return out


def reference_line(args, config, threads):
    """The reference arm: the oracle port of the reference's CPU path, timed on the
    host cores on a bounded sample of the chosen workload, in that workload's metric."""
    from meep_torch_b200 import workloads as W
    wl = args.workload
    vals = []
    t_all = time.perf_counter()
    kind = "port"
    if reference_module() is not None and wl != "cfg5":
        kind = "reference"
        if wl == "cfg2" and args.warmup:
            ref_cfg2(W.cfg2_specs()[:1], 5)                                  # warm-up
            t_all = time.perf_counter()
        sample = unit = None
        cores = 1
        for _ in range(args.steps):
            v_, unit, cores, sample, _k = reference_cpu(wl, args, threads)
            vals.append(v_)
    elif wl == "cfg2":
        unit = "Gcell-updates/s"
        specs = W.cfg2_specs()[:args.cpu_structs]
        for _ in range(args.warmup and 1):
            cpu_sample(specs[:1], 2, 1)
        t_all = time.perf_counter()
        for _ in range(args.steps):
            cells, sec = cpu_sample(specs, args.cpu_steps, threads)
            vals.append(cells / sec / 1e9)
        cores = threads
        sample = (f"oracle numpy float32 TM/TE step + DFT/flux monitors, cfg2 structures "
                  f"0..{len(specs) - 1} x {args.cpu_steps} steps per bench step, {threads} "
                  "threads over structures")
    elif wl == "cfg1":
        unit, cores = "Gcell-updates/s", 1
        for _ in range(args.steps):
            cells, sec = cpu_sample_cfg1(4000)
            vals.append(cells / sec / 1e9)
        sample = "oracle numpy float32 cfg1, the full 4000-step run per bench step, one thread"
    elif wl == "cfg3":
        unit, cores = "Gcell-updates/s", 1
        for _ in range(args.steps):
            cells, sec = cpu_sample_cfg3(8, n=args.n3)
            vals.append(cells / sec / 1e9)
        sample = (f"oracle numpy float32 cfg3 {args.n3}^3 grid with its source and six flux "
                  "faces, 8 steps per bench step, one thread")
    elif wl == "cfg4":
        unit, cores = "gradient-evaluations/s", 1
        n = args.run_steps if args.run_steps != 5000 else W.CFG4["steps"]
        for _ in range(args.steps):
            sec = cpu_sample_cfg4(300)
            vals.append(1.0 / (sec / 300 * 2 * n))
        sample = (f"oracle numpy float32 forward, 300 steps of the cfg4 grid per bench step, "
                  f"one thread; a gradient costed as 2 x {n} steps (the oracle has no reverse "
                  "mode)")
    else:
        unit, cores = "design-iterations/s", 1
        for _ in range(args.steps):
            sec = cpu_sample_cfg5(S_CFG5_STEPS)
            vals.append(1.0 / (2 * sec))
        sample = (f"oracle numpy float32 forward with the 3-frequency DFT, the full "
                  f"{S_CFG5_STEPS}-step run of one cfg5 design per bench step, one thread; a "
                  "plain design iteration costed as two runs (the oracle has no reverse mode "
                  "and no surrogate)")
    wall = time.perf_counter() - t_all
    v = statistics.median(vals)
    metric = CFG5_METRIC if wl == "cfg5" else unit
    return {"metric": metric, "value": v, "unit": unit, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": wall / max(args.steps, 1) * 1e3,
            "higher_is_better": True, "impl": "reference", "dtype": "f32",
            "data": "synthetic", "config": config,
            "cpu_baseline": {"value": v, "unit": unit, "cores": cores, "kind": kind,
                             "sample": sample},
            "e2e": {"value": v, "unit": unit, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def allreduce_sum(x, world, dev):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], device=dev, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def allreduce_max(x, world, dev):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], device=dev, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="cfg2", choices=["cfg1", "cfg2", "cfg3", "cfg4", "cfg5"])
    ap.add_argument("--maps", type=int, default=20000, help="cfg5 training designs")
    ap.add_argument("--epochs", type=int, default=16, help="cfg5 FNO training epochs")
    ap.add_argument("--iters", type=int, default=50,
                    help="cfg5 design iterations (plain loop) / verifications (surrogate)")
    ap.add_argument("--rows", type=int, default=0, help="rows per warp (0 = library default)")
    ap.add_argument("--ring", type=int, default=0, help="DFT ring depth (0 = default)")
    ap.add_argument("--cpu-structs", type=int, default=0, help="0 = host threads, 8..64")
    ap.add_argument("--cpu-steps", type=int, default=300)
    ap.add_argument("--ref-structs", type=int, default=16,
                    help="cfg2 structures of the reference's own CPU run (reference arm)")
    ap.add_argument("--ref-steps", type=int, default=0,
                    help="time steps of the reference's own CPU sample (0 = per workload)")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--structs", type=int, default=256,
                    help="structures per rank (profiling runs use fewer)")
    ap.add_argument("--run-steps", type=int, default=5000,
                    help="time steps per run (profiling runs use fewer)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-suite", action="store_true",
                    help="cfg2 at one GPU: skip the cfg1 / cfg3 / cfg4 lines measured after it")
    ap.add_argument("--n3", type=int, default=256, help="cfg3 grid side")
    ap.add_argument("--shard", default="none", choices=["none", "fixed"],
                    help="under torchrun: none = every rank its own problem (weak "
                         "scaling); fixed = one problem split across the ranks (strong "
                         "scaling): cfg2's batch by LPT on cells with the accumulators "
                         "gathered on rank 0, cfg3's grid into x slabs with halo planes "
                         "exchanged every half step")
    ap.add_argument("--variant", type=int, default=0,
                    help="kernel variant, 0 library default; 2D: 1 row march, 2 tiles, "
                         "3 temporally blocked tiles, 4 cluster-resident; 3D: 1 fused "
                         "x-march, 2 split H / E, 3 one pass")
    ap.add_argument("--geometry", type=int, default=0,
                    help="3D one-pass work split: 0 library default, 1 tile-major shares, "
                         "2 lockstep tiles")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    threads = os.cpu_count() or 1
    if args.cpu_structs <= 0:
        args.cpu_structs = min(max(8, threads), 64)
    if args.workload == "cfg5":
        config = {"workload": "cfg5: surrogate-assisted design of a 64 x 64 px region "
                              "(eps 1..4) in a 256 x 256 TM cell at res 20, 20-cell CPML, "
                              "Gaussian line source (0.65, 0.25), 3000 steps per FDTD run; "
                              "objective mean |Ez|^2 of the 0.6/0.65/0.7 DFT on an 8 x 8 patch "
                              "behind the design",
                  "training_maps": args.maps, "test_maps": 256, "epochs": args.epochs,
                  "maps": "Gaussian random fields, correlation 4 px (0.2 um); half thresholded "
                          "at 0, half soft-thresholded sigmoid(beta g / std g), beta ~ U(0.5, 4); "
                          "conic filter 0.1 um; seed 5",
                  "fno": "4 layers, width 64, 24 x 24 modes; channel mixes and the 64->128 "
                         "projection on the library's tcgen05 kernels (BF16 operands, FP32 "
                         "accumulation in TMEM), forward and backward; FFTs and per-mode "
                         "complex mixes FP32 (cuFFT / cuBLAS)",
                  "loops": f"plain: {args.iters} Adam steps (lr 0.05) on the FDTD adjoint "
                           "gradient; surrogate: first-order-corrected trust region, blocks of "
                           "20 FNO Adam steps (lr 0.2, radius 2 in z) probed after 2/5/10/15/20 "
                           "steps, probes verified by one batched forward FDTD run, an adjoint "
                           "run at each accepted probe, 2 fine-tuning steps per block on the "
                           "verified fields plus replay; stops at 99 % of the plain loop's final "
                           "FOM (at most 2x the plain iteration count in blocks)",
                  "l2": "data generation batches of 1024 x 256^2 designs (~1.5 GB of "
                        "fields): larger than L2; design loops are latency-bound"}
    elif args.workload == "cfg4":
        config = {"workload": "cfg4: gradient of a 600 x 400 TM mode-converter-shaped problem "
                              "(res 25, 25-cell CPML, 160 x 160 design, conic filter + tanh "
                              "projection, line source across the input guide standing in for "
                              "the mode source, output-port flux at 3 wavelengths), 8000 steps "
                              "forward + adjoint sweep per gradient",
                  "time_steps": args.run_steps if args.run_steps != 5000 else 8000,
                  "checkpoint_every": 256, "seed": "4 + 1009*rank",
                  "l2": "L2-resident working set (~10 MB of state): latency-bound"}
    elif args.workload == "cfg1":
        config = {"workload": "cfg1: 2D TM waveguide 320 x 160 (16 x 8 um at res 20), 1 um "
                              "CPML, eps 12 guide, Gaussian Ez source (0.15, 0.1), one "
                              "50-frequency flux line, 4000 steps per run",
                  "time_steps": args.run_steps if args.run_steps != 5000 else 4000,
                  "l2": "L2-resident working set (~1.4 MB): latency-bound; whole DFT ring "
                        "flushes replayed as CUDA graphs"}
    elif args.workload == "cfg3":
        n3 = args.n3
        steps3 = args.run_steps if args.run_steps != 5000 else 2000
        config = {"workload": f"cfg3: 3D {n3}^3 at res 16, 16-cell CPML on all faces, 200 "
                              "random dielectric spheres, Gaussian Ez point dipole, six "
                              "20-frequency flux faces, 2000 steps per run",
                  "grid": [n3, n3, n3], "time_steps": steps3, "seed": 3,
                  "kernel_variant": args.variant or "library default (one pass)",
                  "geometry": args.geometry or "library default",
                  "l2": f"inputs larger than L2 (~{37 * 4 * n3 ** 3 / 1e9:.1f} GB of field "
                        "state)"}
    else:
        config = {"workload": "cfg2: 256 batched 2D TE/TM bend variants (256..768)^2, res 20, "
                              "1 um CPML, Gaussian line source, full-grid DFT 3 freqs + 2 flux "
                              "lines, 5000 steps per run",
                  "structures_per_rank": args.structs, "time_steps": args.run_steps,
                  "seed": "2 + 1009*rank",
                  "l2": "inputs larger than L2 (~1.1 GB of field state per rank)"}

    if args.impl == "reference":
        if rank != 0:
            return
        print(json.dumps(reference_line(args, config, threads)))
        return

    import torch
    if world > 1:
        import torch.distributed as dist
        local = int(os.environ.get("LOCAL_RANK", "0"))
        torch.cuda.set_device(local)
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
        dev = torch.device("cuda", local)
    else:
        torch.cuda.set_device(0)
        dev = torch.device("cuda", 0)
    from meep_torch_b200 import build as B
    if rank == 0:
        B.build()
    barrier(world)

    if args.workload == "cfg4":
        r = run_cfg4(args, rank, world, dev)
        value = r["grad_evals"] / (r["ms"] / 1e3)
        line = {"metric": "gradient-evaluations/s", "value": value,
                "unit": "gradient-evaluations/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": r["ms"] / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32", "data": "synthetic",
                "config": dict(config, parallelism=f"independent problem per rank x{world}"),
                "roofline": {"bound": "latency (L2-resident)", "achieved": None,
                             "peak": peaks()[0], "unit": "GB/s", "frac": None, "traffic": None,
                             "note": "600 x 400 fits in L2; each step is a few microsecond "
                                     "launches, so the HBM roofline does not apply"},
                "e2e": {"value": (args.steps * world / r["e2e_s"]
                                  if r["e2e_s"] == r["e2e_s"] else None),
                        "unit": "gradient-evaluations/s", "h2d_bytes_per_step": r["h2d"],
                        "d2h_bytes_per_step": r["d2h"]},
                "clocks": r["clocks"], "gpu_launches": r["launches"]}
        if rank == 0 and not args.no_cpu:
            sec = cpu_sample_cfg4(300)
            per_grad = sec / 300 * 2 * r["nsteps"]
            line["cpu_baseline"] = {"value": 1.0 / per_grad, "unit": "gradient-evaluations/s",
                                    "cores": 1, "kind": "port",
                                    "sample": f"oracle (numpy float32) forward, 300 steps of the "
                                              f"cfg4 grid in {sec:.1f} s, one thread; a gradient "
                                              f"costed as 2 x {r['nsteps']} steps (the reverse "
                                              "sweep at the forward's cost); the oracle has no "
                                              "reverse mode"}
        if rank == 0:
            print(json.dumps(line))
        if world > 1:
            import torch.distributed as dist
            dist.barrier()
            dist.destroy_process_group()
        return
    if args.workload == "cfg5":
        r = run_cfg5(args, rank, world, dev)
        plain, sur = r["plain"], r["sur"]
        reached = sur["fom"][-1] >= r["target"]
        t_sur = sur["t"][-1]
        n_it = len(plain["fom"])
        peak, peak_kind = peaks()
        step_avg = r["step_ms"] / max(r["step_n"], 1)
        ach = r["bytes_launch"] / (step_avg / 1e3) / 1e9 if step_avg else None
        line = {"metric": CFG5_METRIC,
                "value": n_it / t_sur if reached else None,
                "unit": "design-iterations/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": (plain["seconds"] + sur["seconds"]) * 1e3,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32 FDTD, bf16 FNO", "data": "synthetic",
                "config": dict(config, parallelism=f"independent problem per rank x{world}"),
                "plain_loop": {"iterations": n_it, "seconds": plain["seconds"],
                               "design_iterations_per_s": n_it / plain["seconds"],
                               "fom_start": plain["fom"][0], "fom_final": plain["fom"][-1]},
                "surrogate_loop": {"reached_target": reached, "target_fom": r["target"],
                                   "fom_final": sur["fom"][-1],
                                   "fom_rel_err_vs_plain": abs(sur["fom"][-1] - plain["fom"][-1])
                                   / plain["fom"][-1],
                                   "seconds": t_sur, "fdtd_runs": sur["fdtd_runs"],
                                   "surrogate_steps": sur["surrogate_steps"],
                                   "adjoint_runs": sur["adjoint_runs"],
                                   "accepted": sum(sur["accepted"]) - 1,
                                   "speedup_vs_plain": plain["seconds"] / t_sur
                                   if reached else None},
                "surrogate": {"train_seconds": r["train_s"], "test_rel_l2": r["test_err"],
                              "test_fom_rel_err_median": r["fom_err"],
                              "training_maps": r["n_train"]},
                "data_generation": {"seconds": r["gen_s"],
                                    "gcell_updates_per_s": r["gen_updates"] / r["gen_s"] / 1e9},
                "roofline": {"bound": "hbm", "kernel": "k_tile_tm (data generation, one step "
                             "of a 1024-design batch)", "achieved": ach, "peak": peak,
                             "peak_kind": peak_kind, "unit": "GB/s",
                             "frac": ach / peak if ach else None, "traffic": None,
                             "alg_bytes_per_launch": r["bytes_launch"], "launch_ms": step_avg,
                             "launches": r["step_n"], "dft_contract_ms_total": r["dft_ms"],
                             "note": "the design loops themselves are latency-bound (one "
                                     "256 x 256 structure)"},
                "e2e": {"value": n_it / r["e2e_s"] if r["e2e_reached"] else None,
                        "unit": "design-iterations/s", "h2d_bytes_per_step": r["h2d"],
                        "d2h_bytes_per_step": r["d2h"]},
                "clocks": r["clocks"], "gpu_launches": r["launches"]}
        if rank == 0 and not args.no_cpu:
            sec = cpu_sample_cfg5(S_CFG5_STEPS)
            line["cpu_baseline"] = {"value": 1.0 / (2 * sec), "unit": "design-iterations/s",
                                    "cores": 1, "kind": "port",
                                    "sample": f"oracle (numpy float32) forward with the 3-freq "
                                              f"DFT, the full {S_CFG5_STEPS}-step run of one "
                                              f"cfg5 design in {sec:.1f} s, one thread; one "
                                              "plain design iteration costed as two runs "
                                              "(forward + reverse sweep at the forward's cost)"}
        if rank == 0:
            print(json.dumps(line))
        if world > 1:
            import torch.distributed as dist
            dist.barrier()
            dist.destroy_process_group()
        return
    slabs3 = args.workload == "cfg3" and args.shard == "fixed"
    r = {"cfg1": run_cfg1, "cfg2": run_cfg2,
         "cfg3": run_cfg3_slabs if slabs3 else run_cfg3}[args.workload](args, rank, world, dev)
    peak, peak_kind = peaks()
    cells_total = allreduce_sum(r["cells"], world, dev)       # every rank's own cells
    total_updates = cells_total * r["nsteps"] * args.steps
    value = total_updates / (r["ms"] / 1e3) / 1e9
    step_avg_ms = r["step_ms"] / max(r["step_n"], 1)
    # time steps one step-kernel launch advances: 1 for the one-step kernels, up to 4
    # for the temporally blocked ones (every timed step is covered by a timed launch)
    steps_per_launch = (r.get("timed_steps", r["step_n"]) / max(r["step_n"], 1))
    achieved = r["bytes_launch"] * steps_per_launch / (step_avg_ms / 1e3) / 1e9
    traffic = None
    cfg3 = args.workload == "cfg3"
    prof = os.path.join(ROOT, "profiles", "yee3d_step_cfg3_traffic.json" if cfg3
                        else "yee2d_step_cfg2_traffic.json")
    if os.path.exists(prof) and args.workload in ("cfg2", "cfg3"):
        with open(prof) as f:
            tr = json.load(f)
        eff = args.variant or 3                  # library defaults: TB tiles (2D), one pass (3D)
        entry = tr.get("variants", {}).get(str(eff)) if "variants" in tr else (
            tr if tr.get("variant") == eff else None)
        if entry and round(entry.get("steps_per_launch", 1)) == round(steps_per_launch):
            traffic = entry.get("dram_bytes_per_launch")
    e2e_val = (total_updates / r["e2e_s"] / 1e9
               if r["e2e_s"] == r["e2e_s"] else None)
    kernel = ("k_cl_tm (cluster-resident, a ring of steps per launch; graph replays, step "
              "time = run time / steps)" if args.workload == "cfg1" and args.variant in (0, 4)
              else
              "k_tb_tm (temporally blocked, 4 steps per launch; graph replays, step time = "
              "run time / steps)" if args.workload == "cfg1" and args.variant == 3 else
              "k_tile_tm (one step; graph replays, step time = run time / steps)"
              if args.workload == "cfg1" and args.variant == 2 else
              "k_yee2d_tm (one step; graph replays, step time = run time / steps)"
              if args.workload == "cfg1" else
              "k_yee3d_xm (one pass per step)" if cfg3 and args.variant in (0, 3) else
              "k_yee3d_h + k_yee3d_e (one step)" if cfg3 and args.variant == 2 else
              "k_yee3d_step (one step)" if cfg3 else
              "k_yee2d_tm + k_yee2d_te (one step)" if args.variant == 1 else
              "k_tile_tm + k_tile_te (one step)" if args.variant == 2 else
              "k_tb_tm + k_tb_te (temporally blocked: up to 4 steps per launch)")
    line = {
        "metric": "Gcell-updates/s", "value": value, "unit": "Gcell-updates/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": r["ms"] / args.steps, "higher_is_better": True,
        "scaling": "strong" if args.shard == "fixed" else "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": dict(config, parallelism=(
            f"one batch split across {world} ranks (LPT on cells), accumulators gathered on "
            "rank 0" if (args.shard == "fixed" and args.workload == "cfg2")
            else f"one grid split along x into {world} slabs, halo planes over NCCL "
            "point-to-point, flux accumulators reduced onto rank 0" if slabs3
            else f"independent problem per rank x{world}"),
                       cells_per_rank=r["cells"]),
        "roofline": {"bound": "hbm", "kernel": kernel, "achieved": achieved,
                     "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic,
                     "alg_bytes_per_step": r["bytes_launch"],
                     "steps_per_launch": steps_per_launch,
                     "alg_bytes_per_launch": r["bytes_launch"] * steps_per_launch,
                     "launch_ms": step_avg_ms, "launches": r["step_n"],
                     "dft_contract_ms_total": r["dft_ms"], "dft_contract_launches": r["dft_n"],
                     "step_kernel_share": r["step_ms"] / max(r["ms"], 1e-9),
                     # the measured DRAM bytes of a step (ncu, profiles/) over the live step
                     # time: the raw-bytes rate, beside the algorithmic one above
                     "achieved_raw": (traffic / (step_avg_ms / 1e3) / 1e9
                                      if traffic else None),
                     "frac_raw": (traffic / (step_avg_ms / 1e3) / 1e9 / peak
                                  if traffic else None)},
        "e2e": {"value": e2e_val, "unit": "Gcell-updates/s", "h2d_bytes_per_step": r["h2d"],
                "d2h_bytes_per_step": r["d2h"]},
        "clocks": r["clocks"],
        "gpu_launches": r["launches"],
    }
    # the other configs run before the host-side reference sample: that sample keeps every
    # host thread busy, and cfg4 (host-launch bound) measured 2.9 instead of 5.0
    # gradients/s right after it
    if args.workload == "cfg2" and world == 1 and not args.no_suite:
        line["other_configs"] = config_suite(args, rank, world, dev)
    ref_cpu = (reference_cpu(args.workload, args, threads)
               if rank == 0 and not args.no_cpu else None)
    if ref_cpu is not None:
        v_, u_, cores_, sample_, kind_ = ref_cpu
        line["cpu_baseline"] = {"value": v_, "unit": u_, "cores": cores_, "kind": kind_,
                                "sample": sample_}
    elif rank == 0 and not args.no_cpu:
        if args.workload == "cfg1":
            cells, sec = cpu_sample_cfg1(4000)
            line["cpu_baseline"] = {"value": cells / sec / 1e9, "unit": "Gcell-updates/s",
                                    "cores": 1, "kind": "port",
                                    "sample": f"oracle (numpy float32) cfg1, the full 4000-step "
                                              f"run, one thread, {sec:.1f} s"}
        elif args.workload == "cfg3":
            n3s = 8
            cells, sec = cpu_sample_cfg3(n3s, n=args.n3)
            line["cpu_baseline"] = {"value": cells / sec / 1e9, "unit": "Gcell-updates/s",
                                    "cores": 1, "kind": "port",
                                    "sample": f"oracle (numpy float32) cfg3 {args.n3}^3 grid with "
                                              f"its source and six flux faces, {n3s} steps, one "
                                              f"thread, {sec:.1f} s"}
        else:
            line["cpu_baseline"] = cpu_baseline_line(args.cpu_structs, args.cpu_steps, threads)
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
