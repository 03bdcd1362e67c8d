"""Parity at the benchmark configurations' own sizes and lengths.

The fixtures (``tests/golden/config_*.npz``, made by ``make_config_golden.py``) are the
REFERENCE's own runs of the configurations on the host, in float32 (the parity target)
and float64 (the error floor):

* cfg1: 320 x 160 TM, Gaussian point source, 50-frequency flux line, 4000 steps;
* cfg2: four of the 256 seeded bends (two TM, two TE, among them the largest grids of
  the batch), full-grid 3-frequency DFT and two flux lines, 5000 steps, run here as one
  batched plan the way the benchmark runs the whole batch;
* cfg3: the 256^3 sphere grid, centre Ez dipole, six 20-frequency flux faces, 2000 steps;
* cfg4: the 600 x 400 design problem's objective and d J / d rho through the design
  chain and ``run_tm(checkpoint_every=256)``, 8000 steps (float32; float64 over 2000
  steps), and central differences of the float64 objective on 32 pixels.

Bar: relative L2 < 1e-4 against the reference's float32 run on fields, DFT accumulators
and flux spectra. The float64 error is printed beside it. Large
arrays are compared on the fixture's strided subsample (its stride is in the fixture). The
cfg4 gradient, a derivative accumulated over 8000 reverse steps in float32, is held to
1e-3 against the float64 reference and its objective to 1e-4.
"""
import os

import numpy as np
import pytest
import torch

from tests.conftest import GOLDEN, rel_l2

pytestmark = pytest.mark.gpu

TOL = 1e-4
GRAD_TOL = 1e-3


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    from meep_torch_b200 import build
    build.build()


def _fixture(name):
    path = os.path.join(GOLDEN, f"config_{name}.npz")
    if not os.path.exists(path):
        pytest.skip(f"fixture {name} not generated")
    with np.load(path, allow_pickle=False) as z:
        return {k: z[k] for k in z.files}


def _sub(a, stride, lead=0):
    o = stride // 2
    sl = (slice(None),) * lead + (slice(o, None, stride), slice(o, None, stride))
    return a[sl]


def _np(t):
    return t.detach().cpu().double().numpy()


def _check(name, got, fixtures):
    """got: key -> array comparable with fixtures[prec][key]. Prints both errors and
    returns the float32 ones."""
    errs = {}
    for prec in ("f32", "f64"):
        errs[prec] = {k: rel_l2(v, fixtures[prec][k]) for k, v in got.items()}
    print(f"\n[{name}] max relL2 vs ref fp32: {max(errs['f32'].values()):.2e} "
          f"vs ref fp64: {max(errs['f64'].values()):.2e}  ({len(got)} arrays)")
    for k in got:
        print(f"    {k:>10s}  fp32 {errs['f32'][k]:.2e}  fp64 {errs['f64'][k]:.2e}")
    return errs["f32"]


def test_cfg1_full_run_matches_reference():
    from meep_torch_b200 import workloads as W
    from meep_torch_b200.core.run import run_tm
    fx = {p: _fixture(f"cfg1_{p}") for p in ("f32", "f64")}
    st, m, src, mons = W.cfg1_item("cuda")
    st, (acc,) = run_tm(st, m, int(fx["f32"]["n_steps"]), source=src, monitors=mons)
    s = int(fx["f32"]["field_stride"])
    got = {"acc": _np(acc), "flux": _np(mons[0].flux(acc, W.DX2D))}
    for k in ("Ez", "Hx", "Hy"):
        got["s_" + k] = _sub(_np(getattr(st, k)), s)
    e32 = _check("cfg1", got, fx)
    assert max(e32.values()) < TOL, e32


def _cfg2_fixtures():
    names = sorted(f[len("config_"):-len("_f32.npz")] for f in os.listdir(GOLDEN)
                   if f.startswith("config_cfg2_b") and f.endswith("_f32.npz"))
    if not names:
        pytest.skip("cfg2 fixtures not generated")
    return names


@pytest.mark.parametrize("phase_mode", ["exact", "reference_fp32"])
def test_cfg2_variants_full_run_match_reference(phase_mode):
    from meep_torch_b200 import workloads as W
    from meep_torch_b200.engine2d import Engine2D
    names = _cfg2_fixtures()
    fxs = [{p: _fixture(f"{n}_{p}") for p in ("f32", "f64")} for n in names]
    specs = W.cfg2_specs()
    items = [W.cfg2_item(specs[int(f["f32"]["index"])], "cuda") for f in fxs]
    eng = Engine2D(items, phase_mode=phase_mode)
    try:
        eng.run(0, int(fxs[0]["f32"]["n_steps"]))
        worst = 0.0
        for b, (name, fx) in enumerate(zip(names, fxs)):
            st = eng.state(b)
            dft, ax, ay = eng.accumulators(b)
            mons = items[b][3]
            s, ds = int(fx["f32"]["field_stride"]), int(fx["f32"]["dft_stride"])
            got = {"dft": _sub(_np(dft), ds, lead=2), "acc_x": _np(ax), "acc_y": _np(ay),
                   "flux_x": _np(mons[1].flux(ax, W.DX2D)),
                   "flux_y": _np(mons[2].flux(ay, W.DX2D))}
            comps = ("Ez", "Hx", "Hy") if str(fx["f32"]["pol"]) == "tm" else ("Hz", "Ex", "Ey")
            for k in comps:
                got["s_" + k] = _sub(_np(getattr(st, k)), s)
            e32 = _check(f"cfg2 {name} {fx['f32']['pol']} {int(fx['f32']['nx'])}x"
                         f"{int(fx['f32']['ny'])} phase={phase_mode}", got, fx)
            worst = max(worst, max(e32.values()))
        assert worst < TOL, worst
    finally:
        eng.close()


def test_cfg3_full_run_matches_reference():
    from meep_torch_b200 import workloads as W
    from meep_torch_b200.core.monitors_3d import run_3d
    fx = {p: _fixture(f"cfg3_{p}") for p in ("f32", "f64")}
    s0, c, src, mons = W.cfg3_setup("cuda")
    st, accs = run_3d(s0, c, int(fx["f32"]["n_steps"]), source=src, monitors=mons)
    s, fs = int(fx["f32"]["field_stride"]), int(fx["f32"]["face_stride"])
    o = s // 2
    got = {}
    for k in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz"):
        got["s_" + k] = _np(getattr(st, k))[o::s, o::s, o::s]
    got["ez_mid"] = _np(st.Ez)[:, :, 128]
    for i, (a, mon) in enumerate(zip(accs, mons)):
        got[f"flux_{i}"] = _np(mon.flux(a, c.dx))
        got[f"acc_{i}"] = _sub(_np(a), fs, lead=2)
    e32 = _check("cfg3", got, fx)
    assert max(e32.values()) < TOL, e32


def _cfg4_against(names, ref_prec):
    from meep_torch_b200 import workloads as W
    fx = {p: _fixture(n) for p, n in names.items()}
    opt, n = W.cfg4_setup("cuda", steps=int(fx["f32"]["n_steps"]))
    opt.rho = torch.tensor(fx["f32"]["rho0"], dtype=torch.float32, device="cuda")
    J, g = opt()
    g = np.asarray(g, dtype=np.float64)
    out = {}
    for prec in fx:
        out[prec] = (abs(J - float(fx[prec]["J"])) / abs(float(fx[prec]["J"])),
                     rel_l2(g, fx[prec]["grad"]))
    print(f"\n[cfg4 {n} steps] " + "; ".join(
        f"vs ref {p}: J rel err {v[0]:.2e}, dJ/drho relL2 {v[1]:.2e}" for p, v in out.items()))
    assert all(v[0] < TOL for v in out.values()), out
    assert out[ref_prec][1] < GRAD_TOL, out


def test_cfg4_gradient_matches_reference():
    """The full 8000-step objective and gradient against the reference's float32 autograd
    (run_tm(checkpoint_every=256))."""
    _cfg4_against({"f32": "cfg4_f32"}, "f32")


def test_cfg4_short_gradient_matches_reference_fp64():
    """The same problem over 2000 steps against the reference in float32 and float64 (the
    float64 autograd of the full 8000 steps does not fit this machine's host memory)."""
    _cfg4_against({"f32": "cfg4_2000_f32", "f64": "cfg4_2000_f64"}, "f64")


def test_cfg4_gradient_matches_central_differences():
    """The kernels' d J / d rho (float32 adjoint) on the 32 random design pixels against
    central differences of the reference's float64 objective (h = 1e-4, 8000 steps)."""
    from meep_torch_b200 import workloads as W
    fd = _fixture("cfg4_fd_f64")
    g32 = _fixture("cfg4_f32")
    opt, n = W.cfg4_setup("cuda", steps=int(fd["n_steps"]))
    opt.rho = torch.tensor(g32["rho0"], dtype=torch.float32, device="cuda")
    _, g = opt()
    g = np.asarray(g, dtype=np.float64).reshape(-1)[fd["pixels"]]
    e = rel_l2(g, fd["fd"])
    print(f"\n[cfg4 FD] {len(g)} pixels: dJ/drho relL2 vs central differences {e:.2e}")
    assert e < GRAD_TOL, e
