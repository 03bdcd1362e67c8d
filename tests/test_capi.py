"""CPU-side checks of the C ABI and the host logic (no GPU needed).

* the shared library loads and exports every function include/meep_b200.h
  declares, with ctypes struct layouts matching the C sizes;
* argument validation fails with the documented status codes before any
  device work;
* the host mirror builds the same coefficients as the oracle, and the host
  helpers (coefficient tables, flux windows) match the reference's rules.
"""
import ctypes as C
import os
import re

import numpy as np
import pytest
import torch

from oracle import fdtd as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def lib():
    from meep_torch_b200 import _lib, build
    build.build()
    return _lib.load()


def header_functions():
    txt = open(os.path.join(ROOT, "include", "meep_b200.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(mtb_[a-z0-9_]+)\s*\(", txt)))


def test_every_declared_symbol_is_exported(lib):
    names = header_functions()
    assert len(names) >= 15
    for n in names:
        assert hasattr(lib, n), n


def test_binding_covers_header():
    from meep_torch_b200 import _lib
    assert set(header_functions()) == set(_lib.SIGNATURES)


def test_struct_layouts(lib):
    from meep_torch_b200 import _lib
    for i, cls in enumerate(_lib.STRUCTS):
        assert lib.mtb_struct_size(i) == C.sizeof(cls), cls.__name__
    assert lib.mtb_abi_version() == 1


def test_plan_validation_errors(lib):
    from meep_torch_b200 import _lib as L
    plan = C.c_void_p()
    rc = lib.mtb_yee2d_plan_create(None, 0, None, 0, None, 0, 0, 0, None, C.byref(plan))
    assert rc == L.MTB_INVALID_ARG
    assert b"structure" in lib.mtb_last_error()
    s = (L.Yee2DStruct * 1)()
    s[0].pol, s[0].nx, s[0].ny, s[0].pitch = 7, 10, 10, 12
    assert lib.mtb_yee2d_plan_create(s, 1, None, 0, None, 0, 0, 0, None,
                                     C.byref(plan)) == L.MTB_INVALID_ARG
    s[0].pol, s[0].nx, s[0].ny, s[0].pitch = 0, 10, 10, 10      # pitch not % 4
    assert lib.mtb_yee2d_plan_create(s, 1, None, 0, None, 0, 0, 0, None,
                                     C.byref(plan)) == L.MTB_INVALID_ARG
    s[0].pitch, s[0].dt, s[0].dx = 12, 0.025, 0.05               # null field pointers
    assert lib.mtb_yee2d_plan_create(s, 1, None, 0, None, 0, 0, 0, None,
                                     C.byref(plan)) == L.MTB_INVALID_ARG
    assert b"null" in lib.mtb_last_error()
    s3 = L.Yee3DStruct()
    s3.nx, s3.ny, s3.nz, s3.zpitch = 10, 10, 10, 10
    assert lib.mtb_yee3d_plan_create(C.byref(s3), None, 0, None, 0, 0, None,
                                     C.byref(plan)) == L.MTB_INVALID_ARG
    s3.zpitch = 1024                              # the fused kernel holds z <= 512
    fused = L.Tuning(0, 0, 0, 1)
    assert lib.mtb_yee3d_plan_create(C.byref(s3), None, 0, None, 0, 0, C.byref(fused),
                                     C.byref(plan)) == L.MTB_UNSUPPORTED
    s3.nx = 70000                                 # split kernels: nx is a grid dimension
    assert lib.mtb_yee3d_plan_create(C.byref(s3), None, 0, None, 0, 0, None,
                                     C.byref(plan)) == L.MTB_UNSUPPORTED
    assert lib.mtb_yee2d_run(None, 0, 1, None, None, None) == L.MTB_INVALID_ARG
    assert lib.mtb_pack(None, 1, 1, 1, 1, 1, None, 1, 1, 1, 1, 1, 0, 0, 0, None) == \
        L.MTB_INVALID_ARG


def test_check_maps_status_to_exceptions(lib):
    from meep_torch_b200 import _lib as L
    with pytest.raises(ValueError):
        L.check(L.MTB_INVALID_ARG)
    with pytest.raises(NotImplementedError):
        L.check(L.MTB_UNSUPPORTED)
    with pytest.raises(RuntimeError):
        L.check(L.MTB_CUDA_ERROR)


@pytest.mark.parametrize("npml,pmc", [(8, False), (((4, 6), (0, 5)), False), (6, True)])
def test_tm_coeffs_match_oracle(npml, pmc):
    from meep_torch_b200.core.coeffs import build_tm_coeffs
    from meep_torch_b200.core.grid import Grid
    g = Grid(nx=40, ny=30, dx=0.05, device="cpu")
    m = build_tm_coeffs(g, npml=npml, y_pmc=pmc)
    o = O.tm_coeffs(40, 30, 0.05, npml=npml, y_pmc=pmc, dtype=np.float32)
    for k in ("b_hy", "a_hy", "b_hx", "a_hx", "b_ex", "a_ex", "b_ey", "a_ey"):
        np.testing.assert_allclose(getattr(m, k).numpy(), o[k], rtol=2e-6, atol=1e-7)


FOLDS_TM = [dict(y_mirror=1), dict(y_mirror=-1), dict(x_mirror=1),
            dict(x_mirror=-1, y_mirror=1), dict(y_rot2=1), dict(y_rot2=-1), dict(rot4=1),
            dict(rot4=-1)]


@pytest.mark.parametrize("fold", FOLDS_TM + [dict(y_mirror=1, x_mirror=-1, te=1),
                                             dict(y_mirror=-1, x_mirror=1, te=1)])
def test_fold_coeffs_and_state_match_oracle(fold):
    """Symmetry cuts: the profiles (no absorber on the cut side, E-side slices from the
    cut node) and the TM state shapes (psi over the live Ez region, Hx0 / Hy0)."""
    from meep_torch_b200.core.coeffs import build_te_coeffs, build_tm_coeffs
    from meep_torch_b200.core.grid import Grid
    from meep_torch_b200.core.stepper_tm import init_tm_state
    fold = dict(fold)
    te = fold.pop("te", 0)
    g = Grid(nx=40, ny=40, dx=0.05, device="cpu")
    if te:
        m = build_te_coeffs(g, npml=8, **fold)
        o = O.te_coeffs(40, 40, 0.05, npml=8, dtype=np.float32, **fold)
    else:
        m = build_tm_coeffs(g, npml=8, **fold)
        o = O.tm_coeffs(40, 40, 0.05, npml=8, dtype=np.float32, **fold)
        s, so = init_tm_state(g, **fold), O.tm_state(o)
        for k in ("psi_Hyx", "psi_Hxy", "Hx0", "Hy0"):
            a, b = getattr(s, k), so.get(k)
            assert (a is None) == (b is None), k
            if a is not None:
                assert tuple(a.shape) == b.shape, k
    for k in ("b_hy", "a_hy", "b_hx", "a_hx", "b_ex", "a_ex", "b_ey", "a_ey"):
        np.testing.assert_allclose(getattr(m, k).numpy(), o[k], rtol=2e-6, atol=1e-7)


def test_te_and_3d_coeffs_match_oracle():
    from meep_torch_b200.core.coeffs import build_te_coeffs
    from meep_torch_b200.core.grid import Grid
    from meep_torch_b200.core.stepper_3d import build_3d_coeffs
    rng = np.random.default_rng(0)
    eps = rng.uniform(1, 12, (33, 27))
    m = build_te_coeffs(Grid(nx=33, ny=27, dx=0.05, device="cpu"),
                        eps_inf=torch.tensor(eps, dtype=torch.float32), npml=5)
    o = O.te_coeffs(33, 27, 0.05, eps=eps, npml=5, dtype=np.float32)
    np.testing.assert_array_equal(m.eps_x.numpy(), o["eps_x"])
    np.testing.assert_array_equal(m.eps_y.numpy(), o["eps_y"])
    for k in ("b_hx", "a_hx", "b_hy", "a_hy", "b_ex", "a_ex", "b_ey", "a_ey"):
        np.testing.assert_allclose(getattr(m, k).numpy(), o[k], rtol=2e-6, atol=1e-7)
    c = build_3d_coeffs(20, 18, 16, 1 / 16, npml=4, device="cpu")
    o3 = O.coeffs_3d(20, 18, 16, 1 / 16, npml=4, dtype=np.float32)
    for k in ("hx", "hy", "hz", "ex", "ey", "ez"):
        for a, b in zip(c.cpml[k], o3["cpml"][k]):
            np.testing.assert_allclose(a.numpy(), b, rtol=2e-6, atol=1e-7)


def test_unsupported_features_raise():
    from meep_torch_b200.core.coeffs import build_tm_coeffs
    from meep_torch_b200.core.grid import Grid
    g = Grid(nx=20, ny=20, dx=0.05, device="cpu")
    with pytest.raises(NotImplementedError):          # the reference refuses the pair too
        build_tm_coeffs(g, m_poles=[(1.0, 0.1, 1.0)], mu=2.0)
    with pytest.raises(TypeError):                    # a TE option, as in the reference
        build_tm_coeffs(g, eps_tensor=torch.ones(3, 20, 20))
    m = build_tm_coeffs(g, chi3=torch.ones(20, 20))          # chi2 / chi3: built, flagged
    assert m.has_kerr and not m.has_chi2
    with pytest.raises(ValueError):
        build_tm_coeffs(g, npml=10)


def test_pole_coefficients_match_oracle():
    """poles / pole_masks give the reference's ADE planes (core/coeffs.py:87-106,
    :195-203), as the oracle restates them."""
    from meep_torch_b200.core.coeffs import build_tm_coeffs
    from meep_torch_b200.core.grid import Grid
    poles = [(0.7, 0.05, 1.5), (0.0, 0.1, 1.0, 0.9)]
    masks = [np.zeros((20, 24), dtype=np.float32), np.ones((20, 24), dtype=np.float32)]
    masks[0][5:9, 3:10] = 1.0
    g = Grid(nx=20, ny=24, dx=0.05, device="cpu")
    m = build_tm_coeffs(g, poles=poles, pole_masks=[torch.from_numpy(x) for x in masks])
    c = O.tm_coeffs(20, 24, 0.05, dtype=np.float32, poles=poles, pole_masks=masks)
    for k in ("c1", "c2", "c3"):
        np.testing.assert_array_equal(getattr(m, k).numpy(), c[k])
    from meep_torch_b200.core.coeffs import build_te_coeffs
    t = build_te_coeffs(g, poles=poles, pole_masks=[torch.from_numpy(x) for x in masks])
    ct = O.te_coeffs(20, 24, 0.05, dtype=np.float32, poles=poles, pole_masks=masks)
    for k in ("c1x", "c2x", "c3x", "c1y", "c2y", "c3y"):
        np.testing.assert_allclose(getattr(t, k).numpy(), ct[k], rtol=2.5e-7, atol=0)


def test_conductivity_coefficients_match_oracle():
    """sigma_d gives the reference's (d1, d2) pairs on D (core/coeffs.py:161-166,
    :401-409; the oracle's restatement is pinned by the golden runs) and inert magnetic
    pairs (h1 = 1, h2 = dt)."""
    from meep_torch_b200.core.coeffs import build_te_coeffs, build_tm_coeffs
    from meep_torch_b200.core.grid import Grid
    rng = np.random.default_rng(3)
    sig = (3.0 * rng.random((20, 24))).astype(np.float32)
    g = Grid(nx=20, ny=24, dx=0.05, device="cpu")
    m = build_tm_coeffs(g, sigma_d=torch.from_numpy(sig))
    c = O.tm_coeffs(20, 24, 0.05, dtype=np.float32, sigma=sig)
    # torch's scalar / tensor division and numpy's differ in the last bit
    np.testing.assert_allclose(m.d1.numpy(), c["d1"], rtol=2.5e-7, atol=0)
    np.testing.assert_allclose(m.d2.numpy(), c["d2"], rtol=2.5e-7, atol=0)
    assert bool(torch.all(m.h1x == 1)) and bool(torch.all(m.h2y == torch.tensor(g.dt)))
    t = build_te_coeffs(g, sigma_d=torch.from_numpy(sig))
    ct = O.te_coeffs(20, 24, 0.05, dtype=np.float32, sigma=sig)
    for k in ("d1x", "d2x", "d1y", "d2y"):
        np.testing.assert_allclose(getattr(t, k).numpy(), ct[k], rtol=2.5e-7, atol=0)
    assert bool(torch.all(t.hz1 == 1))


def test_coef_table_matches_per_step_amplitudes():
    from meep_torch_b200.core.grid import Grid
    from meep_torch_b200.core.sources import CustomSource, GaussianPulse, LineSource
    from meep_torch_b200.engine2d import coef_table
    g = Grid(nx=40, ny=30, dx=0.05, device="cpu")
    for prof in (GaussianPulse(0.65, 0.2), CustomSource(lambda t: np.sin(t) ** 2)):
        src = LineSource(g, 5, 3, 20, prof)
        v = coef_table(src, "amplitude", 100, 400, g.dt)
        ref = np.array([g.dt * src.amplitude(t) for t in range(100, 500)])
        np.testing.assert_allclose(v, ref, rtol=1e-13, atol=1e-16)
        # float32 rounding of the coefficient is what the kernel sees
        assert np.array_equal(v.astype(np.float32), ref.astype(np.float32)) or \
            np.max(np.abs(v.astype(np.float32) - ref.astype(np.float32))) <= \
            np.max(np.abs(ref)) * 2 ** -23


def test_line_source_mask_matches_oracle():
    from meep_torch_b200.core.grid import Grid
    from meep_torch_b200.core.sources import GaussianPulse, LineSource
    g = Grid(nx=40, ny=30, dx=0.05, device="cpu")
    for j0, j1 in ((3, 20), (7, 8)):
        m = LineSource(g, 5, j0, j1, GaussianPulse(0.5, 0.2)).mask.numpy()
        np.testing.assert_array_equal(m, O.line_source_mask(40, 30, 0.05, 5, j0, j1,
                                                            dtype=np.float32))


@pytest.mark.parametrize("normal,idx,win,ap", [("x", 5, (2, 15, 3, 12), 0), ("y", 6, None, 2),
                                               ("z", 4, (0, 99, 1, 10), 0)])
def test_flux_window_matches_oracle(normal, idx, win, ap):
    from meep_torch_b200.engine3d import flux_window
    nx, ny, nz = 20, 18, 16
    s = {k: np.zeros(sh, np.float32) for k, sh in
         (("Ex", (nx - 1, ny, nz)), ("Ey", (nx, ny - 1, nz)), ("Ez", (nx, ny, nz - 1)),
          ("Hx", (nx, ny - 1, nz - 1)), ("Hy", (nx - 1, ny, nz - 1)), ("Hz", (nx - 1, ny - 1, nz)))}
    planes = O.flux3d_planes(s, normal, idx, win, ap)
    pairs, (l0, h0, l1, h1) = flux_window(normal, idx, nx, ny, nz, win, ap)
    assert planes[0].shape == (h0 - l0, h1 - l1)


def test_magnetic_coefficients_match_oracle():
    """sigma_b and mu give the reference's magnetic pairs (core/coeffs.py:167-175,
    :410-414), averaged onto Hx / Hy (TM) and Hz (TE) as the oracle restates them;
    the electric pair is built alongside (d1 = 1, d2 = dt without sigma_d)."""
    from meep_torch_b200.core.coeffs import build_te_coeffs, build_tm_coeffs
    from meep_torch_b200.core.grid import Grid
    rng = np.random.default_rng(4)
    sb = (3.0 * rng.random((20, 24))).astype(np.float32)
    mu = (1.0 + 2.0 * rng.random((20, 24))).astype(np.float32)
    g = Grid(nx=20, ny=24, dx=0.05, device="cpu")
    m = build_tm_coeffs(g, sigma_b=torch.from_numpy(sb), mu=torch.from_numpy(mu))
    c = O.tm_coeffs(20, 24, 0.05, dtype=np.float32, sigma_b=sb, mu=mu)
    for k in ("h1x", "h2x", "h1y", "h2y", "d1", "d2"):
        np.testing.assert_allclose(getattr(m, k).numpy(), c[k], rtol=5e-7, atol=0, err_msg=k)
    assert m.h1x.shape == (20, 23) and m.h1y.shape == (19, 24)
    t = build_te_coeffs(g, sigma_b=torch.from_numpy(sb), mu=torch.from_numpy(mu))
    ct = O.te_coeffs(20, 24, 0.05, dtype=np.float32, sigma_b=sb, mu=mu)
    for k in ("hz1", "hz2", "d1x", "d2y"):
        np.testing.assert_allclose(getattr(t, k).numpy(), ct[k], rtol=5e-7, atol=0, err_msg=k)
    assert t.hz1.shape == (19, 23)


def test_magnetic_pole_coefficients_and_state_match_oracle():
    """m_poles: the Hx / Hy recurrences with their masks averaged onto the H nodes, and
    the state's B and M histories."""
    from meep_torch_b200.core.coeffs import build_tm_coeffs
    from meep_torch_b200.core.grid import Grid
    from meep_torch_b200.core.stepper_tm import init_tm_state
    rng = np.random.default_rng(5)
    mp = [(0.6, 0.05, 0.8), (0.9, 0.1, 0.4)]
    masks = [(rng.random((30, 24)) < 0.4).astype(np.float64) for _ in mp]
    g = Grid(nx=30, ny=24, dx=0.05, device="cpu")
    m = build_tm_coeffs(g, npml=5, m_poles=mp,
                        m_pole_masks=[torch.tensor(x, dtype=torch.float32) for x in masks])
    o = O.tm_coeffs(30, 24, 0.05, npml=5, m_poles=mp, m_pole_masks=masks, dtype=np.float32)
    for k in ("mc1x", "mc2x", "mc3x", "mc1y", "mc2y", "mc3y"):
        np.testing.assert_allclose(getattr(m, k).numpy(), o[k], rtol=2e-6, atol=1e-7)
    s, so = init_tm_state(g, n_mpoles=2), O.tm_state(o)
    for k in ("Bx", "By", "Mx_cur", "Mx_prev", "My_cur", "My_prev"):
        assert tuple(getattr(s, k).shape) == so[k].shape, k


def test_te_tensor_coefficients_match_oracle():
    """eps_tensor: the inverse tensor Yee-averaged onto the E nodes; poles_tensor: the
    oriented pole appended to each axis stack with its off-diagonal drives."""
    from meep_torch_b200.core.coeffs import build_te_coeffs
    from meep_torch_b200.core.grid import Grid
    rng = np.random.default_rng(9)
    nx, ny = 26, 22
    exx = rng.uniform(2, 6, (nx, ny)); eyy = rng.uniform(2, 6, (nx, ny))
    exy = rng.uniform(-1, 1, (nx, ny))
    pt = [(0.7, 0.1, (0.6, 0.3, 0.4))]
    pm = [(rng.random((nx, ny)) < 0.5).astype(np.float64)]
    g = Grid(nx=nx, ny=ny, dx=0.05, device="cpu")
    T = lambda a: torch.tensor(a, dtype=torch.float32)  # noqa: E731
    m = build_te_coeffs(g, npml=4, eps_tensor=(T(exx), T(exy), T(eyy)), poles=[(0.5, 0.05, 1.0)],
                        poles_tensor=pt, pole_masks_tensor=[T(x) for x in pm])
    o = O.te_coeffs(nx, ny, 0.05, npml=4, eps_tensor=(exx, exy, eyy), poles=[(0.5, 0.05, 1.0)],
                    poles_tensor=pt, pole_masks_tensor=pm, dtype=np.float32)
    for k in ("inv_xx_x", "inv_xy_x", "inv_yy_y", "inv_xy_y", "c1x", "c2x", "c3x", "c1y",
              "c2y", "c3y", "c3xy", "c3yx"):
        np.testing.assert_allclose(getattr(m, k).numpy(), o[k], rtol=2e-5, atol=1e-7,
                                   err_msg=k)
