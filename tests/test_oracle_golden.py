"""Pin the numpy oracle against fixtures produced by the reference itself.

FP64: the restatement must reproduce the reference to round-off (<= 1e-10
relative L2; measured <= 1e-12). FP32: same operation order, so the residue is
float32 rounding of the transcendental profile functions (exp/cos), measured
<= 2e-7 on E fields and up to 1.4e-5 on the weak scattered Hz of the 3D case;
gated at the parity bar 1e-4.
"""
import json

import numpy as np
import pytest

from oracle import fdtd as O
from tests.conftest import load_golden, rel_l2

TOL = {"f64": 1e-10, "f32": 1e-4}
NPD = {"f64": np.float64, "f32": np.float32}


def test_cpml_profiles_match_reference():
    g = load_golden("pml")
    cases = json.loads(str(g["cases"]))
    for i, (n, npml, off, dt, dx) in enumerate(cases):
        npml = tuple(npml) if isinstance(npml, list) else npml
        for prec in ("f64", "f32"):
            b, a, k = O.cpml_profiles(n, npml, off, dt, dx, dtype=NPD[prec])
            tol = 1e-14 if prec == "f64" else 1e-6
            np.testing.assert_allclose(b, g[f"{i}_{prec}_b"], rtol=tol, atol=tol)
            np.testing.assert_allclose(a, g[f"{i}_{prec}_a"], rtol=tol, atol=tol * 10)
            np.testing.assert_array_equal(k, g[f"{i}_{prec}_k"])


def run_tm_oracle(g, prec):
    dt_np = NPD[prec]
    nx, ny, dx = int(g["nx"]), int(g["ny"]), float(g["dx"])
    poles = json.loads(str(g["poles"])) if "poles" in g else ()
    c = O.tm_coeffs(nx, ny, dx, eps=g["eps"], npml=int(g["npml"]),
                    y_pmc=bool(g["y_pmc"]), dtype=dt_np, sigma=g.get("sigma"),
                    poles=poles, pole_masks=g.get("pole_masks"), sigma_b=g.get("sigma_b"),
                    mu=g.get("mu"), chi2=g.get("chi2"), chi3=g.get("chi3"),
                    m_poles=json.loads(str(g["m_poles"])) if "m_poles" in g else (),
                    m_pole_masks=g.get("m_pole_masks"))
    mask = O.line_source_mask(nx, ny, dx, int(g["src_ix"]), int(g["src_j0"]),
                              int(g["src_j1"]), dtype=dt_np)
    prof = O.gaussian_pulse(float(g["fcen"]), float(g["fwidth"]))
    dt = c["dt"]
    freqs = g["freqs"]
    mx, my = g["monx"], g["mony"]
    mons = [
        lambda s, t: O.flux_tm_sample(s, t, dt, freqs, True, int(mx[0]), int(mx[1]), int(mx[2]), dt_np),
        lambda s, t: O.flux_tm_sample(s, t, dt, freqs, False, int(my[0]), int(my[1]), int(my[2]), dt_np),
        lambda s, t: O.dft_sample(s["Ez"], t, dt, freqs, "Ez", dt_np),
    ]
    s, acc = O.run_2d(O.tm_step, O.tm_state(c), c, int(g["n_steps"]),
                      amp_fn=lambda t: prof(O.src_time(t, dt)), mask=mask, monitors=mons)
    return c, mask, s, acc


@pytest.mark.parametrize("case", ["tm", "tm_point_pmc", "tm_sigma", "tm_poles",
                                  "tm_magnetic", "tm_nonlinear", "tm_mpoles"])
@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_tm_oracle_matches_reference(case, prec):
    g = load_golden(f"{case}_{prec}")
    c, mask, s, acc = run_tm_oracle(g, prec)
    np.testing.assert_allclose(mask, g["mask"], rtol=1e-7)
    for k in ("b_hy", "a_hy", "b_hx", "a_hx", "b_ex", "a_ex", "b_ey", "a_ey"):
        np.testing.assert_allclose(c[k], g["c_" + k], rtol=1e-6, atol=1e-6)
    names = ["Ez", "Hx", "Hy", "Dz", "psi_Ezy", "psi_Ezx", "psi_Hyx", "psi_Hxy"]
    if "s_P_cur" in g:
        names += ["P_cur", "P_prev"]
    if "s_Mx_cur" in g:
        names += ["Bx", "By", "Mx_cur", "Mx_prev", "My_cur", "My_prev"]
    for k in names:
        assert rel_l2(s[k], g["s_" + k]) < TOL[prec], k
    for a, key in zip(acc, ("acc_x", "acc_y", "acc_dft")):
        assert rel_l2(a, g[key]) < TOL[prec], key
    fx = O.line_flux(acc[0], float(g["dx"]), -1.0)
    fy = O.line_flux(acc[1], float(g["dx"]), +1.0)
    assert rel_l2(fx, g["flux_x"]) < TOL[prec]
    assert rel_l2(fy, g["flux_y"]) < TOL[prec]


def run_te_oracle(g, prec):
    dt_np = NPD[prec]
    nx, ny, dx = int(g["nx"]), int(g["ny"]), float(g["dx"])
    poles = json.loads(str(g["poles"])) if "poles" in g else ()
    c = O.te_coeffs(nx, ny, dx, eps=g["eps"], npml=int(g["npml"]), dtype=dt_np,
                    sigma=g.get("sigma"), poles=poles, pole_masks=g.get("pole_masks"),
                    sigma_b=g.get("sigma_b"), mu=g.get("mu"), chi2=g.get("chi2"),
                    chi3=g.get("chi3"), eps_tensor=g.get("eps_tensor"),
                    poles_tensor=json.loads(str(g["poles_tensor"])) if "poles_tensor" in g else (),
                    pole_masks_tensor=g.get("pole_masks_tensor"))
    mask = O.line_source_mask(nx, ny, dx, int(g["src_ix"]), int(g["src_j0"]),
                              int(g["src_j1"]), dtype=dt_np)[:, :-1]
    prof = O.gaussian_pulse(float(g["fcen"]), float(g["fwidth"]))
    dt = c["dt"]
    freqs = g["freqs"]
    mx, my = g["monx"], g["mony"]
    mons = [
        lambda s, t: O.flux_te_sample(s, t, dt, freqs, int(mx[0]), int(mx[1]), int(mx[2]), dt_np),
        lambda s, t: O.flux_tey_sample(s, t, dt, freqs, int(my[0]), int(my[1]), int(my[2]), dt_np),
        lambda s, t: O.dft_sample(s["Hz"], t, dt, freqs, "Hz", dt_np),
    ]
    s, acc = O.run_2d(O.te_step, O.te_state(c), c, int(g["n_steps"]),
                      amp_fn=lambda t: prof(O.src_time(t, dt)), mask=mask, monitors=mons)
    return c, mask, s, acc


@pytest.mark.parametrize("case", ["te", "te_sigma", "te_poles", "te_magnetic",
                                  "te_nonlinear", "te_tensor", "te_tensor_poles"])
@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_te_oracle_matches_reference(case, prec):
    g = load_golden(f"{case}_{prec}")
    c, mask, s, acc = run_te_oracle(g, prec)
    np.testing.assert_allclose(mask, g["mask"], rtol=1e-7)
    names = ["Hz", "Ex", "Ey", "Dx", "Dy", "psi_Eyx", "psi_Exy", "psi_Hzy", "psi_Hzx"]
    if "s_Px_cur" in g:
        names += ["Px_cur", "Px_prev", "Py_cur", "Py_prev"]
    for k in names:
        assert rel_l2(s[k], g["s_" + k]) < TOL[prec], k
    for a, key in zip(acc, ("acc_x", "acc_y", "acc_dft")):
        assert rel_l2(a, g[key]) < TOL[prec], key
    assert rel_l2(O.line_flux(acc[0], float(g["dx"]), +1.0), g["flux_x"]) < TOL[prec]
    assert rel_l2(O.line_flux(acc[1], float(g["dx"]), -1.0), g["flux_y"]) < TOL[prec]


def run_3d_oracle(g, prec, lean=False):
    dt_np = NPD[prec]
    nx, ny, nz, dx = int(g["nx"]), int(g["ny"]), int(g["nz"]), float(g["dx"])
    poles = json.loads(str(g["poles"])) if "poles" in g else ()
    ab = {}
    if "n_abs" in g:
        ab = dict(n_abs=int(g["n_abs"]), absorber_axes=tuple(int(a) for a in g["absorber_axes"]))
    if "pmc_axes" in g:
        ab["pmc_axes"] = tuple(int(a) for a in g["pmc_axes"])
    c = O.coeffs_3d(nx, ny, nz, dx, eps=g["eps"], npml=int(g["npml"]), dtype=dt_np,
                    sigma_d=g.get("sigma_d"), sigma_b=g.get("sigma_b"), poles=poles,
                    pole_masks=g.get("pole_masks"), **ab)
    prof = O.gaussian_pulse(float(g["fcen"]), float(g["fwidth"]))
    dt = c["dt"]
    freqs = g["freqs"]
    win = tuple(int(v) for v in g["win"])
    faces = json.loads(str(g["faces"]))
    mons = [(lambda a, i: (lambda s, t: O.flux3d_sample(s, t, dt, freqs, a, i, win=win)))(a, i)
            for a, i in faces]
    i, j, k = (int(v) for v in g["src"])
    s, acc = O.run_3d(O.state_3d(c), c, int(g["n_steps"]),
                      amp_fn=lambda t: prof(O.src_time(t, dt)), src=("Ez", i, j, k),
                      monitors=mons, point_sign=-1.0 if lean else 1.0)
    return c, s, acc


@pytest.mark.parametrize("case", ["3d", "3d_sigma", "3d_poles", "3d_abs", "3d_mixed",
                                  "3d_pmc"])
@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_3d_oracle_matches_reference(case, prec):
    """3D cases; 3d_abs runs the matched-sigma absorber on every face (no CPML, so
    the reference state carries no CPML memory), 3d_mixed the absorber on z beside
    x / y CPML, 3d_pmc PMC walls on y beside x / z CPML."""
    g = load_golden(f"{case}_{prec}")
    c, s, acc = run_3d_oracle(g, prec)
    names = ["Ex", "Ey", "Ez", "Hx", "Hy", "Hz"]
    names += [k for k in ("psi_Ez_y", "psi_Hx_y", "psi_Hz_x") if "s_" + k in g]
    names += [k[2:] for k in g if k.startswith("s_P")]
    for k in names:
        assert rel_l2(s[k], g["s_" + k]) < TOL[prec], k
    for n, a in enumerate(acc):
        assert rel_l2(a, g[f"acc_{n}"]) < TOL[prec]
        assert rel_l2(O.flux3d(a, float(g["dx"])), g[f"flux_{n}"]) < TOL[prec]


@pytest.mark.parametrize("case", ["3d_lean", "3d_lean_poles"])
@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_3d_lean_sign_convention(case, prec):
    """The lean stepper subtracts the point current and multiplies by 1/eps;
    the oracle's point_sign=-1 reproduces it to the rounding of that form. With
    poles the lean stepper's folded-D update is the functional stepper's."""
    g = load_golden(f"{case}_{prec}")
    c, s, acc = run_3d_oracle(g, prec, lean=True)
    tol = 1e-9 if prec == "f64" else 1e-4
    for k in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz"):
        assert rel_l2(s[k], g["s_" + k]) < tol, k
    for n, a in enumerate(acc):
        assert rel_l2(a, g[f"acc_{n}"]) < tol


@pytest.mark.parametrize("case", ["grad_tm", "grad_tm_lossy", "grad_tm_poles", "grad_tm_pmc",
                                  "grad_tm_mirror", "grad_tm_mirror_odd", "grad_tm_rot2",
                                  "grad_tm_rot4", "grad_tm_mpoles"])
def test_reference_gradient_matches_oracle_finite_differences(case):
    """The golden d J / d eps (reference autograd, float64) against central
    finite differences of the oracle's float64 run at a few pixels; the lossy case
    adds sigma_d, sigma_b and mu, the dispersive one a Lorentz and a Drude pole, the
    mirror ones even / odd mirror cuts on the low edges, the rotation ones an odd Rotate2
    / Rotate4 (pixels on the cuts are probed; the loss adds the final on-plane lines)."""
    g = load_golden(f"{case}_f64")
    extra = dict(sigma=g.get("sigma"), sigma_b=g.get("sigma_b"), mu=g.get("mu"),
                 y_pmc=bool(g.get("y_pmc", 0)))
    if "poles" in g:
        extra.update(poles=json.loads(str(g["poles"])), pole_masks=g["pole_masks"])
    if "fold" in g:
        extra.update(json.loads(str(g["fold"])))
    if "m_poles" in g:
        extra.update(m_poles=[tuple(p) for p in json.loads(str(g["m_poles"]))],
                     m_pole_masks=g["m_pole_masks"])
    nx, ny, dx, npml, n = (int(g["nx"]), int(g["ny"]), float(g["dx"]), int(g["npml"]),
                           int(g["n_steps"]))
    freqs = [float(f) for f in g["freqs"]]
    mxi, mxl, mxh = (int(v) for v in g["monx"])
    myi, myl, myh = (int(v) for v in g["mony"])

    def J_of(eps):
        c = O.tm_coeffs(nx, ny, dx, eps=eps, npml=npml, dtype=np.float64, **extra)
        dt = c["dt"]
        mask = O.line_source_mask(nx, ny, dx, int(g["src_ix"]), int(g["src_j0"]),
                                  int(g["src_j1"]), dtype=np.float64)
        prof = O.gaussian_pulse(float(g["fcen"]), float(g["fwidth"]))
        mons = [lambda s, t: O.flux_tm_sample(s, t, dt, freqs, True, mxi, mxl, mxh, np.float64),
                lambda s, t: O.flux_tm_sample(s, t, dt, freqs, False, myi, myl, myh, np.float64),
                lambda s, t: O.dft_sample(s["Ez"], t, dt, freqs, "Ez", np.float64)]
        s, (ax, ay, ad) = O.run_2d(O.tm_step, O.tm_state(c), c, n,
                                   amp_fn=lambda t: prof(O.src_time(t, dt)), mask=mask,
                                   monitors=mons)
        w = np.array([1.0, -0.5, 0.25])
        fx, fy = O.line_flux(ax, dx, -1.0), O.line_flux(ay, dx, +1.0)
        return float((w * fx).sum() + (w[::-1] * fy).sum() + 1e-3 * (ad * ad).sum()
                     + 0.1 * (s["Ez"] ** 2).sum() + 0.05 * (s["Hy"] ** 2).sum()
                     - 0.02 * (s["Hx"] ** 2).sum()
                     + sum(c * (s[k] ** 2).sum() for k, c in (("Hx0", 0.3), ("Hy0", -0.2))
                           if k in s))

    eps = g["eps"].astype(np.float64)
    assert abs(J_of(eps) - float(g["J"])) <= 1e-9 * abs(float(g["J"]))
    h = 1e-4
    cells = [(33, 24), (24, 17), (36, 12)] + ([(0, 14), (10, 0), (0, 0)] if "fold" in g else [])
    for (i, j) in cells:
        ep, em = eps.copy(), eps.copy()
        ep[i, j] += h
        em[i, j] -= h
        fd = (J_of(ep) - J_of(em)) / (2 * h)
        ref = float(g["grad"][i, j])
        assert abs(fd - ref) <= 1e-5 * abs(ref) + 1e-16, (i, j, fd, ref)


@pytest.mark.parametrize("case", ["grad3d", "grad3d_sigma", "grad3d_poles", "grad3d_pmc"])
def test_reference_3d_gradient_matches_oracle_finite_differences(case):
    """The golden d J / d eps of run_3d_adjoint (float64) against central finite
    differences of the oracle's float64 3D run at two cells; the sigma case adds a
    lossy slab (sigma_d) and a magnetically lossy patch (sigma_b), the poles case a
    Lorentz and a Drude pole on two boxes (cells inside both are probed), the pmc case
    PMC walls on y (cells on and next to the wall are probed)."""
    g = load_golden(f"{case}_f64")
    n, dx, npml, steps = int(g["n"]), float(g["dx"]), int(g["npml"]), int(g["n_steps"])
    freqs = [float(f) for f in g["freqs"]]
    si, sj, sk = (int(v) for v in g["src"])
    prof = O.gaussian_pulse(float(g["fcen"]), float(g["fwidth"]))
    w = np.array([1.0, -0.7, 0.4])

    def J_of(eps):
        kw = {}
        if "poles" in g:
            kw = dict(poles=[tuple(p) for p in json.loads(str(g["poles"]))],
                      pole_masks=[g["pm0"], g["pm1"]])
        if "pmc_axes" in g:
            kw = dict(pmc_axes=tuple(int(a) for a in g["pmc_axes"]))
        c = O.coeffs_3d(n, n, n, dx, eps=eps, npml=npml, dtype=np.float64,
                        sigma_d=g.get("sigma_d"), sigma_b=g.get("sigma_b"), **kw)
        dt = c["dt"]
        mons = [lambda s, t: O.flux3d_sample(s, t, dt, freqs, "x", 15, (5, 15, 5, 15)),
                lambda s, t: O.flux3d_sample(s, t, dt, freqs, "z", 6, (5, 15, 5, 15))]
        _, (a0, a1) = O.run_3d(O.state_3d(c), c, steps, amp_fn=lambda t: prof(O.src_time(t, dt)),
                               src=("Ez", si, sj, sk), monitors=mons)
        return 1e15 * float((w * O.flux3d(a0, dx)).sum() + (w[::-1] * O.flux3d(a1, dx)).sum()
                            + 1e-3 * ((a0 * a0).sum() + (a1 * a1).sum()))

    eps = g["eps"].astype(np.float64)
    assert abs(J_of(eps) - float(g["L"])) <= 1e-9 * abs(float(g["L"]))
    h = 1e-4
    cells = [(12, 9, 11), (14, 12, 8)] + ([(9, 7, 10), (12, 11, 8)] if "poles" in g else []) \
        + ([(10, 0, 11), (11, 1, 10), (9, 19, 12)] if "pmc_axes" in g else [])
    for (i, j, k) in cells:
        ep, em = eps.copy(), eps.copy()
        ep[i, j, k] += h
        em[i, j, k] -= h
        fd = (J_of(ep) - J_of(em)) / (2 * h)
        ref = float(g["grad"][i, j, k])
        assert abs(fd - ref) <= 1e-5 * abs(ref) + 1e-12, (i, j, k, fd, ref)


@pytest.mark.parametrize("case", ["grad_te", "grad_te_lossy", "grad_te_poles", "grad_te_mirror",
                                  "grad_te_mirror_even"])
def test_reference_te_gradient_matches_oracle_finite_differences(case):
    """The golden TE d J / d eps_inf (reference autograd, float64) against central
    finite differences of the oracle's float64 TE run at two pixels; the lossy case adds
    sigma_d, sigma_b and mu, the dispersive one a Lorentz and a Drude pole on both E
    axes, the mirror one odd mirror cuts on the low edges (pixels on the cuts probed)."""
    g = load_golden(f"{case}_f64")
    extra = dict(sigma=g.get("sigma"), sigma_b=g.get("sigma_b"), mu=g.get("mu"))
    if "poles" in g:
        extra.update(poles=json.loads(str(g["poles"])), pole_masks=g["pole_masks"])
    if "fold" in g:
        extra.update(json.loads(str(g["fold"])))
    if "m_poles" in g:
        extra.update(m_poles=[tuple(p) for p in json.loads(str(g["m_poles"]))],
                     m_pole_masks=g["m_pole_masks"])
    nx, ny, dx, npml, n = (int(g["nx"]), int(g["ny"]), float(g["dx"]), int(g["npml"]),
                           int(g["n_steps"]))
    freqs = [float(f) for f in g["freqs"]]
    mxi, mxl, mxh = (int(v) for v in g["monx"])
    myi, myl, myh = (int(v) for v in g["mony"])

    def J_of(eps):
        c = O.te_coeffs(nx, ny, dx, eps=eps, npml=npml, dtype=np.float64, **extra)
        dt = c["dt"]
        mask = O.line_source_mask(nx, ny, dx, int(g["src_ix"]), int(g["src_j0"]),
                                  int(g["src_j1"]), dtype=np.float64)[:, :-1]
        prof = O.gaussian_pulse(float(g["fcen"]), float(g["fwidth"]))
        mons = [lambda s, t: O.dft_sample(s["Hz"], t, dt, freqs, "Hz", np.float64),
                lambda s, t: O.flux_te_sample(s, t, dt, freqs, mxi, mxl, mxh, np.float64),
                lambda s, t: O.flux_tey_sample(s, t, dt, freqs, myi, myl, myh, np.float64)]
        s, (ad, ax, ay) = O.run_2d(O.te_step, O.te_state(c), c, n,
                                   amp_fn=lambda t: prof(O.src_time(t, dt)), mask=mask,
                                   monitors=mons)
        w = np.array([1.0, -0.5, 0.25])
        fx, fy = O.line_flux(ax, dx, +1.0), O.line_flux(ay, dx, -1.0)
        return 1e6 * float((w * fx).sum() + (w[::-1] * fy).sum() + 1e-3 * (ad * ad).sum()
                           + 0.1 * (s["Hz"] ** 2).sum() + 0.05 * (s["Ex"] ** 2).sum()
                           - 0.02 * (s["Ey"] ** 2).sum())

    eps = g["eps"].astype(np.float64)
    assert abs(J_of(eps) - float(g["J"])) <= 1e-9 * abs(float(g["J"]))
    h = 1e-4
    for (i, j) in [(30, 26), (20, 18)] + ([(0, 15), (12, 0)] if "fold" in g else []):
        ep, em = eps.copy(), eps.copy()
        ep[i, j] += h
        em[i, j] -= h
        fd = (J_of(ep) - J_of(em)) / (2 * h)
        ref = float(g["grad"][i, j])
        assert abs(fd - ref) <= 1e-5 * abs(ref) + 1e-12, (i, j, fd, ref)


FOLD_CASES = [("tm", n) for n in ("ym_even", "ym_odd", "xm_even", "xm_odd_ym_even", "rot2_even",
                                  "rot2_odd", "rot4_even", "rot4_odd")] + \
    [("te", n) for n in ("ym_even_xm_odd", "ym_odd_xm_even")]


@pytest.mark.parametrize("pol,name", FOLD_CASES)
@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_fold_oracle_matches_reference(pol, name, prec):
    """Symmetry-folded runs (mirrors, Rotate2, Rotate4 cuts on the low edges): every
    state array, the on-plane H rows of odd / rotated cuts included, and the DFT
    accumulator match the reference's own run."""
    g = load_golden(f"{pol}_fold_{name}_{prec}")
    dt_np = NPD[prec]
    nx, ny, dx = int(g["nx"]), int(g["ny"]), float(g["dx"])
    fold = json.loads(str(g["fold"]))
    make = O.tm_coeffs if pol == "tm" else O.te_coeffs
    c = make(nx, ny, dx, eps=g["eps"], npml=int(g["npml"]), dtype=dt_np, **fold)
    mask = O.line_source_mask(nx, ny, dx, int(g["src_ix"]), int(g["src_j0"]), int(g["src_j1"]),
                              dtype=dt_np)
    if pol == "te":
        mask = mask[:, :-1]
    np.testing.assert_allclose(mask, g["mask"], rtol=1e-7)
    prof = O.gaussian_pulse(float(g["fcen"]), float(g["fwidth"]))
    dt = c["dt"]
    comp = "Ez" if pol == "tm" else "Hz"
    mon = lambda s, t: O.dft_sample(s[comp], t, dt, g["freqs"], comp, dt_np)  # noqa: E731
    state0 = O.tm_state(c) if pol == "tm" else O.te_state(c)
    s, (acc,) = O.run_2d(O.tm_step if pol == "tm" else O.te_step, state0, c, int(g["n_steps"]),
                         amp_fn=lambda t: prof(O.src_time(t, dt)), mask=mask, monitors=[mon])
    keys = [k[2:] for k in g if k.startswith("s_") and not k.startswith("s_P")]
    assert ("Hx0" in keys) == ("Hx0" in s) and ("Hy0" in keys) == ("Hy0" in s)
    for k in keys:
        assert s[k].shape == g["s_" + k].shape, k
        assert rel_l2(s[k], g["s_" + k]) < TOL[prec], k
    assert rel_l2(acc, g["acc_dft"]) < TOL[prec]


def test_cw_operator_and_solve_match_reference():
    """meep's CW solve on a 2D TM cell: the oracle's operator A x = (step(x) - x)/dt +
    i Omega x matches the reference's on seeded random vectors (FP64 rounding), its
    right-hand side matches, and its BiCGSTAB(2) reaches the reference's solution
    (both stop at |r| <= 1e-8 |b|) in about the same number of iterations."""
    g = load_golden("cw_tm_f64")
    nx, ny, dx = int(g["nx"]), int(g["ny"]), float(g["dx"])
    c = O.tm_coeffs(nx, ny, dx, eps=g["eps"], npml=int(g["npml"]), dtype=np.float64)
    names, pack, unpack, A = O.cw_tm(c, float(g["freq"]))
    assert list(names) == json.loads(str(g["names"]))
    def crel(a, r):                                  # complex relative L2
        return float(np.linalg.norm(np.asarray(a) - r) / np.linalg.norm(r))
    for v, av in (("v0", "Av0"), ("v1", "Av1")):
        assert crel(A(g[v]), g[av]) < 1e-12, v
    mask = O.line_source_mask(nx, ny, dx, int(g["src_ix"]), int(g["src_j0"]), int(g["src_j1"]))
    np.testing.assert_allclose(mask, g["mask"], rtol=1e-12)
    b = O.cw_rhs_tm(c, names, pack, 1.0 + 0.0j, mask)
    assert crel(b, g["b"]) < 1e-14
    x = np.zeros_like(b)
    ierr, it = O.bicgstab_l(2, A, b, x, tol=1e-8, maxiters=5000)
    assert ierr == 0 and abs(it - int(g["iters"])) <= max(5, int(g["iters"]) // 10)
    assert float(np.linalg.norm(A(x) - b)) <= 1e-8 * float(np.linalg.norm(b)) * 1.01
    re, im = unpack(x)
    for k in list(names) + ["Ez"]:
        if re[k].size:
            assert rel_l2(re[k], g["re_" + k]) < 1e-6, k
            assert rel_l2(im[k], g["im_" + k]) < 1e-6, k
