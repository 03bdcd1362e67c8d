"""The CW (frequency-domain) solve on the kernels against the reference's own
``fields.solve_cw`` (mp/cpp/core.py:666-778), from the fixture ``golden_cw_tm_f64`` (a
40 x 30 TM cell with a guide, f = 0.6; seeded random vectors, the reference's right-hand
side and its BiCGSTAB(2) solution at |r| <= 1e-8 |b|, all in float64). The operator is
checked against the oracle's float64 operator, which the oracle tests pin to the
reference's own on the same vectors to 1e-12.

The kernels step in float32, so the operator is compared at float32 precision and the
solve stops at a float32-reachable residual; the solution is checked against the
reference's float64 solution and its residual under the float64 operator of the oracle
(which the oracle tests pin to the reference's to 1e-12).
"""
import json

import numpy as np
import pytest
import torch

import oracle.fdtd as O
from tests.conftest import load_golden, rel_l2

pytestmark = pytest.mark.gpu

OP_TOL = 1e-4


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")


def _crel(a, r):
    return float(np.linalg.norm(np.asarray(a) - r) / np.linalg.norm(r))


def _setup():
    from meep_torch_b200.core.coeffs import build_tm_coeffs
    from meep_torch_b200.core.grid import Grid
    from meep_torch_b200.core.stepper_tm import init_tm_state
    from meep_torch_b200.cw import CWOperator
    g = load_golden("cw_tm_f64")
    grid = Grid(nx=int(g["nx"]), ny=int(g["ny"]), dx=float(g["dx"]), device="cuda")
    m = build_tm_coeffs(grid, eps_inf=torch.tensor(g["eps"], dtype=torch.float32),
                        npml=int(g["npml"]))
    st = init_tm_state(grid)
    op = CWOperator(st, m, float(g["freq"]))
    return g, m, st, op, json.loads(str(g["names"]))


def _states(st, m, names, v):
    """(real, imaginary) states of a packed complex vector, Ez = (Dz - sum P) / eps."""
    parts = [{}, {}]
    i = 0
    for k in names:
        shape = tuple(getattr(st, k).shape)
        n = int(np.prod(shape))
        c = np.asarray(v[i:i + n])
        i += n
        for p, arr in zip(parts, (c.real, c.imag)):
            p[k] = torch.tensor(arr.reshape(shape), dtype=torch.float32, device="cuda")
    out = []
    for p in parts:
        p["Ez"] = (p["Dz"] - p["P_cur"].sum(0)) / m.eps_inf
        out.append(st._replace(**p))
    return out


def _packed(re, im, names):
    r = np.concatenate([getattr(re, k).double().cpu().numpy().ravel() for k in names])
    i = np.concatenate([getattr(im, k).double().cpu().numpy().ravel() for k in names])
    return r + 1j * i


def _outside_zeroed(st, m, names, v):
    """v with the CPML memory zeroed where its profile is inert (b = 1, a = 0). The
    kernels keep that memory at zero (a Krylov space started from zero fields never
    fills it: nothing but itself feeds it), so the operator is compared on that
    subspace."""
    def inert(b, a):
        return ((b.reshape(-1) == 1) & (a.reshape(-1) == 0)).cpu().numpy()
    where = {"psi_Ezy": (None, inert(m.b_hy, m.a_hy)), "psi_Ezx": (inert(m.b_hx, m.a_hx), None),
             "psi_Hyx": (inert(m.b_ex, m.a_ex), None), "psi_Hxy": (None, inert(m.b_ey, m.a_ey))}
    v = np.array(v, copy=True)
    i = 0
    for k in names:
        shape = tuple(getattr(st, k).shape)
        n = int(np.prod(shape))
        if k in where:
            rows, cols = where[k]
            blk = v[i:i + n].reshape(shape)
            if rows is not None:
                blk[rows, :] = 0
            if cols is not None:
                blk[:, cols] = 0
        i += n
    return v


def test_cw_operator_matches_reference():
    """A x on the kernels (both parts in one launch) against the float64 operator on
    seeded random vectors (the fixture's, CPML memory outside the layers zeroed)."""
    g, m, st, op, names = _setup()
    c64 = O.tm_coeffs(int(g["nx"]), int(g["ny"]), float(g["dx"]), eps=g["eps"],
                      npml=int(g["npml"]), dtype=np.float64)
    _, _, _, A64 = O.cw_tm(c64, float(g["freq"]))
    try:
        for v in ("v0", "v1"):
            vz = _outside_zeroed(st, m, names, g[v])
            re, im = _states(st, m, names, vz)
            x = op.from_states(re, im)
            r2, i2 = op.to_states(x)                 # the layout round trip is exact
            for k in names:
                assert torch.equal(getattr(r2, k), getattr(re, k)), k
                assert torch.equal(getattr(i2, k), getattr(im, k)), k
            y = op(x)
            e = _crel(_packed(*op.to_states(y), names), A64(vz))
            print(f"\n[cw] A {v}: relL2 vs the float64 operator {e:.2e}")
            assert e < OP_TOL, (v, e)
    finally:
        op.close()


def test_cw_rhs_and_solve_match_reference():
    """b from a unit source, BiCGSTAB(2) on the kernels, the solution against the
    reference's and its residual under the float64 operator."""
    from meep_torch_b200.cw import bicgstab_l
    g, m, st, op, names = _setup()
    mask = torch.tensor(g["mask"], dtype=torch.float32, device="cuda")

    class Unit:                                      # a unit CW current on the mask
        pass
    src = Unit()
    src.mask = mask
    src.amplitude = lambda t: 1.0
    try:
        b = op.rhs([src], 0)
        assert _crel(_packed(*op.to_states(b), names), g["b"]) < 1e-6
        x = op.zeros()
        ierr, iters = bicgstab_l(op, b, x, L=2, tol=1e-5, maxiters=4000)
        re, im = op.to_states(x)
        errs = {k: max(rel_l2(getattr(re, k).cpu().numpy(), g["re_" + k]),
                       rel_l2(getattr(im, k).cpu().numpy(), g["im_" + k]))
                for k in list(names) + ["Ez"] if getattr(re, k).numel()}
        c64 = O.tm_coeffs(int(g["nx"]), int(g["ny"]), float(g["dx"]), eps=g["eps"],
                          npml=int(g["npml"]), dtype=np.float64)
        _, pack64, _, A64 = O.cw_tm(c64, float(g["freq"]))
        xs = _packed(re, im, names)
        res = float(np.linalg.norm(A64(xs) - g["b"]) / np.linalg.norm(g["b"]))
        print(f"\n[cw solve] ierr {ierr}, {iters} iterations ({op.matvecs} matvecs); "
              f"true residual (float64 operator) {res:.2e}; solution relL2 vs the reference "
              f"max {max(errs.values()):.2e} ({max(errs, key=errs.get)})")
        assert ierr == 0
        assert res < 1e-4
        assert max(errs.values()) < 1e-3, errs
    finally:
        op.close()
