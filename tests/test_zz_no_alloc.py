"""The allocation-free entry point, mtb_yee2d_run_noalloc, against the plan path.

Some callers cannot call cudaMalloc, e.g. a host that hands the library a
fixed device-memory budget, or a latency-critical loop that cannot take
cudaMalloc's device synchronisation. For them, mtb_yee2d_run_noalloc runs one
2D structure with all of its scratch in one fixed-size device array. This
test drives it through the C ABI on the same inputs as mtb_yee2d_plan_create
+ mtb_yee2d_run, for two calls in a row (the second continuing the first,
with the time index and ping-pong buffer carried over; the second call is
longer than the entry point's 256-step table chunk, so a chunk boundary is
crossed), and compares fields and DFT/flux accumulators within the parity
tolerance used elsewhere (1e-4 relative L2). It also checks the property the
entry point exists for: once the library is loaded and the first call has
done its one-time set-up, a call leaves the device's free memory unchanged.
Calls the entry point rejects leave the caller's arrays untouched. The file is
named so pytest collects it last.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from tests.conftest import rel_l2

pytestmark = pytest.mark.gpu
TOL = 1e-4


def _items(pol, device):
    from meep_torch_b200.core.coeffs import build_te_coeffs, build_tm_coeffs
    from meep_torch_b200.core.grid import Grid
    from meep_torch_b200.core.monitors import (DFTFieldsMonitor, FluxMonitorTE, FluxMonitorTEY,
                                               FluxMonitorTM)
    from meep_torch_b200.core.sources import GaussianPulse, LineSource, TESource
    from meep_torch_b200.core.stepper_te import init_te_state
    from meep_torch_b200.core.stepper_tm import init_tm_state
    rng = np.random.default_rng(21)
    nx, ny = 150, 261
    eps = np.ones((nx, ny), dtype=np.float32)
    eps[:, 120:140] = 12.0
    eps[60:90, 40:80] = rng.uniform(2, 10, (30, 40))
    g = Grid(nx=nx, ny=ny, dx=0.05, device=device)
    src = LineSource(g, ix=30, j0=115, j1=145, profile=GaussianPulse(0.65, 0.3))
    freqs = [0.55, 0.65, 0.75]
    e = torch.from_numpy(eps)
    if pol == "tm":
        m = build_tm_coeffs(g, eps_inf=e, npml=12)
        mons = [DFTFieldsMonitor(g, freqs, "Ez"),
                FluxMonitorTM(g, freqs, x_normal=True, idx=110, lo=100, hi=160),
                FluxMonitorTM(g, freqs, x_normal=False, idx=200, lo=20, hi=130)]
        return init_tm_state(g), m, src, mons
    m = build_te_coeffs(g, eps_inf=e, npml=12)
    mons = [DFTFieldsMonitor(g, freqs, "Hz"),
            FluxMonitorTE(g, freqs, ix=110, lo=100, hi=160),
            FluxMonitorTEY(g, freqs, iy=200, lo=20, hi=130)]
    return init_te_state(g), m, TESource(src), mons


def _coefs(eng, t0, k):
    """The per-step coefficient columns the engine hands mtb_yee2d_run."""
    from meep_torch_b200.engine2d import coef_table
    ce = ch = None
    for col, src, attr, dt, kind in eng._amp_sources:
        assert col == 0
        v = np.ascontiguousarray(coef_table(src, attr, t0, k, dt))
        if kind == "e":
            ce = v
        else:
            ch = v
    return ce, ch


@pytest.mark.parametrize("pol", ["tm", "te"])
def test_noalloc_matches_plan_two_calls(pol):
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    from meep_torch_b200 import _lib as L
    from meep_torch_b200 import build
    from meep_torch_b200.engine2d import Engine2D
    build.build()
    lib = L.load()
    dev = "cuda"
    # the no-alloc entry point runs the row-march kernels: the plan path is
    # pinned to the same kernels (variant 1), so the comparison is of the
    # entry points, not of two kernels' rounding
    ref = Engine2D([_items(pol, dev)], ring_slots=8, variant=1)   # plan path
    new = Engine2D([_items(pol, dev)], ring_slots=8, variant=1)   # buffers for the no-alloc call
    stream = torch.cuda.current_stream().cuda_stream
    parity = 0
    t0 = 0
    for k in (70, 300):                                   # two calls in a row
        ref.run(t0, k)
        ce, ch = _coefs(new, t0, k)
        pe = ce.ctypes.data_as(C.POINTER(C.c_double)) if ce is not None else None
        ph = ch.ctypes.data_as(C.POINTER(C.c_double)) if ch is not None else None
        rc = lib.mtb_yee2d_run_noalloc(new.structs, new.regions, new.n_regions, new.groups,
                                       new.n_groups, new.ring_elems, 8, parity, t0, k, pe, ph,
                                       stream)
        L.check(rc, "mtb_yee2d_run_noalloc")
        parity ^= k & 1
        t0 += k
        torch.cuda.synchronize()
        assert ref.current == parity
        st_ref = ref.state(0)
        # the no-alloc call does not move the second engine's plan parity; read
        # its buffers at the parity it reports
        new_plan_par = new.current
        if new_plan_par != parity:
            for it in new.items:
                for key in ("main", "x", "y"):
                    it.box[key].reverse()
                for pr in it.box["psi"]:
                    pr.reverse()
        st_new = new.state(0)
        if new_plan_par != parity:
            for it in new.items:
                for key in ("main", "x", "y"):
                    it.box[key].reverse()
                for pr in it.box["psi"]:
                    pr.reverse()
        for name in st_ref._fields:
            a, b = getattr(st_new, name), getattr(st_ref, name)
            if isinstance(a, torch.Tensor) and a.numel():
                assert rel_l2(a.cpu().numpy(), b.cpu().numpy()) < TOL, (pol, t0, name)
        for a, b in zip(new.accumulators(0), ref.accumulators(0)):
            assert rel_l2(a.cpu().numpy(), b.cpu().numpy()) < TOL, (pol, t0)
    ref.close()
    new.close()


def _snapshot(eng):
    """Copies of every device array a call may write: fields, CPML memory, accumulators."""
    out = []
    for it in eng.items:
        for key in ("main", "x", "y"):
            out += [t.clone() for t in it.box[key]]
        for pr in it.box["psi"]:
            out += [t.clone() for t in pr]
    out += [a.clone() for a in eng.accumulators(0)]
    return out


def _same(a, b):
    return all(torch.equal(x, y) for x, y in zip(a, b))


def test_noalloc_allocates_nothing():
    """After a first call (which may do the one-time set-up), further calls leave
    the device's free memory exactly where it was."""
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    from meep_torch_b200 import _lib as L
    from meep_torch_b200.engine2d import Engine2D
    lib = L.load()
    eng = Engine2D([_items("tm", "cuda")], ring_slots=8, variant=1)
    stream = torch.cuda.current_stream().cuda_stream
    parity = eng.current
    ce, ch = _coefs(eng, 0, 600)

    def call(t, k):
        ph = (ch[t:].ctypes.data_as(C.POINTER(C.c_double)) if ch is not None else None)
        rc = lib.mtb_yee2d_run_noalloc(eng.structs, eng.regions, eng.n_regions, eng.groups,
                                       eng.n_groups, eng.ring_elems, 8, parity ^ (t & 1), t, k,
                                       ce[t:].ctypes.data_as(C.POINTER(C.c_double)), ph,
                                       stream)
        L.check(rc, "mtb_yee2d_run_noalloc")

    call(0, 20)                                           # warm-up: one-time set-up
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    call(20, 300)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)
    eng.close()


def test_noalloc_rejects_bad_row_ptr_before_any_step():
    """A source row_ptr that does not start at 0 is refused, and the state is untouched:
    the check runs on the device and its verdict is read back before any step kernel."""
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    from meep_torch_b200 import _lib as L
    from meep_torch_b200 import engine2d
    lib = L.load()
    ok = engine2d.Engine2D([_items("tm", "cuda")], ring_slots=8, variant=1)
    it = ok.items[0]
    row_ptr, col, w = engine2d._cells(it.source.mask, it.nx, "cuda")
    bad_rp = row_ptr.clone()
    bad_rp[0] = 5                                         # rp[0] != 0: the list is malformed
    S = ok.structs[0]
    S.src_e.row_ptr, S.src_e.col, S.src_e.w = (L.ptr(t) for t in (bad_rp, col, w))
    stream = torch.cuda.current_stream().cuda_stream
    ce, _ = _coefs(ok, 0, 4)
    before = _snapshot(ok)
    rc = lib.mtb_yee2d_run_noalloc(ok.structs, ok.regions, ok.n_regions, ok.groups,
                                   ok.n_groups, ok.ring_elems, 8, ok.current, 0, 4,
                                   ce.ctypes.data_as(C.POINTER(C.c_double)), None, stream)
    assert rc == L.MTB_INVALID_ARG
    assert b"row_ptr" in lib.mtb_last_error()
    torch.cuda.synchronize()
    assert _same(before, _snapshot(ok))
    del bad_rp, row_ptr, col, w
    ok.close()


def test_noalloc_rejects_oversize():
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    from meep_torch_b200 import _lib as L
    from meep_torch_b200.engine2d import Engine2D
    lib = L.load()
    eng = Engine2D([_items("tm", "cuda")], ring_slots=8)
    stream = torch.cuda.current_stream().cuda_stream
    # a ring far beyond the fixed array is refused before any device work
    rc = lib.mtb_yee2d_run_noalloc(eng.structs, eng.regions, eng.n_regions, eng.groups,
                                   eng.n_groups, 5_000_000, 1, 0, 0, 1, None, None, stream)
    assert rc == L.MTB_INVALID_ARG
    assert b"scratch" in lib.mtb_last_error()
    eng.close()



def _reversed_rows(cells):
    """A CSR source list with each row's columns (and weights) in descending order."""
    row_ptr, col, w = cells
    rp = row_ptr.cpu().tolist()
    col, w = col.clone(), w.clone()
    for r in range(len(rp) - 1):
        if rp[r + 1] - rp[r] > 1:
            col[rp[r]:rp[r + 1]] = col[rp[r]:rp[r + 1]].flip(0)
            w[rp[r]:rp[r + 1]] = w[rp[r]:rp[r + 1]].flip(0)
    return row_ptr, col, w


def test_source_columns_must_ascend(monkeypatch):
    """The kernels binary-search a row's source columns, so both entry points refuse
    a row whose columns descend: the plan before any device work, the
    allocation-free call with MTB_INVALID_ARG once its set-up kernel has flagged it,
    before any step kernel, so the state is untouched (every search probe stays inside
    the row's cell range either way)."""
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    from meep_torch_b200 import _lib as L
    from meep_torch_b200 import engine2d
    lib = L.load()
    orig = engine2d._cells
    ok = engine2d.Engine2D([_items("tm", "cuda")], ring_slots=8)
    monkeypatch.setattr(engine2d, "_cells", lambda m, n, d: _reversed_rows(orig(m, n, d)))
    with pytest.raises(ValueError, match="ascending"):
        engine2d.Engine2D([_items("tm", "cuda")], ring_slots=8)
    it = ok.items[0]
    bad = _reversed_rows(orig(it.source.mask, it.nx, "cuda"))
    S = ok.structs[0]
    S.src_e.row_ptr, S.src_e.col, S.src_e.w = (L.ptr(t) for t in bad)
    stream = torch.cuda.current_stream().cuda_stream
    ce, _ = _coefs(ok, 0, 4)
    pe = ce.ctypes.data_as(C.POINTER(C.c_double))
    before = _snapshot(ok)
    rc = lib.mtb_yee2d_run_noalloc(ok.structs, ok.regions, ok.n_regions, ok.groups,
                                   ok.n_groups, ok.ring_elems, 8, ok.current, 0, 4, pe, None,
                                   stream)
    assert rc == L.MTB_INVALID_ARG
    assert b"ascending" in lib.mtb_last_error()
    torch.cuda.synchronize()
    assert _same(before, _snapshot(ok))                   # rejected before any step kernel
    del bad
    ok.close()
