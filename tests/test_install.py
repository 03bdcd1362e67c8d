"""install() / uninstall(): the reference's hot-path entry points routed to this package.

A fake reference package checks the rules: modules that bound the names are patched,
routing follows the route predicate, NotImplementedError propagates unless fallback is
on, and uninstall() restores every original. When the reference itself is importable
(its checkout named by MEEP_TORCH_REF, the variable the fixture recipe reads), the real
modules are patched and restored; nothing is run through them here.
"""
import os
import sys
import types

import pytest
import torch

from meep_torch_b200 import install as I


@pytest.fixture
def fake_pkg():
    names = ["fakeref", "fakeref.core", "fakeref.core.run", "fakeref.core.monitors_3d",
             "fakeref.user"]
    mods = {n: types.ModuleType(n) for n in names}
    calls = []

    def _run_chunk(step_fn, state, coeffs, step0, k, source, monitors):
        calls.append("ref_chunk")
        return "ref"

    def run_tm(state, coeffs, n, **kw):
        calls.append("ref_tm")
        return "ref"

    def run_3d(state, coeffs, n, **kw):
        calls.append("ref_3d")
        return "ref"
    mods["fakeref.core.run"]._run_chunk = _run_chunk
    mods["fakeref.core.run"].run_tm = run_tm
    mods["fakeref.core.monitors_3d"].run_3d = run_3d
    mods["fakeref.user"].run_tm = run_tm                 # a `from ..core.run import run_tm`
    mods["fakeref.user"]._run_chunk = _run_chunk
    mods["fakeref"].core = mods["fakeref.core"]
    saved = {n: sys.modules.get(n) for n in names}
    sys.modules.update(mods)
    yield mods, calls, (_run_chunk, run_tm, run_3d)
    I.uninstall()
    for n, m in saved.items():
        if m is None:
            sys.modules.pop(n, None)
        else:
            sys.modules[n] = m


def test_install_patches_bound_names_and_restores(fake_pkg):
    mods, calls, (chunk, tm, r3) = fake_pkg
    ours = {"_run_chunk": lambda *a, **k: calls.append("ours_chunk") or "ours",
            "run_tm": lambda *a, **k: calls.append("ours_tm") or "ours",
            "run_3d": lambda *a, **k: calls.append("ours_3d") or "ours"}
    n = I.install("fakeref", ours=ours, route=lambda a, k: True)
    assert n == 5 and I.installed()
    assert mods["fakeref.user"].run_tm is mods["fakeref.core.run"].run_tm
    assert mods["fakeref.core.run"].run_tm.__wrapped__ is tm
    assert mods["fakeref.user"].run_tm(None, None, 3) == "ours"
    assert mods["fakeref.core.monitors_3d"].run_3d(None, None, 3) == "ours"
    with pytest.raises(RuntimeError):
        I.install("fakeref", ours=ours)
    assert I.uninstall() == 5 and not I.installed()
    assert mods["fakeref.core.run"].run_tm is tm and mods["fakeref.user"]._run_chunk is chunk
    assert mods["fakeref.core.monitors_3d"].run_3d is r3


def test_routing_and_fallback_rules(fake_pkg):
    mods, calls, _ = fake_pkg

    def unsupported(*a, **k):
        raise NotImplementedError("feature outside the kernels")
    I.install("fakeref", ours={"run_tm": unsupported}, route=lambda a, k: True)
    with pytest.raises(NotImplementedError):
        mods["fakeref.core.run"].run_tm(None, None, 1)
    I.uninstall()
    I.install("fakeref", ours={"run_tm": unsupported}, route=lambda a, k: True, fallback=True)
    assert mods["fakeref.core.run"].run_tm(None, None, 1) == "ref"
    I.uninstall()

    def missing_library(*a, **k):
        raise OSError("libmeep_b200.so not built")
    I.install("fakeref", ours={"run_tm": missing_library}, route=lambda a, k: True,
              fallback=True)
    with pytest.raises(OSError):                       # never swallowed
        mods["fakeref.core.run"].run_tm(None, None, 1)
    I.uninstall()
    # the default route: CPU tensors go to the reference's own function
    I.install("fakeref", ours={"run_tm": unsupported})
    st = (torch.zeros(3), torch.zeros(2))
    assert mods["fakeref.core.run"].run_tm(st, None, 1) == "ref"


def test_cuda_f32_predicate():
    assert not I.cuda_f32(((torch.zeros(2), 1),), {})
    assert not I.cuda_f32((None, 3), {})
    if torch.cuda.is_available():
        assert I.cuda_f32(((torch.zeros(2, device="cuda"),),), {})
        assert not I.cuda_f32(((torch.zeros(2, device="cuda", dtype=torch.float64),),), {})


def test_fields_method_predicate():
    """fields.solve_cw routes on the fields object's state, not on its arguments."""
    class F:
        _state = (torch.zeros(2), torch.zeros(3))
    assert not I.fields_cuda_f32((F(),), {})
    assert not I.fields_cuda_f32((), {})
    if torch.cuda.is_available():
        F._state = (torch.zeros(2, device="cuda"),)
        assert I.fields_cuda_f32((F(),), {})


def test_install_on_the_reference_package():
    from tests.golden.reference_path import find_reference
    ref = find_reference()
    if ref is None:
        pytest.skip("reference not present")
    sys.path.insert(0, ref)
    try:
        mt = pytest.importorskip("meep_torch")
        import importlib
        for m in ("meep_torch.core.run", "meep_torch.core.monitors_3d", "meep_torch.solvers",
                  "meep_torch.mp.cpp.core", "meep_torch.mp.simulation",
                  "meep_torch.core.stepper_3d_lean", "meep_torch.core.adjoint3d"):
            importlib.import_module(m)
        run_mod = sys.modules["meep_torch.core.run"]
        orig = {n: getattr(run_mod, n) for n in ("_run_chunk", "run_tm", "run_te")}
        fcls = sys.modules["meep_torch.mp.cpp.core"].fields
        orig_cw = vars(fcls)["solve_cw"]
        n = I.install("meep_torch")
        try:
            assert n >= 7
            assert getattr(vars(fcls)["solve_cw"], "_meep_b200_router", False)
            assert getattr(run_mod.run_tm, "_meep_b200_router", False)
            assert sys.modules["meep_torch.solvers"].run_tm is run_mod.run_tm
            assert getattr(sys.modules["meep_torch.mp.cpp.core"]._run_chunk,
                           "_meep_b200_router", False)
            assert getattr(sys.modules["meep_torch.mp.simulation"].run_3d,
                           "_meep_b200_router", False)
        finally:
            I.uninstall()
        for k, v in orig.items():
            assert getattr(run_mod, k) is v
        assert vars(fcls)["solve_cw"] is orig_cw
        assert mt is not None
    finally:
        sys.path.remove(ref)
