"""Route the reference's hot-path entry points to this package (the Python drop-in).

``install()`` replaces, inside an imported ``meep_torch`` package, the functions the
reference's step loop enters through, each with a router:

========================================  ==============================================
reference (module : name)                 this package
========================================  ==============================================
``core.run : _run_chunk`` (:10-40)        ``meep_torch_b200.core.run._run_chunk``
``core.run : run_tm`` / ``run_te``        ``meep_torch_b200.core.run.run_tm`` / ``run_te``
``core.monitors_3d : run_3d`` (:192)      ``meep_torch_b200.core.monitors_3d.run_3d``
``core.stepper_3d_lean : run_3d_lean``    ``meep_torch_b200.core.stepper_3d_lean.run_3d_lean``
``core.adjoint3d : run_3d_adjoint``       ``meep_torch_b200.core.adjoint3d.run_3d_adjoint``
``mp.cpp.core : fields.solve_cw``         ``meep_torch_b200.cw.solve_cw_fields``
========================================  ==============================================

Modules that bound one of these names by ``from ... import`` (``mp/cpp/core.py``,
``mp/simulation.py``, ``solvers.py``, ``ports/smatrix.py``) are patched too: every
loaded module of the package whose attribute *is* the original function gets the
router. ``uninstall()`` puts every original back.

A router sends a call to this package when its field arrays are float32 CUDA tensors
and to the reference's own function otherwise (this package has no CPU path). With
``fallback=True`` a NotImplementedError from this package (a feature outside the
kernels) sends the call to the reference's function instead of propagating. A
missing or unloadable CUDA library is never caught: it fails loudly either way.
"""
from __future__ import annotations

import importlib
import sys

import torch

__all__ = ["install", "uninstall", "installed"]

# (reference module, function name, this package's module, its function name)
TARGETS = (
    ("core.run", "_run_chunk", "meep_torch_b200.core.run", "_run_chunk"),
    ("core.run", "run_tm", "meep_torch_b200.core.run", "run_tm"),
    ("core.run", "run_te", "meep_torch_b200.core.run", "run_te"),
    ("core.monitors_3d", "run_3d", "meep_torch_b200.core.monitors_3d", "run_3d"),
    ("core.stepper_3d_lean", "run_3d_lean", "meep_torch_b200.core.stepper_3d_lean",
     "run_3d_lean"),
    ("core.adjoint3d", "run_3d_adjoint", "meep_torch_b200.core.adjoint3d", "run_3d_adjoint"),
)

# methods: (reference module, class, method, this package's module, its function)
METHOD_TARGETS = (
    ("mp.cpp.core", "fields", "solve_cw", "meep_torch_b200.cw", "solve_cw_fields"),
)

_patched: list = []          # (module or class, attribute, original) in patch order


def _first_tensor(obj, depth: int = 0):
    """The first tensor in an argument: the tensor itself, or the first tensor field
    of a state / coefficient NamedTuple (one level of nesting)."""
    if torch.is_tensor(obj):
        return obj
    if depth < 2 and isinstance(obj, tuple):
        for v in obj:
            t = _first_tensor(v, depth + 1)
            if t is not None:
                return t
    return None


def cuda_f32(args, kwargs) -> bool:
    """True when the call's first tensor argument is a float32 CUDA tensor."""
    for v in list(args) + list(kwargs.values()):
        t = _first_tensor(v)
        if t is not None:
            return bool(t.is_cuda) and t.dtype == torch.float32
    return False


def fields_cuda_f32(args, kwargs) -> bool:
    """True when a fields method's object (the first argument) holds a float32 CUDA
    state."""
    st = getattr(args[0], "_state", None) if args else None
    t = _first_tensor(st)
    return t is not None and bool(t.is_cuda) and t.dtype == torch.float32


def _router(original, ours, fallback: bool, route):
    def routed(*args, **kwargs):
        if route(args, kwargs):
            try:
                return ours(*args, **kwargs)
            except NotImplementedError:
                if not fallback:
                    raise
        return original(*args, **kwargs)
    routed.__name__ = getattr(original, "__name__", "routed")
    routed.__doc__ = getattr(original, "__doc__", None)
    routed.__wrapped__ = original
    routed._meep_b200_router = True
    return routed


def install(package: str = "meep_torch", *, fallback: bool = False, ours=None,
            route=cuda_f32) -> int:
    """Patch the imported ``package`` (the reference) so that its hot-path entry
    points run on this package's kernels. Returns the number of attributes patched.
    ``ours`` maps a function name to a replacement (default: this package's own);
    ``route(args, kwargs)`` decides per call (default: float32 CUDA tensors)."""
    if _patched:
        raise RuntimeError("meep_torch_b200.install(): already installed; uninstall() first")
    importlib.import_module(package)
    routers = {}
    for mod_name, name, our_mod, our_name in TARGETS:
        try:
            mod = importlib.import_module(f"{package}.{mod_name}")
        except ImportError:
            continue
        original = getattr(mod, name, None)
        if original is None:
            continue
        target = (ours or {}).get(name)
        if target is None:
            target = getattr(importlib.import_module(our_mod), our_name)
        routers[id(original)] = (original, _router(original, target, fallback, route))
    # every loaded module of the package that holds one of the originals
    for mname, mod in list(sys.modules.items()):
        if mod is None or not (mname == package or mname.startswith(package + ".")):
            continue
        for attr, val in list(vars(mod).items()):
            hit = routers.get(id(val))
            if hit is not None and hit[0] is val:
                setattr(mod, attr, hit[1])
                _patched.append((mod, attr, val))
    # methods of the reference's classes, routed on the object's state
    for mod_name, cls_name, meth, our_mod, our_name in METHOD_TARGETS:
        try:
            mod = importlib.import_module(f"{package}.{mod_name}")
        except ImportError:
            continue
        cls = getattr(mod, cls_name, None)
        original = vars(cls).get(meth) if isinstance(cls, type) else None
        if original is None:
            continue
        target = (ours or {}).get(meth)
        if target is None:
            target = getattr(importlib.import_module(our_mod), our_name)
        setattr(cls, meth, _router(original, target, fallback, fields_cuda_f32))
        _patched.append((cls, meth, original))
    return len(_patched)


def uninstall() -> int:
    """Restore every attribute install() replaced. Returns how many."""
    n = 0
    while _patched:
        mod, attr, original = _patched.pop()
        setattr(mod, attr, original)
        n += 1
    return n


def installed() -> bool:
    return bool(_patched)
