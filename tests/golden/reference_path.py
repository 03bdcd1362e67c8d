"""Where tests and fixture recipes find the reference (meep_torch), read-only.

Two places are looked at, in order: the checkout named by the MEEP_TORCH_REF
environment variable, then the reference arm's install beside this repository
(``baseline/_ref``, made by ``baseline/install_reference.py``). No machine path is
built in."""
import os

_REPO = os.path.abspath(os.path.join(os.path.dirname(os.path.abspath(__file__)), "..", ".."))
_INSTALLED = os.path.join(_REPO, "baseline", "_ref")


def find_reference():
    """The directory holding the ``meep_torch`` package, or None."""
    for ref in (os.environ.get("MEEP_TORCH_REF"), _INSTALLED):
        if ref and os.path.isdir(os.path.join(ref, "meep_torch")):
            return ref
    return None


def reference_root() -> str:
    """Like find_reference(), for the fixture recipes: refuses to run without one."""
    ref = find_reference()
    if ref is None:
        raise SystemExit("no reference found: set MEEP_TORCH_REF to a meep_torch checkout "
                         "or run baseline/install_reference.py")
    return ref
