"""Install the reference (meep_torch) into ``baseline/_ref`` for the reference arm.

The offline route is ``pip install --no-index --no-build-isolation --find-links
<wheelhouse> --target baseline/_ref <checkout>``. The reference builds with hatchling
(pyproject.toml ``build-backend = "hatchling.build"``), which the offline wheelhouse
does not hold, so that route fails before anything is built. The reference's wheel
target is just its pure-Python package (``[tool.hatch.build.targets.wheel] packages =
["meep_torch"]``), so the fallback places the same files where ``pip --target`` would:
``baseline/_ref/meep_torch``, unmodified, without bytecode. The dependencies the
benchmarked path imports (torch, numpy, scipy) are already in the interpreter.

``baseline/_ref`` is git-ignored: the reference is a run-time input of the reference
arm, never part of this repository's sources.

Usage: ``python baseline/install_reference.py <reference checkout>``
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
TARGET = os.path.join(HERE, "_ref")
WHEELHOUSE = "/opt/wheelhouse"


def install(checkout: str) -> str:
    pkg = os.path.join(checkout, "meep_torch")
    if not os.path.isdir(pkg):
        raise SystemExit(f"{checkout!r} holds no meep_torch package")
    cmd = [sys.executable, "-m", "pip", "install", "--no-index", "--no-build-isolation",
           "--find-links", WHEELHOUSE, "--target", TARGET, checkout]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode == 0:
        return "pip"
    dst = os.path.join(TARGET, "meep_torch")
    if os.path.isdir(dst):
        shutil.rmtree(dst)
    os.makedirs(TARGET, exist_ok=True)
    shutil.copytree(pkg, dst, ignore=shutil.ignore_patterns("__pycache__", "*.pyc"))
    with open(os.path.join(TARGET, "INSTALLED_BY"), "w") as f:
        f.write("copy of the reference's pure-Python wheel contents (pip could not build: "
                + (r.stderr.strip().splitlines() or ["?"])[-1] + ")\n")
    return "copy"


if __name__ == "__main__":
    if len(sys.argv) != 2:
        raise SystemExit(__doc__)
    print(install(sys.argv[1]))
