"""bench.py's reference arm prints one JSON line in the chosen workload's metric, with its
cpu_baseline and a zero-copy e2e block. The arm times the reference's own CPU path when
the reference is installed beside the repository (baseline/_ref), else the oracle port;
the samples here are kept tiny."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _line(*args):
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        *args], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr
    lines = [x for x in r.stdout.splitlines() if x.startswith("{")]
    assert len(lines) == 1, r.stdout
    return json.loads(lines[0])


@pytest.mark.parametrize("args,unit", [
    (["--cpu-structs", "8", "--cpu-steps", "3", "--ref-structs", "1", "--ref-steps", "3"],
     "Gcell-updates/s"),
    (["--workload", "cfg4", "--ref-steps", "4"], "gradient-evaluations/s"),
])
def test_reference_arm_line(args, unit):
    d = _line(*args, "--steps", "1", "--warmup", "0")
    assert d["impl"] == "reference" and d["unit"] == unit and d["metric"] == unit
    _common(d, unit)


def test_reference_arm_cfg5_line():
    """cfg5's reference arm: one full oracle run of a cfg5 design on the host, a plain
    design iteration costed as two, in the surrogate metric's unit and name."""
    d = _line("--workload", "cfg5", "--steps", "1", "--warmup", "0")
    assert d["unit"] == "design-iterations/s" and d["metric"].startswith("design-iterations/s")
    _common(d, "design-iterations/s")


def _common(d, unit):
    assert d["value"] > 0 and d["higher_is_better"] is True
    assert d["cpu_baseline"]["kind"] in ("port", "reference")
    assert d["cpu_baseline"]["value"] == d["value"]
    assert d["e2e"] == {"value": d["value"], "unit": unit, "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}
    assert "workload" in d["config"]
