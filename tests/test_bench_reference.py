"""The benchmark's reference arm on the host: one converged oracle solve of the einzel lens.

``bench.py --impl reference`` times whole converged solves of the benchmark's lens by the
oracle (SciPy's LU field solve, the C trace and deposit on every host core), needs no GPU,
and prints one JSON line with the metric, unit and configuration of the device arm.
"""

from __future__ import annotations

import json
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def test_reference_arm_prints_one_converged_solve():
    out = subprocess.run(
        [sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--steps", "1",
         "--warmup", "0"],
        cwd=ROOT, capture_output=True, text=True, timeout=600, check=True,
    )  # fmt: skip
    lines = [line for line in out.stdout.splitlines() if line.startswith("{")]
    assert len(lines) == 1
    line = json.loads(lines[-1])
    assert line["impl"] == "reference"
    assert line["unit"] == "solves/s" and line["higher_is_better"] is True
    assert line["value"] > 0.0
    assert line["e2e"] == {"value": line["value"], "unit": "solves/s", "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}  # fmt: skip
    base = line["cpu_baseline"]
    assert base["kind"] == "port" and base["cores"] >= 1
    assert "7 iterations" in base["sample"]  # the lens converges as on the device
    assert line["config"]["mesh"] == [801, 201] and line["config"]["trajectories"] == 20000
    moments = line["moments"]
    assert sorted(moments) == ["70mm", "79mm"]
    assert moments["79mm"]["current"] > 0.0 and moments["79mm"]["rms_angle"] > 0.0


def test_reference_arm_loads_no_device_library():
    """The reference arm builds its problem on the host alone: it never loads libbt200."""
    code = (
        "import sys, runpy; sys.argv = ['bench.py', '--impl', 'reference', '--steps', '1', "
        "'--warmup', '0']; runpy.run_path('bench.py', run_name='__main__'); "
        "maps = open('/proc/self/maps').read(); "
        "assert 'libbt200' not in maps, 'libbt200 loaded'; print('no-libbt200')"
    )
    out = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True,
                         text=True, timeout=600, check=True)  # fmt: skip
    assert "no-libbt200" in out.stdout
