"""bench.py's reference arm on CPU: it runs the reference's own core and maps
none of this repository's native libraries.

The arm times oracle/_ref/libwgref.so (the reference core compiled from its
sources) on a row sample of the products workload.  Its seeded inputs come
from the generators' file, loaded by path, so the package's native module
(``_wolfgang_core``, ``libwgpauli.so``, ``libwolfgang.so``) is never loaded in
that process.  The test runs the arm in a fresh interpreter and reads the
process's own memory map at the end.
"""

from __future__ import annotations

import json
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]

SCRIPT = r"""
import json, sys
sys.argv = ["bench.py", "--impl", "reference", "--steps", "1", "--warmup", "0", "--ref-rows", "4"]
sys.path.insert(0, ROOT)
import bench
args = bench.build_parser().parse_args(sys.argv[1:])
line = bench.reference_arm(args, 1, 0)
with open("/proc/self/maps") as f:
    maps = sorted({l.split()[-1] for l in f if l.strip().endswith(".so") or ".so." in l})
print(json.dumps({"line": line, "maps": maps, "modules": sorted(m for m in sys.modules if m.startswith("wolfgang"))}))
"""


def test_reference_arm_loads_only_the_reference_core():
    from oracle import Reference

    if not Reference.available():
        pytest.skip("reference core library (oracle/_ref) was not built")
    proc = subprocess.run([sys.executable, "-c", SCRIPT.replace("ROOT", repr(str(ROOT)))], capture_output=True,
                          text=True, timeout=600, cwd=str(ROOT))
    assert proc.returncode == 0, proc.stderr
    out = json.loads(proc.stdout.strip().splitlines()[-1])
    own = [m for m in out["maps"] if str(ROOT / "wolfgang_b200") in m]
    assert own == [], own
    assert out["modules"] == []
    assert any(m.endswith("oracle/_ref/libwgref.so") for m in out["maps"])
    line = out["line"]
    assert line["impl"] == "reference" and line["extrapolated"] is True
    assert line["cpu_baseline"]["nproc"] >= 1 and line["cpu_baseline"]["cpu_model"]
    assert line["value"] > 0
