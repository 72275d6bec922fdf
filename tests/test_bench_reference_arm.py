"""bench.py's reference arm on CPU: it times the oracle port on the host cores and must
not load any part of libworld_b200 (the library under test), so that the ratio of the
two arms compares the library against the reference's algorithm alone."""
from __future__ import annotations

import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

_PROBE = r"""
import json, sys
sys.argv = ["bench.py", "--impl", "reference", "--grains", "4096", "--steps", "2", "--warmup", "1"]
import bench
rc = bench.main()
maps = open("/proc/self/maps").read()
print(json.dumps({"rc": rc, "library_mapped": "libworld_b200" in maps,
                  "oracle_mapped": "libdem_oracle" in maps,
                  "binding_imported": "world_b200._lib" in sys.modules}))
"""


def test_reference_arm_runs_the_oracle_without_the_library():
    res = subprocess.run([sys.executable, "-c", _PROBE], cwd=ROOT, capture_output=True,
                         text=True, timeout=600)
    assert res.returncode == 0, res.stderr[-2000:]
    lines = [json.loads(l) for l in res.stdout.splitlines() if l.startswith("{")]
    line, probe = lines[0], lines[-1]
    assert probe == {"rc": 0, "library_mapped": False, "oracle_mapped": True,
                     "binding_imported": False}
    assert line["impl"] == "reference" and line["value"] > 0
    assert line["warmup"] == 1 and line["steps"] == 2
    assert line["cpu_baseline"]["kind"] == "port"
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["value"] == line["value"]
    assert line["config"]["workload"] == "collapse_1m_sie_mu05"
