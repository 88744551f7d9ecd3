"""The reference arm of bench.py times the reference's CPU path on inputs it
builds itself: it must not load the library under test (CPU only)."""
import json
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent

PROBE = r"""
import json, sys
sys.path.insert(0, %r)
import numpy as np
import bench
kind, threads, run, words = bench.cpu_reference_rate()
out_pairs = run(0, 2)
maps = [l.split()[-1] for l in open('/proc/self/maps') if l.rstrip().endswith('.so')]
print(json.dumps({"kind": kind, "pairs": int(out_pairs), "shape": list(words.shape),
                  "libs": sorted(set(m for m in maps if m.startswith(%r)))}))
"""


def test_reference_arm_maps_no_library_under_test():
    res = subprocess.run([sys.executable, "-c", PROBE % (str(ROOT), str(ROOT))],
                         capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert res.returncode == 0, res.stderr
    info = json.loads(res.stdout.strip().splitlines()[-1])
    assert info["shape"] == [4096, 8, 156 * 14]
    assert info["pairs"] == 4095 + 4094
    assert info["libs"], "the oracle library should be mapped"
    for lib in info["libs"]:
        assert lib.startswith(str(ROOT / "oracle")), lib


def test_both_arms_report_the_same_config():
    sys.path.insert(0, str(ROOT))
    import bench
    a, b = bench.workload_config(), bench.workload_config()
    assert a == b and "threads" not in a and "tile_config" not in a
    json.dumps(a)
