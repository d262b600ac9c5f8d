"""bench.py's reference arm on CPU: it runs the reference's own core (oracle/_ref),
prints one JSON line whose config equals the device arm's, times exactly the steps
it reports, and maps none of this repository's device code."""

import json
import subprocess
import sys
import time
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent

SCRIPT = r"""
import json, sys
sys.path.insert(0, {root!r})
import bench
bench.main(["--impl", "reference", "--steps", "2", "--warmup", "1", "--instances", "3"])
maps = open("/proc/self/maps").read()
print(json.dumps({{"maps_has_product": "libses_b200" in maps}}))
"""


def test_reference_arm_line_and_no_device_library():
    from oracle.oracle import Reference
    if not Reference.available():
        pytest.skip("reference core not built")
    t0 = time.perf_counter()
    r = subprocess.run([sys.executable, "-c", SCRIPT.format(root=str(ROOT))], capture_output=True, text=True,
                       timeout=600, cwd=str(ROOT))
    wall = time.perf_counter() - t0
    assert r.returncode == 0, r.stderr
    lines = [json.loads(x) for x in r.stdout.splitlines() if x.startswith("{")]
    line, maps = lines[0], lines[1]
    assert maps["maps_has_product"] is False
    assert line["impl"] == "reference" and line["steps"] == 2 and line["warmup"] == 1
    assert line["ms_per_step"] * line["steps"] / 1e3 <= wall
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["cpu_baseline"]["kind"] == "reference"
    import bench
    args = bench.parse_args(["--instances", "3"])
    specs = bench.c4_all_specs(args, 1)
    assert line["config"] == bench.c4_config(specs, 1, args)
