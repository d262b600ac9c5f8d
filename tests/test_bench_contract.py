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


def test_single_roofline_follows_the_step_form():
    """The single-instance roofline credits the plane pass of the two-sweep form
    with both y transforms (8E + E_tab model bytes, 2E + E_tab moved) and the
    four-pass x pass with 4E + E_tab (3E moved); the dominant launch is the
    slowest kind profiled."""
    import bench
    npts = 64 ** 3
    prof_two = {"x_mid": 0.010, "fused": 0.006}
    prof_four = {"x_mid": 0.006, "y_fwd": 0.003, "fused": 0.005, "y_inv": 0.003}
    two = bench.single_roofline(prof_two, npts, "c128", 6537.0, "measured", {}, "c1",
                                "x:64 ...; step: two sweeps (x-y plane pass on 2 CTAs per plane, z pass)")
    four = bench.single_roofline(prof_four, npts, "c128", 6537.0, "measured", {}, "c1",
                                 "x:64 ...; step: four axis passes")
    E = 16
    assert two["kernel"] == "x_mid" and two["step_form"] == "two sweeps"
    assert two["algorithmic_bytes_per_launch"] == (8 * E + E) * npts
    assert abs(two["achieved"] - (8 * E + E) * npts / 0.010e-3 / 1e9) < 0.2
    assert abs(two["moved_gbs"] - 3 * E * npts / 0.010e-3 / 1e9) < 0.2
    assert four["kernel"] == "x_mid" and four["step_form"] == "four axis passes"
    assert four["algorithmic_bytes_per_launch"] == (4 * E + E) * npts
    assert bench.two_sweep("step: two sweeps (x-y plane pass on 1 CTA per plane, z pass)")
    assert not bench.two_sweep("step: four axis passes")
    assert bench.TWO_SWEEP_BYTES["c128"] == 80 and bench.ACTUAL_BYTES["c128"] == 144
