"""bench.py's host-side contract, on the CPU: the reference arm's JSON line
(the reference's own openmpMdiscr, compiled from its sources into oracle/_ref,
run on the GPU arm's seeded input) and the per-launch DRAM traffic the GPU
arm reads from profiles/."""
import json
import os
import subprocess
import sys

import pytest

import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


def test_reference_arm_line_on_a_small_input():
    if not oracle.ref_available():
        pytest.skip("oracle/_ref (the reference's OpenmpMdiscr build) is not built")
    res = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                          "--n", str(1 << 20), "--steps", "3", "--warmup", "3"],
                         capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert res.returncode == 0, res.stderr
    line = json.loads(res.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference"
    assert line["metric"] == bench.METRIC and line["unit"] == "Gelem/s"
    assert line["higher_is_better"] is True and line["steps"] == 3 and line["warmup"] >= 3
    assert line["value"] > 0 and line["config"]["n"] == 1 << 20 and line["config"]["m"] == 8
    cb = line["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["same_input"] is True and cb["value"] == line["value"]
    assert cb["cores"] >= 1
    e2e = line["e2e"]
    assert e2e["value"] == line["value"] and e2e["h2d_bytes_per_step"] == 0
    assert e2e["d2h_bytes_per_step"] == 0


def test_traffic_figures_from_profiles():
    tr = bench.traffic_from_profiles()
    n = 1 << 28
    # per launch at the headline size: the count reads the input once, the
    # scatter re-reads it and writes the output (within the L2 reuse and the
    # count's few MB of writes)
    assert 0.95 * n * 4 <= tr["count_kernel_bytes"] <= 1.1 * n * 4
    assert 1.85 * n * 4 <= tr["scatter_kernel_bytes"] <= 2.05 * n * 4


def test_peak_denominator_is_stated():
    peak, src = bench.peaks()
    assert peak > 1000 and src
