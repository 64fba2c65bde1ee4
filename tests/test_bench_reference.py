"""The bench's reference arm (`bench.py --impl reference`) runs on host
cores only: its JSON line carries the contract's keys."""
import json
import os
import subprocess
import sys

import pytest

import bench

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.timeout(600)
def test_reference_arm_json_line():
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl",
                        "reference", "--steps", "3", "--warmup", "3"],
                       capture_output=True, text=True, timeout=540, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference"
    assert line["metric"] == bench.METRIC
    assert line["unit"] == "particle-steps/s" and line["higher_is_better"] is True
    assert line["value"] > 0 and line["steps"] == 3 and line["warmup"] == 3
    cb = line["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == line["value"]
    assert line["e2e"] == {"value": line["value"], "unit": "particle-steps/s",
                           "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert line["dtype"] == "f64" and line["data"] == "synthetic"


def test_fp64_pipe_roofline_arithmetic():
    r = bench.fp64_pipe_roofline(1.0e10)
    assert r["f_alg"] == bench.F_ALG
    assert r["achieved"] == pytest.approx(1.0e10 * bench.F_ALG / 1e12)
    assert r["frac"] == pytest.approx(r["achieved"] / r["peak"])
