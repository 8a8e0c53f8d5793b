"""bench.py's reference arm on CPU: the JSON line the driver reads.

`bench.py --impl reference` times the reference's own tracers.c (compiled
unmodified into oracle/_ref) on a bounded sample of the workload and prints
one JSON line with the contract's keys; these tests run it as the driver
does, in a subprocess, on small samples.
"""
import json
import os
import subprocess
import sys

import pytest

import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

pytestmark = pytest.mark.skipif(not oracle.ref_available(omp=True),
                                reason="reference build oracle/_ref not present")


def run_bench(*args):
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference"] +
                       list(args), cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout
    return json.loads(lines[0])


def check_line(d, workload):
    assert d["impl"] == "reference"
    assert d["unit"] == "tracer cell-steps/s" and d["value"] > 0
    assert d["higher_is_better"] is True and d["n_gpus"] == 1
    assert d["config"]["workload"] == workload
    cb = d["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] >= 1 and cb["value"] == d["value"]
    e = d["e2e"]
    assert e["value"] == d["value"] and e["h2d_bytes_per_step"] == 0
    assert e["d2h_bytes_per_step"] == 0


def test_reference_arm_line():
    d = run_bench("--workload", "stiff2048", "--cpu-sample", "64x32", "--steps", "2",
                  "--warmup", "1")
    check_line(d, "stiff2048")
    assert d["steps"] == 2 and "64x32" in d["cpu_baseline"]["sample"]


def test_reference_arm_multi_basin_sample():
    """The multi-basin workload's sample is the eight basins at 1/16 size."""
    d = run_bench("--workload", "batch8", "--steps", "1", "--warmup", "0")
    check_line(d, "batch8")
    assert "1/16" in d["cpu_baseline"]["sample"]
