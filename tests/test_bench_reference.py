"""bench.py's reference arm on CPU: the JSON line the driver reads.

`bench.py --impl reference` times the reference's own tracers.c (compiled
unmodified into oracle/_ref) on the workload window and prints one JSON line
with the contract's keys; these tests run it as the driver does, in a
subprocess, on small windows of the workloads (--size, and the multi-basin
batch at 1/16 size).  The process builds its window with the oracle's build
of the window builder and loads no library of the package.
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
    d = run_bench("--workload", "stiff2048", "--size", "96x64", "--steps", "2", "--warmup", "1")
    check_line(d, "stiff2048@96x64")
    assert d["steps"] == 2 and "full stiff2048 window (96x64x50" in d["cpu_baseline"]["sample"]
    assert d["config"]["wet_cells"] > 0 and d["config"]["tracers"] == 24


def test_reference_arm_multi_basin():
    d = run_bench("--workload", "batch8small", "--steps", "1", "--warmup", "0")
    check_line(d, "batch8small")
    assert d["config"]["cell_tracers"] < d["config"]["wet_cells"] * d["config"]["tracers"]


def test_reference_arm_loads_no_package_library():
    """The reference arm's process maps only oracle/ libraries of this
    repository (the window builder included)."""
    code = ("import runpy, sys; sys.argv = ['bench.py', '--impl', 'reference', '--workload', "
            "'small', '--steps', '1', '--warmup', '0']; runpy.run_path('bench.py', "
            "run_name='__main__'); print(open('/proc/self/maps').read())")
    r = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    libs = {l.split()[-1] for l in r.stdout.splitlines() if l.endswith(".so") and ROOT in l}
    assert libs and all(os.sep + "oracle" + os.sep in p for p in libs), libs


def test_reference_arm_bounds_full_window_steps():
    """On the full window the arm times at most REF_MAX_STEPS of the steps
    asked for, and says so in its line."""
    d = run_bench("--workload", "stiff2048", "--size", "64x48", "--steps", "7", "--warmup", "2")
    check_line(d, "stiff2048@64x48")
    assert d["steps"] == 3 and d["steps_requested"] == 7 and d["warmup"] == 1
    assert "3 timed steps in one call (of 7 requested)" in d["cpu_baseline"]["sample"]
