"""Writes tests/golden/long_runs.json with the REFERENCE's own tracer step on
the full-size FP64 configurations, too large to commit as arrays:

  drop512    512x512 cells, 40 layers, 10 tracers, 500 steps
  batch2048  2048x1024 curvilinear, 50 layers, 24 tracers, 3 steps

The reference (model/hd/tracers/tracers.c, compiled unmodified into
oracle/_ref by oracle/build.py, OpenMP tracer loop) steps each window from
its seeded initial state; the file keeps, per run, the SHA-256 of the input
arrays, the status, the range-warning count, the SHA-256 of every tracer's
final values over cells 1..sgsiz-1 (slot 0 is the reference's scratch slot)
and of the surface vectors, and 64 sampled cells per tracer with their
values (to locate a difference when a hash differs).  Equal hashes mean
bit-for-bit equal results.

Run from the repository root in a checkout that has the reference build:
    python tests/golden/make_hashes.py [name ...] [--threads N]
"""
import hashlib
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
sys.path.insert(0, HERE)

import oracle  # noqa: E402
from cases import input_digest  # noqa: E402

OUT = os.path.join(HERE, "long_runs.json")

# name -> (workload, overrides, steps)
LONG_RUNS = {
    "drop512": ("drop512", {}, 500),
    "batch2048": ("batch2048", {}, 3),
}


def build(name):
    from ems_b200 import synth
    wl, kw, nsteps = LONG_RUNS[name]
    return synth.make(wl, **kw), nsteps


def tracer_hashes(tr):
    """SHA-256 of each tracer's values over cells 1..S-1 (float64 bytes)."""
    return [hashlib.sha256(np.ascontiguousarray(tr[n, 1:]).tobytes()).hexdigest()
            for n in range(tr.shape[0])]


def int_hash(a):
    return hashlib.sha256(np.ascontiguousarray(a, np.int32).tobytes()).hexdigest()


def sample_cells(case, n=64, seed=0):
    wet = case.win.wet_cells()
    rng = np.random.default_rng(seed)
    return np.sort(rng.choice(wet, size=min(n, len(wet)), replace=False)).astype(np.int64)


def main():
    argv = sys.argv[1:]
    nthr = os.cpu_count() or 1
    if "--threads" in argv:
        i = argv.index("--threads")
        nthr = int(argv[i + 1])
        del argv[i:i + 2]
    if not oracle.ref_available(omp=True):
        raise SystemExit("reference build oracle/_ref missing (run oracle/build.py)")
    out = {}
    if os.path.exists(OUT):
        with open(OUT) as f:
            out = json.load(f)
    for name in argv or LONG_RUNS:
        case, nsteps = build(name)
        cells = sample_cells(case)
        t0 = time.time()
        rc, tr, sur, nsur, d = oracle.run_ref(case, nsteps, nthreads=nthr)
        out[name] = {
            "workload": LONG_RUNS[name][0], "overrides": LONG_RUNS[name][1],
            "steps": nsteps, "seed": int(case.seed), "wet_cells": int(case.nwet),
            "tracers": int(case.ntr), "sgsiz": int(case.win.sgsiz),
            "input_sha256": input_digest(case), "status": int(rc),
            "nwarn": int(d.nwarn),
            "tracer_sha256": tracer_hashes(tr),
            "sur_t_sha256": int_hash(sur), "nsur_t_sha256": int_hash(nsur),
            "sample_cells": cells.tolist(),
            "sample_values": [[float(v).hex() for v in tr[n, cells]] for n in range(case.ntr)],
            "reference_seconds": round(time.time() - t0, 1), "threads": nthr,
        }
        with open(OUT, "w") as f:
            json.dump(out, f, indent=1)
        print("%-10s status %d  %d steps  %.0f s" % (name, rc, nsteps, time.time() - t0),
              flush=True)


if __name__ == "__main__":
    main()
