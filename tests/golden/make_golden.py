"""Writes tests/golden/*.npz with the REFERENCE's own tracer step.

Runs model/hd/tracers/tracers.c, compiled unmodified into oracle/_ref by
oracle/build.py, on each case of cases.py and stores the final tracer arrays,
surface vectors and range-warning count.  Run from the repository root in a
checkout that has the reference tree:  python tests/golden/make_golden.py
[name ...]  (default: every case).
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
sys.path.insert(0, HERE)

import oracle  # noqa: E402
from cases import ALL_CASES, build, input_digest  # noqa: E402


def main():
    if not oracle.ref_available():
        raise SystemExit("reference build oracle/_ref missing (run oracle/build.py)")
    for name in sys.argv[1:] or ALL_CASES:
        case, nsteps = build(name)
        rc, tr, sur, nsur, d = oracle.run_ref(case, nsteps)
        path = os.path.join(HERE, name + ".npz")
        np.savez_compressed(path, status=rc, tr=tr, sur_t=sur, nsur_t=nsur,
                            nwarn=d.nwarn, nsteps=nsteps, digest=input_digest(case))
        print("%-26s status %d  wet %7d  steps %3d  %6.1f KB" %
              (name, rc, case.nwet, nsteps, os.path.getsize(path) / 1024))


if __name__ == "__main__":
    main()
