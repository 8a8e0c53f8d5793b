"""Full-size FP64 runs against the reference, and the multi-basin batch at
full size in FP32-mixed against the plain FP64 path.

* drop512 (512x512, 40 layers, 10 tracers) for 500 steps and batch2048
  (2048x1024 curvilinear, 50 layers, 24 tracers) for 3 steps: the FP64 path's
  final tracers and surface vectors hash (SHA-256) to what the reference's own
  tracers.c gave on the same inputs (tests/golden/long_runs.json, written by
  tests/golden/make_hashes.py).  Equal hashes are bitwise equality, which
  implies the 1e-12 relative bar.
* batch8 (eight independent basins, 4-32 tracers, one window): FP32-mixed and
  FP64 step side by side; per basin and tracer the largest difference is
  within 1e-5 of the basin's largest value (compared on the device).
"""
import json
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

from cases import input_digest  # noqa: E402
from make_hashes import LONG_RUNS, int_hash, tracer_hashes  # noqa: E402
from ems_b200 import gpu, synth  # noqa: E402

pytestmark = [pytest.mark.gpu, pytest.mark.slow, pytest.mark.usefixtures("need_gpu")]

FIXTURE = os.path.join(HERE, "golden", "long_runs.json")
REL_TOL_FP32 = 1e-5


def fixtures():
    if not os.path.exists(FIXTURE):
        return {}
    with open(FIXTURE) as f:
        return json.load(f)


@pytest.mark.parametrize("name", sorted(LONG_RUNS))
def test_fp64_full_size_matches_reference_hashes(name):
    fx = fixtures().get(name)
    if fx is None:
        pytest.skip("no reference hashes for %s" % name)
    wl, kw, nsteps = LONG_RUNS[name]
    case = synth.make(wl, **kw)
    assert input_digest(case) == fx["input_sha256"], "inputs differ from the fixture's"
    assert fx["status"] == 0
    t = gpu.TracerStep(case, precision=gpu.FP64)
    t.start()
    t.run(nsteps)
    d = t.sync()
    tr = t.download()
    sur, nsur = t.surface()
    t.close()
    got = tracer_hashes(tr)
    bad = [n for n in range(case.ntr) if got[n] != fx["tracer_sha256"][n]]
    if bad:
        cells = np.asarray(fx["sample_cells"])
        n = bad[0]
        want = np.array([float.fromhex(v) for v in fx["sample_values"][n]])
        raise AssertionError("%s: tracers %s differ from the reference; tracer %d at the "
                             "sampled cells: max |diff| %.3e" %
                             (name, bad, n, np.abs(tr[n, cells] - want).max()))
    assert int_hash(sur) == fx["sur_t_sha256"]
    assert int_hash(nsur) == fx["nsur_t_sha256"]
    assert d.nwarn == fx["nwarn"]


def test_batch8_fp32mixed_against_fp64_per_basin():
    case = synth.make("batch8")
    nb = len(case.basins)
    steps = 20
    a = gpu.TracerStep(case, precision=gpu.FP32_MIXED)
    b = gpu.TracerStep(case, precision=gpu.FP64)
    for t in (a, b):
        t.start()
        t.run(steps)
        t.sync()
    d = a.compare(b, region=case.basin2d, nregion=nb)
    a.close()
    b.close()
    for k, (bx, by, L, T) in enumerate(case.basins):
        rel = d["max_rel"][k, :T]
        assert np.all(np.isfinite(rel)), (k, rel)
        assert rel.max() <= REL_TOL_FP32, "basin %d (%dx%d, %d tracers): %s" % (k, bx, by, T,
                                                                               rel.max())
        # tracers a basin does not carry are compared nowhere
        assert np.all(d["max_ref"][k, T:] == 0.0)
