"""The drop-in step on host arrays (shoc_tr_gpu_step), which moves the tracers
in chunks of slots: up on one copy stream, stepped, back on another.

Per tracer the chunked step runs the kernels of a whole step in the same
order, and the general path carries tr_bounds' thin-surface cursor from chunk
to chunk, so with one slot per chunk (the smallest chunks, the most
boundaries) the results must equal the reference's fixtures bit for bit in
FP64, and the device-resident FP32-mixed step bit for bit in FP32-mixed.
"""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

import oracle  # noqa: E402
from cases import CASES, build, input_digest  # noqa: E402
from ems_b200 import gpu, synth  # noqa: E402

pytestmark = [pytest.mark.gpu, pytest.mark.usefixtures("need_gpu")]


def dropin(case, nsteps, precision, tracers_per_chunk):
    tr, sur, nsur = case.copy_state()
    t = gpu.TracerStep(case, precision=precision)
    t.set_tiling(tracers=tracers_per_chunk)
    nsub = []
    for _ in range(nsteps):
        nsub.append(t.step(tr, sur, nsur).nsub)
    t.close()
    return tr, sur, nsur, nsub


def resident(case, nsteps, precision):
    t = gpu.TracerStep(case, precision=precision)
    t.start()
    t.run(nsteps)
    t.sync()
    tr = t.download()
    sur, nsur = t.surface()
    t.close()
    return tr, sur, nsur


@pytest.mark.parametrize("name", [n for n in sorted(CASES) if n != "basin64"])
def test_chunked_dropin_matches_reference_fixture(name):
    case, nsteps = build(name)
    g = np.load(os.path.join(HERE, "golden", name + ".npz"))
    tr, sur, nsur, _ = dropin(case, nsteps, gpu.FP64, 1)
    np.testing.assert_array_equal(sur, g["sur_t"])
    np.testing.assert_array_equal(nsur, g["nsur_t"])
    want = g["tr"] if input_digest(case) == str(g["digest"]) else \
        oracle.run_oracle(case, nsteps)[1]
    cells = np.arange(1, case.win.sgsiz)
    assert np.array_equal(tr[:, cells], want[:, cells]), name


@pytest.mark.parametrize("name", ["small_crossing_substeps", "small_crossing_thin",
                                  "small_hdiff"])
@pytest.mark.parametrize("chunk", [1, 2])
def test_chunked_dropin_fp32_mixed_equals_resident(name, chunk):
    case, nsteps = build(name)
    a = dropin(case, nsteps, gpu.FP32_MIXED, chunk)
    b = resident(case, nsteps, gpu.FP32_MIXED)
    cells = np.arange(1, case.win.sgsiz)
    assert np.array_equal(a[0][:, cells], b[0][:, cells])
    np.testing.assert_array_equal(a[1], b[1])
    np.testing.assert_array_equal(a[2], b[2])


def test_substeps_are_exercised():
    """Several sub-steps per step, each carried chunk by chunk (the
    crossing cases, which tests/test_oracle.py shows move the surface cell of
    most columns, exercise the general path)."""
    case, nsteps = build("small_crossing_substeps")
    assert max(dropin(case, nsteps, gpu.FP64, 1)[3]) > 1


def test_chunked_dropin_batch_of_basins():
    case = synth.make("batch8small")
    tr, _, _, _ = dropin(case, 2, gpu.FP64, 3)
    ref = resident(case, 2, gpu.FP64)[0]
    cells = np.arange(1, case.win.sgsiz)
    assert np.array_equal(tr[:, cells], ref[:, cells])
