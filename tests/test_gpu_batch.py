"""Uneven batch of independent basins in one window (one launch per kernel).

batch8small: the eight basins of the multi-basin configuration at 1/16 of
their horizontal size (20-60 layers, 4-32 tracers each), side by side and
separated by land.  Each water column carries only its basin's tracers
(shoc_tr_opts.ntr2d).  The basins do not interact and the tracers do not
interact, so every carried (column, tracer) pair must equal a run of the
whole window with every tracer everywhere (the oracle), bit for bit in FP64,
and the pairs a column does not carry must keep their values.
"""
import numpy as np
import pytest

import oracle
from ems_b200 import gpu, synth

pytestmark = [pytest.mark.gpu, pytest.mark.usefixtures("need_gpu")]


def carried(case):
    """Boolean (ntr, wet cells) mask of the carried pairs and the wet cells."""
    w = case.win.wet_cells()
    nt = case.ntr2d[case.win.m2d[w]]
    return np.arange(case.ntr)[:, None] < nt[None, :], w


def run(case, nsteps, prec):
    t = gpu.TracerStep(case, precision=prec)
    t.start()
    t.run(nsteps)
    t.sync()
    out = t.download()
    t.close()
    return out


@pytest.fixture(scope="module")
def batch():
    case = synth.make("batch8small")
    ref = oracle.run_oracle(case, 3)[1]
    return case, ref


def test_batch_fp64_carried_pairs_bitwise(batch):
    case, ref = batch
    got = run(case, 3, gpu.FP64)
    m, w = carried(case)
    g, r, t0 = got[:, w], ref[:, w], case.tr[:, w]
    assert np.array_equal(g[m], r[m])
    assert np.array_equal(g[~m], t0[~m])  # not carried: unchanged
    assert m.sum() > 0 and (~m).sum() > 0


def test_batch_fp32_mixed_within_tolerance(batch):
    case, ref = batch
    got = run(case, 3, gpu.FP32_MIXED)
    m, w = carried(case)
    g, r = got[:, w], ref[:, w]
    for n in range(case.ntr):
        sel = m[n]
        if not sel.any():
            continue
        e = np.abs(g[n, sel] - r[n, sel]).max() / np.abs(r[n, sel]).max()
        assert e <= 1e-5, (n, e)
    assert np.allclose(g[~m], case.tr[:, w][~m], rtol=1e-7, atol=0)


def test_batch_mass_per_carried_columns(batch):
    """The mass diagnostic sums each tracer over the columns that carry it."""
    case, _ = batch
    t = gpu.TracerStep(case, precision=gpu.FP64)
    t.start()
    m = t.mass()
    t.close()
    # tracer 31 is carried by the largest basin only, tracer 0 by all
    assert m[0] > m[31] > 0


def test_batch_fp32_comp_within_tolerance(batch):
    """FP32_COMP on the batch: every carried pair within 1e-7 of the oracle
    after 3 steps, and the pairs a column does not carry come back as
    uploaded to the compensation's precision (2^-32)."""
    case, ref = batch
    got = run(case, 3, gpu.FP32_COMP)
    m, w = carried(case)
    g, r = got[:, w], ref[:, w]
    for n in range(case.ntr):
        sel = m[n]
        if not sel.any():
            continue
        e = np.abs(g[n, sel] - r[n, sel]).max() / np.abs(r[n, sel]).max()
        assert e <= 1e-7, (n, e)
    assert np.allclose(g[~m], case.tr[:, w][~m], rtol=1e-9, atol=0)
