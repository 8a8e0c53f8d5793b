"""FP32-mixed path against the FP64 oracle.

FP32 tracers, face values and Thomas sweeps; FP64 flux divergence, surface
column-mass sums, implicit-solve residual and one refinement step.  Error
measure per tracer: max |gpu - oracle| / max |oracle| over the wet cells
(scale-aware; tracers span 1e-3..1e2), bar 1e-5.
"""
import numpy as np
import pytest

import oracle
from ems_b200 import _abi, gpu, synth

pytestmark = [pytest.mark.gpu, pytest.mark.usefixtures("need_gpu")]

TOL = 1e-5


def errors(case, got, ref):
    c = case.win.wet_cells()
    g, r = got[:, c], ref[:, c]
    scale = np.abs(r).max(axis=1)
    emax = np.abs(g - r).max(axis=1) / scale
    erms = np.sqrt(((g - r) ** 2).mean(axis=1)) / np.sqrt((r ** 2).mean(axis=1))
    return emax, erms


def run(case, nsteps):
    t = gpu.TracerStep(case, precision=gpu.FP32_MIXED)
    t.start()
    t.run(nsteps)
    d = t.sync()
    out = t.download()
    sur, nsur = t.surface()
    t.close()
    return out, sur, nsur, d


@pytest.mark.parametrize("kw", [
    {}, dict(trasc=_abi.VANLEER, ultimate=0), dict(trasc=_abi.VANLEER, ultimate=1),
    dict(ultimate=0), dict(dt=2000.0), dict(hdiff=(40.0, [1, 1, 1])),
    dict(hdiff=(40.0, [1, 0, 1])), dict(trasc=_abi.VANLEER, ultimate=0, hdiff=(40.0, [0, 1, 1]))])
def test_small_windows_within_tolerance(kw):
    case = synth.make("small", seed=61, **kw)
    out, sur, nsur, d = run(case, 10)
    ref = oracle.run_oracle(case, 10)
    emax, erms = errors(case, out, ref[1])
    assert np.all(emax <= TOL), (emax, erms)
    np.testing.assert_array_equal(sur, ref[2])
    np.testing.assert_array_equal(nsur, ref[3])


@pytest.mark.parametrize("kw", [{}, dict(dt=1500.0), dict(hmin=1.2)])
def test_surface_crossing_general_path(kw):
    """Layer faces at -1.0 and 0.6 m between eta and oldeta: the surface
    cell of most columns changes during the step, and those columns take the
    general path (with hmin=1.2 also tr_bounds' thin-surface cursor).

    eta and oldeta are held apart with a flow whose depth sum has no
    divergence, so every step squeezes the old water of some columns into a
    thin new surface cell: their values grow about 30-fold per step (1e12 in
    6 steps), and surf_conc's balance magnifies the FP32 rounding of their
    neighbours with them (2e-5 relative after 6 steps, against 4e-8 for the
    same inputs rounded to FP32 between FP64 steps).  Two steps keep the case
    inside the range the bound is meant for; the FP64 path is compared bit
    for bit on these cases over 3-6 steps by the golden fixtures."""
    case = synth.make("small", seed=62, eta_offset=(1.9, -1.7),
                      layers=np.array([-30.0, -22.0, -14.0, -8.0, -3.0, -1.0, 0.6, 2.5]), **kw)
    out, sur, nsur, d = run(case, 2)
    ref = oracle.run_oracle(case, 2)
    emax, _ = errors(case, out, ref[1])
    assert np.all(emax <= TOL), emax


def test_basin64_fp32_mixed():
    case = synth.make("basin64")
    out, *_ = run(case, 100)
    ref = oracle.run_oracle(case, 100)[1]
    emax, erms = errors(case, out, ref)
    assert np.all(emax <= TOL), (emax, erms)


@pytest.mark.slow
def test_drop512_fp32_mixed():
    case = synth.make("drop512")
    out, *_ = run(case, 3)
    ref = oracle.run_oracle(case, 3)[1]
    emax, erms = errors(case, out, ref)
    assert np.all(emax <= TOL), (emax, erms)


def test_accuracy_report_small():
    """ems_b200.accuracy: FP32-mixed against the FP64 GPU path over 20 steps;
    the FP64 path conserves the tracer mass to round-off."""
    from ems_b200 import accuracy
    case = synth.make("small")
    rows = accuracy.compare(case, 20, 10)
    assert [r["step"] for r in rows] == [10, 20]
    assert max(rows[-1]["max_rel"]) <= TOL
    assert max(rows[-1]["rms_rel"]) <= TOL
    assert max(rows[-1]["mass_drift_fp64"]) <= 1e-12


def run_kernels(case, nsteps, kernels):
    """FP32-mixed run with the fused sub-step kernel or the two-kernel split
    (SHOC_TR_GPU_KERNELS, read when a handle is created)."""
    import os
    old = os.environ.get("SHOC_TR_GPU_KERNELS")
    os.environ["SHOC_TR_GPU_KERNELS"] = kernels
    try:
        t = gpu.TracerStep(case, precision=gpu.FP32_MIXED)
    finally:
        if old is None:
            del os.environ["SHOC_TR_GPU_KERNELS"]
        else:
            os.environ["SHOC_TR_GPU_KERNELS"] = old
    t.start()
    m0 = t.mass()
    t.run(nsteps)
    t.sync()
    out = t.download()
    m1 = t.mass()
    t.close()
    return out, m0, m1


@pytest.mark.parametrize("kw", [{}, dict(dt=2000.0), dict(trasc=_abi.VANLEER, ultimate=1),
                                dict(hdiff=(40.0, [1, 0, 1]))])
def test_fused_and_split_kernels_agree(kw):
    """The fused sub-step kernel and the advection + column kernel pair give
    the same tracers to FP32 rounding (the fused one keeps the advected
    values in FP64 until tr_bounds and carries the rounded-off mass)."""
    case = synth.make("small", seed=63, **kw)
    a = run_kernels(case, 10, "fused")[0]
    b = run_kernels(case, 10, "split")[0]
    ref = oracle.run_oracle(case, 10)[1]
    ea, _ = errors(case, a, ref)
    eb, _ = errors(case, b, ref)
    assert np.all(ea <= TOL) and np.all(eb <= TOL), (ea, eb)
    c = case.win.wet_cells()
    assert np.all(np.abs(a[:, c] - b[:, c]).max(axis=1) <= TOL * np.abs(ref[:, c]).max(axis=1))


@pytest.mark.parametrize("kernels", ["split", "fused"])
@pytest.mark.parametrize("name,steps", [("basin64", 100), ("small", 50)])
def test_fp32mixed_conserves_mass(name, steps, kernels):
    """FP32 storage loses mass at every rounding; the per-column FP64 carry
    gives it back (the two-kernel sub-step from the advection kernel's
    rounding residuals, the fused one from its FP64 accumulators), so the
    stored values plus the carry conserve each tracer's mass to 1e-12
    relative, as the FP64 path does."""
    case = synth.make(name)
    _, m0, m1 = run_kernels(case, steps, kernels)
    assert np.all(np.abs(m1 - m0) <= 1e-12 * np.abs(m0)), np.abs(m1 - m0) / np.abs(m0)


@pytest.mark.parametrize("warps", [2, 5, 16])
def test_column_kernel_layouts_agree(warps):
    """k_vd32 with any number of warps per block, with and without staging
    the next tracer's column during the solve, gives the same tracers bit
    for bit (each (column, tracer) is solved by one thread either way)."""
    case = synth.make("small", seed=64)
    out = []
    for kw in ({}, dict(tracers_per_block=warps, prefetch=1),
               dict(tracers_per_block=warps, prefetch=0)):
        t = gpu.TracerStep(case, precision=gpu.FP32_MIXED)
        t.start()
        if kw:
            t.set_tuning(fused=0, **kw)
        t.run(5)
        t.sync()
        out.append(t.download())
        t.close()
    np.testing.assert_array_equal(out[0], out[1])
    np.testing.assert_array_equal(out[0], out[2])
