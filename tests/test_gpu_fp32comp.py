"""FP32_COMP: the FP32-mixed step with a 16-bit compensation stored beside
every FP32 tracer value.

The FP32-mixed step rounds every value to FP32 at the end of each step, so a
value that changes by less than half an FP32 ulp per step does not change at
all, and over N steps the largest error grows towards N ulp / 2.  FP32_COMP
keeps v - (float)v beside it as a bfloat16, and every kernel that reads a
value back adds it, so the stored state is accurate to about 2^-32.

The advection kernel reads every stencil value with its compensation and
runs the ULTIMATE limiter on compensated differences, with the Courant-capped
flux in FP64: a face capped at |cr| moves the whole upwind difference in one
step, so FP32 rounding there is not damped by the Courant number.

Checked here: the error bar of the FP32-mixed tests, an error well below
the FP32-mixed step's own on the same inputs, 1000 stiff steps within 5e-6,
mass conservation, bitwise
agreement of the column kernel's layouts, of the drop-in step on FP64 host
arrays with the resident step, of a checkpoint round trip and of steps after
the autotuner's trial steps, and the configurations the mode refuses.
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
    return np.abs(g - r).max(axis=1) / np.abs(r).max(axis=1)


def run(case, nsteps, precision=gpu.FP32_COMP, **tuning):
    t = gpu.TracerStep(case, precision=precision)
    t.start()
    if tuning:
        t.set_tuning(fused=0, **tuning)
    m0 = t.mass()
    t.run(nsteps)
    t.sync()
    out = t.download()
    sur, nsur = t.surface()
    m1 = t.mass()
    t.close()
    return out, sur, nsur, m0, m1


@pytest.mark.parametrize("kw", [
    {}, dict(trasc=_abi.VANLEER, ultimate=1), dict(dt=2000.0), dict(hdiff=(40.0, [1, 0, 1]))])
def test_small_windows_within_tolerance(kw):
    case = synth.make("small", seed=61, **kw)
    out, sur, nsur, _, _ = run(case, 10)
    ref = oracle.run_oracle(case, 10)
    e = errors(case, out, ref[1])
    assert np.all(e <= TOL), e
    np.testing.assert_array_equal(sur, ref[2])
    np.testing.assert_array_equal(nsur, ref[3])


def test_basin64_error_below_fp32_mixed():
    """100 steps of basin64 against the FP64 oracle: the compensated step
    stays within 2e-8 (3.3e-9 measured), a twentieth of the FP32-mixed
    step's error on the same inputs or less (8.5e-7 measured)."""
    case = synth.make("basin64")
    ref = oracle.run_oracle(case, 100)[1]
    ec = errors(case, run(case, 100)[0], ref)
    em = errors(case, run(case, 100, gpu.FP32_MIXED)[0], ref)
    assert np.all(ec <= 2e-8), ec
    assert ec.max() <= 0.05 * em.max(), (ec, em)


def test_stiff_window_1000_steps():
    """The stiff workload (0.5 m surface layers, Kz up to 1) on a 512x256
    window, 1000 steps against the plain FP64 GPU path (bitwise equal to the
    reference on every parity case): every tracer's largest error stays
    below 5e-6 at every 250th step (at most 1.9e-6 measured) and the mass is
    conserved to 1e-12.  The FP32-mixed step passes 1e-5 here by step 500."""
    from ems_b200 import accuracy
    case = synth.make("stiff2048", nx=512, ny=256)
    rows = accuracy.compare(case, 1000, 250, precision=gpu.FP32_COMP)
    for r in rows:
        assert max(r["max_rel"]) <= 5e-6, (r["step"], max(r["max_rel"]))
        assert max(r["mass_drift_fp32mixed"]) <= 1e-12


@pytest.mark.parametrize("name,steps", [("basin64", 100), ("small", 50)])
def test_conserves_mass(name, steps):
    case = synth.make(name)
    *_, m0, m1 = run(case, steps)
    assert np.all(np.abs(m1 - m0) <= 1e-12 * np.abs(m0)), np.abs(m1 - m0) / np.abs(m0)


@pytest.mark.parametrize("warps", [2, 16])
def test_column_kernel_layouts_agree(warps):
    case = synth.make("small", seed=64)
    a = run(case, 5)[0]
    b = run(case, 5, tracers_per_block=warps, prefetch=1)[0]
    c = run(case, 5, tracers_per_block=warps, prefetch=0)[0]
    np.testing.assert_array_equal(a, b)
    np.testing.assert_array_equal(a, c)


def test_surface_crossing_general_path():
    """Columns whose surface cell changes take the general path, which
    steps their FP32 values and restarts their compensation at 0: the error
    bar still holds (two steps, as for the FP32-mixed step)."""
    case = synth.make("small", seed=62, eta_offset=(1.9, -1.7),
                      layers=np.array([-30.0, -22.0, -14.0, -8.0, -3.0, -1.0, 0.6, 2.5]))
    out, *_ = run(case, 2)
    ref = oracle.run_oracle(case, 2)[1]
    e = errors(case, out, ref)
    assert np.all(e <= TOL), e


@pytest.mark.parametrize("chunk", [1, 2])
def test_dropin_equals_resident(chunk):
    """The drop-in call hands back value + compensation as FP64 and takes it
    again next step; the encoding keeps the trip exact."""
    case = synth.make("small", seed=65)
    tr, sur, nsur = case.copy_state()
    t = gpu.TracerStep(case, precision=gpu.FP32_COMP)
    t.set_tiling(tracers=chunk)
    for _ in range(4):
        t.step(tr, sur, nsur)
    t.close()
    want, ws, wn, _, _ = run(case, 4)
    cells = np.arange(1, case.win.sgsiz)
    np.testing.assert_array_equal(tr[:, cells], want[:, cells])
    np.testing.assert_array_equal(sur, ws)
    np.testing.assert_array_equal(nsur, wn)


def test_checkpoint_round_trip():
    case = synth.make("small", seed=66)
    t = gpu.TracerStep(case, precision=gpu.FP32_COMP)
    t.start()
    t.run(3)
    t.sync()
    blob = t.save_state()
    t.run(3)
    t.sync()
    a = t.download()
    t.load_state(blob)
    t.run(3)
    t.sync()
    b = t.download()
    t.close()
    np.testing.assert_array_equal(a, b)


def test_autotune_keeps_state():
    case = synth.make("small", seed=67)
    want = run(case, 4)[0]
    t = gpu.TracerStep(case, precision=gpu.FP32_COMP)
    t.start()
    t.autotune_ex(1, use_cache=False)
    assert t.get_tuning()["fused"] == 0
    t.run(4)
    t.sync()
    got = t.download()
    t.close()
    np.testing.assert_array_equal(got, want)


def test_refused_configurations():
    case = synth.make("small", seed=68)
    t = gpu.TracerStep(case, precision=gpu.FP32_COMP)
    t.start()
    with pytest.raises(RuntimeError):
        t.set_tuning(fused=1, tile_x=8, phase_b_warps=1)
    t.close()
