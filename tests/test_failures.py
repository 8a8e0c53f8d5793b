"""Failure detection and recovery of the tracer step, injected on the host.

The reference stops the model (hd_quit_and_dump) on a zero pivot in the
implicit solve (model/hd/tracers/tracers.c:4188-4193), on too many sub-steps
(:664-668) and, through check_unstable (model/hd/momentum/vel2d.c:4007,
called at tracers.c:313), on a NaN in a tracer; the library returns
SHOC_TR_EPIVOT, SHOC_TR_ESUBSTEP and SHOC_TR_ENAN instead, and
SHOC_TR_EGEOM for window maps that fail its layout checks (at create, before
any device work).  Every failure here comes from the inputs: no test makes a
kernel fault or wait.  Checkpoint and resume: a run saved and resumed equals
the unbroken run bit for bit.
"""
import ctypes as C
import os

import numpy as np
import pytest

import oracle
from ems_b200 import _abi, gpu, synth

EGEOM, ENAN, EPIVOT, EUNSUPPORTED = 4, 3, 2, 5


def corrupted(case, field, fn):
    """A copy of the window's geometry struct with one int map replaced."""
    g = case.win.geom
    G = _abi.Geom()
    C.pointer(G)[0] = g
    arr = np.array(getattr(case.win, field), np.int32, copy=True)
    fn(arr)
    setattr(G, field, arr.ctypes.data_as(_abi.IP))
    return G, arr


def create_status(case, geom):
    keep = []
    opts = case.make_opts(keep)
    h = C.c_void_p()
    L = gpu.lib()
    rc = L.shoc_tr_gpu_create(C.byref(geom), C.byref(opts), case.ntr, gpu.FP64, 0, C.byref(h))
    if rc == 0:
        L.shoc_tr_gpu_destroy(h)
    return rc


@pytest.mark.parametrize("field,how", [
    ("xp1", "out_of_range"), ("zm1", "sediment_not_self"), ("m2d", "out_of_range"),
    ("yp1", "not_reciprocal")])
def test_bad_geometry_is_refused_at_create(field, how):
    case = synth.make("small", seed=81)
    wet = case.win.wet_cells()
    c = int(wet[len(wet) // 2])

    def fn(a):
        if how == "out_of_range":
            a[c] = case.win.sgsiz + 5
        elif how == "sediment_not_self":
            bot = case.win.bot_t[1]
            sed = case.win.zm1[bot]
            a[sed] = bot  # the sediment cell no longer maps onto itself
        else:
            # a wet neighbour whose backward map does not come back
            yp = case.win.yp1[c]
            assert case.win.is_wet[yp]
            a[c] = case.win.xp1[c] if case.win.xp1[c] != yp else 0
    G, keep = corrupted(case, field, fn)
    assert create_status(case, G) == EGEOM


def test_unsupported_scheme_is_refused_at_create():
    case = synth.make("small", seed=82, trasc=0x080000)  # FFSL, not built
    with pytest.raises(_abi.StatusError) as e:
        gpu.TracerStep(case)
    assert e.value.code == EUNSUPPORTED


def pivot_case():
    """Two 1 m layers, dt = 1 s and Kz = -0.5 m2/s at the interior face: the
    top row's pivot of the implicit solve is exactly zero (the bottom row
    B = 1 - 0.5, ud = 0.5 / 0.5 = 1, the top row 0.5 - 0.5 * 1)."""
    case = synth.make("small", seed=83, layers=np.array([-2.0, -1.0, 0.0]), depth=(3.0, 9.0),
                      dt=1.0)
    case.Kz[:] = -0.5
    return case


def test_reference_also_stops_on_the_zero_pivot():
    if not oracle.ref_available():
        pytest.skip("reference build oracle/_ref not present")
    assert oracle.run_ref(pivot_case(), 1)[0] == EPIVOT
    assert oracle.run_oracle(pivot_case(), 1)[0] == EPIVOT


@pytest.mark.gpu
@pytest.mark.usefixtures("need_gpu")
@pytest.mark.parametrize("prec", [gpu.FP64, gpu.FP32_MIXED])
def test_zero_pivot_is_reported(prec):
    t = gpu.TracerStep(pivot_case(), precision=prec)
    t.start()
    with pytest.raises(_abi.StatusError) as e:
        t.run(1)
        t.sync()
    assert e.value.code == EPIVOT
    t.close()


@pytest.mark.gpu
@pytest.mark.usefixtures("need_gpu")
@pytest.mark.parametrize("prec,kernels", [(gpu.FP64, ""), (gpu.FP32_MIXED, "fused"),
                                          (gpu.FP32_MIXED, "split")])
@pytest.mark.parametrize("which", ["advected", "not_diffused"])
def test_nan_in_a_tracer_is_reported(prec, kernels, which):
    """A NaN in one cell of one tracer reaches every value the step stores
    around it; the step reports SHOC_TR_ENAN, also for a tracer that is
    neither advected nor vertically diffused (its values are only copied)."""
    case = synth.make("small", seed=84)
    if which == "not_diffused":
        case.opts_arrays_orig = case.opts_arrays

        def opts():
            a = case.opts_arrays_orig()
            a["tbdy"] = np.array([0, 1], np.int32)
            a["tdif_v"] = np.array([0, 1], np.int32)
            return a
        case.opts_arrays = opts
    wet = case.win.wet_cells()
    n = 2 if which == "not_diffused" else 0
    case.tr[n, wet[len(wet) // 3]] = np.nan
    old = os.environ.get("SHOC_TR_GPU_KERNELS")
    if kernels:
        os.environ["SHOC_TR_GPU_KERNELS"] = kernels
    try:
        t = gpu.TracerStep(case, precision=prec)
    finally:
        if old is None:
            os.environ.pop("SHOC_TR_GPU_KERNELS", None)
        else:
            os.environ["SHOC_TR_GPU_KERNELS"] = old
    t.start()
    with pytest.raises(_abi.StatusError) as e:
        t.run(1)
        t.sync()
    assert e.value.code == ENAN
    # the next step is clean again only once the NaN is gone: the status word
    # was cleared by the sync that reported it
    t.close()


@pytest.mark.gpu
@pytest.mark.usefixtures("need_gpu")
def test_nan_through_the_dropin_step():
    case = synth.make("small", seed=85)
    tr, sur, nsur = case.copy_state()
    tr[1, case.win.wet_cells()[5]] = np.nan
    t = gpu.TracerStep(case)
    with pytest.raises(_abi.StatusError) as e:
        t.step(tr, sur, nsur)
    assert e.value.code == ENAN
    t.close()


@pytest.mark.gpu
@pytest.mark.usefixtures("need_gpu")
@pytest.mark.parametrize("prec", [gpu.FP64, gpu.FP32_MIXED])
def test_checkpoint_resume_is_bitwise(prec, tmp_path):
    case = synth.make("small", seed=86, eta_offset=(0.4, -0.3))
    a = gpu.TracerStep(case, precision=prec)
    a.start()
    a.run(4)
    a.sync()
    path = str(tmp_path / "state.bin")
    head = a.checkpoint(path, step=4)
    a.run(5)
    a.sync()
    want = a.download()
    want_sur = a.surface()
    want_mass = a.mass()
    a.close()
    b = gpu.TracerStep(case, precision=prec)
    b.start()           # flow fields (and a throw-away state)
    assert b.resume(path)["step"] == head["step"] == 4
    b.run(5)
    b.sync()
    got = b.download()
    np.testing.assert_array_equal(got[:, 1:], want[:, 1:])
    for x, y in zip(b.surface(), want_sur):
        np.testing.assert_array_equal(x, y)
    np.testing.assert_array_equal(b.mass(), want_mass)
    b.close()


@pytest.mark.gpu
@pytest.mark.usefixtures("need_gpu")
def test_checkpoint_of_another_window_is_refused(tmp_path):
    a = gpu.TracerStep(synth.make("small", seed=87))
    a.start()
    path = str(tmp_path / "s.bin")
    a.checkpoint(path)
    a.close()
    b = gpu.TracerStep(synth.make("small", seed=87), precision=gpu.FP32_MIXED)
    b.start()
    with pytest.raises(_abi.StatusError) as e:
        b.resume(path)
    assert e.value.code == 7
    b.close()
