"""The SHOC-side binding (include/shoc_tr_shim.h), compiled against the
reference's own model/hd/include headers (oracle/build.py shim_lib, as a SHOC
build with HAVE_B200_TRACERS would compile it).

On the CPU: the window description the shim fills from SHOC's window structs
is, field by field, the description those structs were built from.  On the
GPU: steps through b200_tracer_step, the call tracer_step_3d makes in such a
build, equal the library's own resident steps bit for bit.
"""
import ctypes as C
import os

import numpy as np
import pytest

from ems_b200 import _abi, gpu, synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SHIM = os.path.join(ROOT, "oracle", "_ref", "libshoc_shim.so")

pytestmark = pytest.mark.skipif(not os.path.exists(SHIM), reason="oracle/_ref shim not built")


def shim():
    gpu.lib()  # the product library the shim binds
    L = C.CDLL(SHIM)
    for f in (L.shim_fields, L.shim_step):
        f.restype = C.c_int
    L.shim_fields.argtypes = [C.POINTER(_abi.Geom), C.POINTER(_abi.State), C.POINTER(_abi.Opts)]
    L.shim_step.argtypes = [C.POINTER(_abi.Geom), C.POINTER(_abi.State), C.POINTER(_abi.Opts),
                            C.c_int]
    return L


def call(fn, case, *extra):
    keep = []
    tr, sur, nsur = case.copy_state()
    st = case.make_state(tr, sur, nsur, keep)
    op = case.make_opts(keep)
    rc = fn(C.byref(case.win.geom), C.byref(st), C.byref(op), *extra)
    return rc, tr, sur, nsur


@pytest.mark.parametrize("kw", [{}, dict(hdiff=(40.0, [1, 0, 1]))])
def test_shim_maps_every_field(kw):
    case = synth.make("small", seed=95, **kw)
    assert call(shim().shim_fields, case)[0] == 0


@pytest.mark.gpu
@pytest.mark.usefixtures("need_gpu")
def test_steps_through_the_shim_equal_resident_steps():
    case = synth.make("small", seed=96, eta_offset=(0.4, -0.3))
    rc, tr, sur, nsur = call(shim().shim_step, case, 5)
    assert rc == 0
    t = gpu.TracerStep(case)
    t.start()
    t.run(5)
    t.sync()
    want = t.download()
    wsur, wnsur = t.surface()
    t.close()
    np.testing.assert_array_equal(tr[:, 1:], want[:, 1:])
    np.testing.assert_array_equal(sur, wsur)
    np.testing.assert_array_equal(nsur, wnsur)
