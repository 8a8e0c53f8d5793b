"""The mass reduction entry point that allocates no device memory.

Some callers cannot allocate device memory while they step: host frameworks
that hand out all device memory from a pool reserved at start-up and forbid
any other allocation during the run.  shoc_tr_gpu_mass_noalloc keeps its
partial sums in a fixed device array instead; it must give what
shoc_tr_gpu_mass gives -- bit for bit, since both sum the same block partials
in the same compensated order -- on repeated calls (the array keeps the
previous call's contents), and refuse tracer counts beyond its fixed
capacity.  This file is collected last on purpose.
"""
import numpy as np
import pytest

from ems_b200 import _abi, gpu, synth

pytestmark = [pytest.mark.gpu, pytest.mark.usefixtures("need_gpu")]


@pytest.mark.parametrize("precision", [gpu.FP64, gpu.FP32_MIXED])
def test_noalloc_mass_matches_allocating_entry_point(precision):
    case = synth.make("small", seed=71)
    t = gpu.TracerStep(case, precision=precision)
    t.start()
    t.run(3)
    t.sync()
    for _ in range(2):  # two calls in a row: the second reuses the fixed array
        want = t.mass()
        got = t.mass_noalloc()
        np.testing.assert_array_equal(got, want)
        t.run(1)
        t.sync()
    t.close()


def test_noalloc_mass_refuses_too_many_tracers():
    case = synth.make("small", seed=72, ntr=65)
    t = gpu.TracerStep(case)
    t.start()
    with pytest.raises(_abi.StatusError) as e:
        t.mass_noalloc()
    assert e.value.code == 9  # SHOC_TR_ESCRATCH
    t.close()
