"""The other per-column tridiagonal solves of SHOC, batched on the GPU:

  shoc_tr_gpu_tridiag     the closures' tridiagonal (model/hd/closure/
                          MY2-5.c:499-536; MY2-5, k-e and k-w closures)
  shoc_tr_gpu_vdiff_cols  implicit_vdiff_at_cc (model/hd/tracers/
                          tracers.c:7407-7545) for every column at once

Each is compared bit for bit with the reference's own function, compiled
unmodified into oracle/_ref, on the same seeded systems: diagonally dominant
coefficients of the closures' and the diffusion's form, with sources, fluxes
and a scale, on windows whose columns hold one to all layers.  A zero divisor
is reported as the reference reports it.
"""
import numpy as np
import pytest

import oracle
from ems_b200 import gpu, synth

pytestmark = pytest.mark.skipif(not oracle.ref_available(), reason="oracle/_ref not present")


def systems(case, seed):
    """Seeded coefficients of the diffusion form: C = dz/dt - Cm1 - Cp1 with
    Cm1, Cp1 = -K / dzface <= 0 (diagonally dominant), and values."""
    rng = np.random.default_rng(seed)
    S = case.win.sgsiz
    dz = rng.uniform(0.3, 12.0, S)
    K = 10.0 ** rng.uniform(-6, 0, S)
    Cm1 = -K / rng.uniform(0.5, 10.0, S)
    Cp1 = -np.roll(K, 1) / rng.uniform(0.5, 10.0, S)
    dt = 60.0
    Cd = dz / dt - Cm1 - Cp1
    var = rng.lognormal(0.0, 1.0, S)
    rhs = dz / dt * var
    return dict(dz=dz, Cm1=Cm1, Cp1=Cp1, C=Cd, var=var, rhs=rhs, dt=dt)


def windows():
    return [synth.make("small", seed=91), synth.make("drop512", nx=48, ny=40, seed=92),
            synth.make("small", seed=93, eta_offset=(1.9, -1.7),
                       layers=np.linspace(-30, 2.0, 8))]


def test_reference_tridiag_runs_on_cpu():
    case = windows()[0]
    s = systems(case, 1)
    var = np.zeros(case.win.sgsiz)
    assert oracle.ref_tridiag(case, s["C"], s["Cm1"], s["Cp1"], s["rhs"], var, 0.0) == 0
    wet = case.win.wet_cells()
    assert np.all(var[wet] >= 0.0) and var[wet].max() > 0.0


@pytest.mark.gpu
@pytest.mark.usefixtures("need_gpu")
@pytest.mark.parametrize("minvar", [0.0, 0.7])
def test_tridiag_bitwise(minvar):
    for i, case in enumerate(windows()):
        s = systems(case, 10 + i)
        want = np.full(case.win.sgsiz, -1.0)
        assert oracle.ref_tridiag(case, s["C"], s["Cm1"], s["Cp1"], s["rhs"], want, minvar) == 0
        t = gpu.TracerStep(case)
        t.start()
        got = np.full(case.win.sgsiz, -1.0)
        t.tridiag(s["C"], s["Cm1"], s["Cp1"], s["rhs"], got, minvar)
        t.close()
        np.testing.assert_array_equal(got, want)


@pytest.mark.gpu
@pytest.mark.usefixtures("need_gpu")
@pytest.mark.parametrize("sources", [False, True])
def test_vdiff_cols_bitwise(sources):
    for i, case in enumerate(windows()):
        s = systems(case, 20 + i)
        rng = np.random.default_rng(30 + i)
        S2 = case.win.sgsizS
        fb, ft = rng.normal(0, 1e-3, S2), rng.normal(0, 1e-3, S2)
        scale = rng.uniform(0.5, 1.0, S2)
        Sp = rng.uniform(0, 1e-5, case.win.sgsiz) if sources else None
        Sm = -rng.uniform(0, 1e-6, case.win.sgsiz) if sources else None
        want = s["var"].copy()
        assert oracle.ref_vdiff_cols(case, want, s["dz"], s["C"], s["Cm1"], s["Cp1"], fb, ft,
                                     scale, s["dt"], Sp, Sm) == 0
        t = gpu.TracerStep(case)
        t.start()
        got = s["var"].copy()
        t.vdiff_cols(got, s["dz"], s["C"], s["Cm1"], s["Cp1"], fb, ft, scale, s["dt"], Sp, Sm)
        t.close()
        np.testing.assert_array_equal(got, want)


@pytest.mark.gpu
@pytest.mark.usefixtures("need_gpu")
def test_tridiag_zero_divisor_is_reported():
    """Two unit rows with C = 1, Cm1 = Cp1 = 1 eliminate to a zero pivot."""
    from ems_b200 import _abi
    case = synth.make("small", seed=94, layers=np.array([-2.0, -1.0, 0.0]), depth=(3.0, 9.0))
    S = case.win.sgsiz
    one = np.ones(S)
    want = np.zeros(S)
    assert oracle.ref_tridiag(case, one, one, one, one, want, 0.0) == 2
    t = gpu.TracerStep(case)
    t.start()
    with pytest.raises(_abi.StatusError) as e:
        t.tridiag(one, one, one, one, np.zeros(S), 0.0)
    assert e.value.code == 2
    t.close()
