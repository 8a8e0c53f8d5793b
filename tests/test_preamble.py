"""The transport-mode flow preamble (transport.c:436-462): dzu1 / dzu2,
u1flux3d / u2flux3d and w from the velocities and the surface.

CPU: the restatement (oracle/flow_preamble.py) against the reference's own
set_dz_at_u1 / _u2, set_flux_3d, set_dz and vel_w_update (model/hd/momentum/
vel3d.c, compiled unmodified into oracle/_ref/libshoc_ref_vel.so), bit for bit.
GPU: the device preamble (shoc_tr_gpu_set_preamble) against both, and steps
with it against steps given the reference's fields.
"""
import numpy as np
import pytest

import oracle
from ems_b200 import gpu, synth

LAYERS = np.array([-30.0, -22.0, -14.0, -8.0, -3.0, -1.0, 0.6, 2.5])
CASES = {
    "small": dict(seed=71),
    "small_moving": dict(seed=72, eta_offset=(1.9, -1.7), layers=LAYERS),
    "small_vanleer_hdiff": dict(seed=73, trasc=0x80, ultimate=0, hdiff=(40.0, [1, 1, 1])),
}
FIELDS = ("dzu1", "dzu2", "u1flux3d", "u2flux3d", "w")


def _case(name):
    kw = dict(CASES[name])
    return synth.make("small", **kw)


def _detadt(case):
    return (case.eta - case.oldeta) / case.dt


def _need_ref_vel():
    if oracle._load("ref_vel") is None:
        pytest.skip("oracle/_ref/libshoc_ref_vel.so not built (no reference tree)")


@pytest.mark.parametrize("name", sorted(CASES))
def test_restatement_matches_reference(name):
    _need_ref_vel()
    case = _case(name)
    d = _detadt(case)
    ref = oracle.ref_preamble(case, d)
    got = oracle.preamble(case, d)
    for k in FIELDS:
        np.testing.assert_array_equal(got[k], ref[k], err_msg=k)
    # the preamble did something: fluxes and a vertical velocity
    assert np.abs(ref["u1flux3d"]).max() > 0 and np.abs(ref["w"]).max() > 0


def test_restatement_basin64():
    _need_ref_vel()
    case = synth.make("basin64")
    d = _detadt(case)
    ref = oracle.ref_preamble(case, d)
    got = oracle.preamble(case, d)
    for k in FIELDS:
        np.testing.assert_array_equal(got[k], ref[k], err_msg=k)


@pytest.mark.gpu
@pytest.mark.usefixtures("need_gpu")
@pytest.mark.parametrize("precision", [gpu.FP64, gpu.FP32_MIXED])
@pytest.mark.parametrize("name", sorted(CASES))
def test_device_preamble_bitwise(name, precision):
    """One step with the preamble on: the device's fields equal the
    reference's for the state the step started from."""
    case = _case(name)
    d = _detadt(case)
    sur0, nsur0 = case.sur_t.copy(), case.nsur_t.copy()
    ref = oracle.ref_preamble(case, d, sur0, nsur0)
    t = gpu.TracerStep(case, precision=precision)
    t.start()
    t.set_preamble(True, d)
    t.run(1)
    t.sync()
    got = t.get_flow()
    t.close()
    for k in FIELDS:
        np.testing.assert_array_equal(got[k], ref[k], err_msg=k)


@pytest.mark.gpu
@pytest.mark.usefixtures("need_gpu")
@pytest.mark.parametrize("name", sorted(CASES))
def test_steps_with_device_preamble_equal_given_fields(name):
    """FP64, 3 steps: the preamble on the device gives the tracers and
    surfaces of steps handed the reference preamble's fields each step."""
    case = _case(name)
    d = _detadt(case)
    a = gpu.TracerStep(case, precision=gpu.FP64)
    a.start()
    a.set_preamble(True, d)
    a.run(3)
    a.sync()
    tra = a.download()
    sa = a.surface()
    a.close()

    b = gpu.TracerStep(case, precision=gpu.FP64)
    b.start()
    sur, nsur = case.sur_t.copy(), case.nsur_t.copy()
    for _ in range(3):
        f = oracle.ref_preamble(case, d, sur, nsur)
        case.w, case.u1flux3d, case.u2flux3d = f["w"], f["u1flux3d"], f["u2flux3d"]
        if case.dzu1 is not None:
            case.dzu1, case.dzu2 = f["dzu1"], f["dzu2"]
        b.set_flow(sur, nsur)
        b.run(1)
        b.sync()
        sur, nsur = b.surface()
    trb = b.download()
    b.close()
    c = case.win.wet_cells()
    np.testing.assert_array_equal(tra[:, c], trb[:, c])
    np.testing.assert_array_equal(sa[0], sur)
    np.testing.assert_array_equal(sa[1], nsur)


@pytest.mark.gpu
@pytest.mark.usefixtures("need_gpu")
@pytest.mark.parametrize("precision", [gpu.FP64, gpu.FP32_MIXED, gpu.FP32_COMP])
def test_dropin_steps_with_preamble_equal_resident(precision):
    """The drop-in call on host arrays runs the preamble too: 3 drop-in steps
    with it on give the resident run's tracers and surfaces bit for bit, and
    the fields the host state carries for w and the fluxes are not read."""
    case = _case("small_moving")
    d = _detadt(case)
    a = gpu.TracerStep(case, precision=precision)
    a.start()
    a.set_preamble(True, d)
    a.run(3)
    a.sync()
    tra = a.download()
    sa = a.surface()
    a.close()

    b = gpu.TracerStep(case, precision=precision)
    b.set_preamble(True, d)
    tr, sur, nsur = case.copy_state()
    # garbage in the fields the preamble computes: they must not be read
    case.w = np.full_like(case.w, np.nan)
    case.u1flux3d = np.full_like(case.u1flux3d, np.nan)
    case.u2flux3d = np.full_like(case.u2flux3d, np.nan)
    for _ in range(3):
        b.step(tr, sur, nsur)
    b.close()
    c = case.win.wet_cells()
    np.testing.assert_array_equal(tra[:, c], tr[:, c])
    np.testing.assert_array_equal(sa[0], sur)
    np.testing.assert_array_equal(sa[1], nsur)
