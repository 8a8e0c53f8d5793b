"""CUDA path (FP64 plain) against the oracle and the reference's fixtures.

Bar: bitwise equality with the reference's FP64 results (both follow
tracers.c operation by operation, no FMA contraction, IEEE division), which
implies the <= 1e-12 relative tolerance of the drop-in spec.  Slot 0 of every
tracer array is the reference's unused scratch slot (tracers.c:776 and
:4128-4131, :4209-4212 write into it) and is not compared.
"""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

import oracle  # noqa: E402
from cases import CASES, SCHEME_CASES, build, input_digest  # noqa: E402
from ems_b200 import _abi, gpu, synth  # noqa: E402

pytestmark = [pytest.mark.gpu, pytest.mark.usefixtures("need_gpu")]

REL_TOL = 1e-12   # the drop-in tolerance; the comparisons below are bitwise


def assert_same(got, want, case, what):
    cells = np.arange(1, case.win.sgsiz)
    if not np.array_equal(got[:, cells], want[:, cells]):
        err = oracle.max_rel_err(got, want, cells)
        raise AssertionError("%s: not bitwise equal; max rel err per tracer %s" % (what, err))


def run_resident(case, nsteps, precision=gpu.FP64):
    t = gpu.TracerStep(case, precision=precision)
    t.start()
    t.run(nsteps)
    d = t.sync()
    tr = t.download()
    sur, nsur = t.surface()
    t.close()
    return tr, sur, nsur, d


@pytest.mark.parametrize("name", sorted(CASES))
def test_resident_run_matches_reference_fixture(name):
    case, nsteps = build(name)
    g = np.load(os.path.join(HERE, "golden", name + ".npz"))
    tr, sur, nsur, d = run_resident(case, nsteps)
    np.testing.assert_array_equal(sur, g["sur_t"])
    np.testing.assert_array_equal(nsur, g["nsur_t"])
    if input_digest(case) == str(g["digest"]):
        assert_same(tr, g["tr"], case, name)
    else:  # inputs regenerated with different rounding on this host
        ref = oracle.run_oracle(case, nsteps)[1]
        assert_same(tr, ref, case, name + " vs oracle")


@pytest.mark.parametrize("name", ["small_quickest_ultimate", "small_moving_surface",
                                  "small_clip", "small_thin_surface", "small_crossing_thin"])
def test_warning_count_matches(name):
    case, nsteps = build(name)
    g = np.load(os.path.join(HERE, "golden", name + ".npz"))
    t = gpu.TracerStep(case)
    t.start()
    nwarn = 0
    for _ in range(nsteps):
        t.run(1)
        nwarn += t.sync().nwarn
    t.close()
    assert nwarn == int(g["nwarn"])


def test_dropin_step_on_host_arrays():
    case = synth.make("small", seed=31)
    tr, sur, nsur = case.copy_state()
    t = gpu.TracerStep(case)
    for _ in range(5):
        d = t.step(tr, sur, nsur)
        assert d.nsub == 1
    t.close()
    rc, ref, rsur, rnsur, _ = oracle.run_oracle(case, 5)
    assert rc == 0
    assert_same(tr, ref, case, "drop-in step")
    np.testing.assert_array_equal(sur, rsur)
    np.testing.assert_array_equal(nsur, rnsur)


@pytest.mark.parametrize("seed", [41, 43])
@pytest.mark.parametrize("scheme", [(_abi.QUICKEST, 1), (_abi.QUICKEST, 0), (_abi.VANLEER, 0),
                                    (_abi.VANLEER, 1)])
def test_random_windows_bitwise(seed, scheme):
    case = synth.make("small", seed=seed, trasc=scheme[0], ultimate=scheme[1],
                      layers=np.linspace(-30, 2.0, 8), eta_offset=(0.6, -0.4))
    tr = run_resident(case, 6)[0]
    assert_same(tr, oracle.run_oracle(case, 6)[1], case, "seed %d" % seed)


def test_basin64_against_oracle_and_mass():
    case = synth.make("basin64")
    t = gpu.TracerStep(case)
    t.start()
    m0 = t.mass()
    t.run(100)
    t.sync()
    m1 = t.mass()
    tr = t.download()
    t.close()
    assert_same(tr, oracle.run_oracle(case, 100)[1], case, "basin64")
    assert np.all(np.abs(m1 - m0) <= 1e-12 * np.abs(m0))


@pytest.mark.slow
def test_drop512_against_oracle():
    case = synth.make("drop512")
    tr = run_resident(case, 3)[0]
    assert_same(tr, oracle.run_oracle(case, 3)[1], case, "drop512")


def test_determinism_and_tiling():
    case = synth.make("small", seed=47)
    a = run_resident(case, 4)[0]
    t = gpu.TracerStep(case)
    t.set_tiling(tracers=1)
    t.start()
    t.run(4)
    t.sync()
    b = t.download()
    t.close()
    np.testing.assert_array_equal(a[:, 1:], b[:, 1:])


def test_substep_limit_raises():
    case = synth.make("small", dt=40000.0)
    t = gpu.TracerStep(case)
    t.start()
    with pytest.raises(_abi.StatusError) as e:
        t.run(1)
    assert e.value.code == 1
    t.close()


@pytest.mark.parametrize("prec", [gpu.FP64, gpu.FP32_MIXED])
def test_autotune_keeps_state(prec, tmp_path, monkeypatch):
    """The autotuner's trial steps start from a device copy of the state and
    the state is put back: 3 steps after autotuning equal 3 plain steps with
    the chosen configuration, bit for bit.  The choice is cached per GPU and
    configuration: a second handle gets it without trial steps."""
    monkeypatch.setenv("SHOC_TR_TUNE_CACHE", str(tmp_path / "tuning.txt"))
    case = synth.make("small", seed=48)
    t = gpu.TracerStep(case, precision=prec)
    t.start()
    t.run(2)
    t.sync()
    best, cached = t.autotune_ex(1)
    assert not cached and best["tracers_per_block"] in (2, 3, 4, 5, 6, 8, 12, 16)
    assert prec == gpu.FP32_MIXED or not best["fused"]
    t.run(3)
    t.sync()
    b = t.download()
    t.close()
    ref = gpu.TracerStep(case, precision=prec)
    ref.start()
    ref.set_tuning(**best)
    ref.run(5)
    ref.sync()
    a = ref.download()
    ref.close()
    np.testing.assert_array_equal(a[:, 1:], b[:, 1:])
    u = gpu.TracerStep(case, precision=prec)
    u.start()
    best2, cached2 = u.autotune_ex(1)
    u.close()
    assert cached2 and best2 == best


@pytest.mark.parametrize("tx", [8, 16, 32])
def test_fused_tile_shapes_agree(tx):
    """FP32-mixed fused sub-step: every tile width and phase-B warp count
    gives the same tracers bit for bit (tiles only regroup columns)."""
    case = synth.make("small", seed=49)
    out = []
    for tile_x, nwb in ((8, None), (tx, 1)):
        t = gpu.TracerStep(case, precision=gpu.FP32_MIXED)
        t.start()
        kw = dict(fused=1, tile_x=tile_x)
        if nwb:
            kw["phase_b_warps"] = nwb
        else:
            kw["phase_b_warps"] = t.get_tuning()["phase_b_warps"] or 1
        t.set_tuning(**kw)
        t.run(4)
        t.sync()
        out.append(t.download())
        t.close()
    np.testing.assert_array_equal(out[0], out[1])


@pytest.mark.parametrize("name", sorted(SCHEME_CASES))
def test_other_schemes_match_reference_fixture(name):
    """ORDER1, ORDER2, ORDER4, QUICKEST_CO and ORDER2_UW, with and without
    ULTIMATE, sub-steps, a moving surface and horizontal diffusion: bitwise
    equal to the reference's own tracers.c (tests/golden, make_golden.py)."""
    case, nsteps = build(name)
    g = np.load(os.path.join(HERE, "golden", name + ".npz"))
    assert input_digest(case) == str(g["digest"])
    tr, sur, nsur, d = run_resident(case, nsteps)
    np.testing.assert_array_equal(sur, g["sur_t"])
    np.testing.assert_array_equal(nsur, g["nsur_t"])
    assert_same(tr, g["tr"], case, name)
    # the same scheme with FP32 storage (FP64 arithmetic in the general path)
    tr32 = run_resident(case, nsteps, precision=gpu.FP32_MIXED)[0]
    wet = case.win.wet_cells()
    err = np.abs(tr32[:, wet] - g["tr"][:, wet]).max(axis=1) / np.abs(g["tr"][:, wet]).max(axis=1)
    assert np.all(err <= 1e-5), err
