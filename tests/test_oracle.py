"""The CPU oracle against the reference's own tracer step (CPU only).

Golden fixtures (tests/golden, written by tests/golden/make_golden.py with the
reference's tracers.c compiled unmodified) pin the restatement in
oracle/shoc_oracle.c; where oracle/_ref is built, extra seeds are compared
with the reference directly.
"""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

import oracle  # noqa: E402
from cases import CASES, build, input_digest  # noqa: E402
from ems_b200 import _abi, synth  # noqa: E402


def load_golden(name):
    return np.load(os.path.join(HERE, "golden", name + ".npz"))


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_matches_reference_fixture(name):
    case, nsteps = build(name)
    g = load_golden(name)
    rc, tr, sur, nsur, d = oracle.run_oracle(case, nsteps)
    assert rc == int(g["status"])
    np.testing.assert_array_equal(sur, g["sur_t"])
    np.testing.assert_array_equal(nsur, g["nsur_t"])
    assert d.nwarn == int(g["nwarn"])
    if input_digest(case) == str(g["digest"]):
        # same inputs bit for bit: every slot equal, the scratch slot 0 included
        np.testing.assert_array_equal(tr, g["tr"])
    else:
        cells = np.arange(1, case.win.sgsiz)
        assert oracle.max_rel_err(tr, g["tr"], cells).max() <= 1e-12


@pytest.mark.parametrize("name", ["small_crossing", "small_crossing_substeps",
                                  "small_crossing_thin"])
def test_crossing_cases_move_the_surface_cell(name):
    """In the crossing cases eta and oldeta of most columns lie in different
    layers, so the surface cell changes during every step (the general path
    of surf_conc, and with a thin surface layer tr_bounds' cursor)."""
    case, _ = build(name)
    w = case.win
    c = w.wet_cells()
    j = w.m2d[c]
    n_new = np.bincount(j, weights=w.gridz[c] < case.eta[j], minlength=len(case.eta))
    n_old = np.bincount(j, weights=w.gridz[c] < case.oldeta[j], minlength=len(case.eta))
    assert np.sum(n_new != n_old) > 50


needs_ref = pytest.mark.skipif(not oracle.ref_available(), reason="reference build not present")


@needs_ref
@pytest.mark.parametrize("seed", [3, 17, 101])
@pytest.mark.parametrize("scheme", ["quickest", "vanleer"])
def test_oracle_bitwise_vs_reference_random_seeds(seed, scheme):
    kw = dict(trasc=_abi.QUICKEST if scheme == "quickest" else _abi.VANLEER,
              ultimate=1 if scheme == "quickest" else 0)
    case = synth.make("small", seed=seed, **kw)
    a = oracle.run_oracle(case, 8)
    b = oracle.run_ref(case, 8)
    assert a[0] == b[0] == 0
    np.testing.assert_array_equal(a[1], b[1])
    np.testing.assert_array_equal(a[2], b[2])
    np.testing.assert_array_equal(a[3], b[3])


@needs_ref
def test_reference_openmp_build_matches_serial():
    case = synth.make("small", seed=5)
    a = oracle.run_ref(case, 5)
    b = oracle.run_ref(case, 5, nthreads=4)
    cells = np.arange(1, case.win.sgsiz)
    np.testing.assert_array_equal(a[1][:, cells], b[1][:, cells])


def test_substep_limit_is_an_error():
    # more than 20 sub-steps: the reference quits (tracers.c:664-668)
    case = synth.make("small", dt=40000.0)
    rc = oracle.run_oracle(case, 1)[0]
    assert rc == 1
    if oracle.ref_available():
        assert oracle.run_ref(case, 1)[0] == 1


def test_scheme_fixtures_are_distinct_and_reproducible():
    """The other schemes' fixtures come from the same regenerated inputs and
    differ from each other and from QUICKEST (each scheme really ran)."""
    from cases import SCHEME_CASES
    seen = {}
    for name in sorted(SCHEME_CASES):
        case, nsteps = build(name)
        g = load_golden(name)
        assert input_digest(case) == str(g["digest"]) and int(g["status"]) == 0
        seen[name] = g["tr"][:, 1:]
    base = load_golden("small_quickest_ultimate")["tr"][:, 1:]
    for a in ("small_order1", "small_order2", "small_order4", "small_quickest_co",
              "small_order2_uw"):
        assert np.abs(seen[a] - base).max() > 0.0
        for b in ("small_order1", "small_order2", "small_order4", "small_quickest_co",
                  "small_order2_uw"):
            if a < b:
                assert np.abs(seen[a] - seen[b]).max() > 0.0, (a, b)
