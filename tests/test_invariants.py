"""Physical invariants of the tracer step, checked on the CPU oracle:
constant fields stay constant (tracers.c:970-976), column / total mass is
conserved by the flux form and the implicit solve (:4145-4161), and the
ULTIMATE limiter creates no new extrema (:3546-3554)."""
import numpy as np

import oracle
from ems_b200 import synth


def total_mass(case, tr):
    """sum(tr * dz * area) over wet cells with the step's own dz (fixed eta)."""
    w = case.win
    c = w.wet_cells()
    top = w.cell_top(case.eta)
    bot = w.cell_bot()
    vol = (top[c] - bot[c]) * w.cellarea[w.m2d[c]]
    return (tr[:, c] * vol[None, :]).sum(axis=1)


def test_constant_field_stays_constant():
    case = synth.make("small", seed=7)
    c = case.win.wet_cells()
    case.tr[:, c] = 3.25
    rc, tr, *_ = oracle.run_oracle(case, 10)
    assert rc == 0
    assert np.abs(tr[:, c] - 3.25).max() <= 1e-12 * 3.25


def test_mass_conserved():
    case = synth.make("small", seed=9)
    m0 = total_mass(case, case.tr)
    rc, tr, *_ = oracle.run_oracle(case, 20)
    assert rc == 0
    m1 = total_mass(case, tr)
    assert np.all(np.abs(m1 - m0) <= 1e-12 * np.abs(m0))


def test_ultimate_creates_no_new_extrema():
    case = synth.make("small", seed=13, tracers="step")
    c = case.win.wet_cells()
    lo, hi = case.tr[:, c].min(axis=1), case.tr[:, c].max(axis=1)
    rc, tr, *_ = oracle.run_oracle(case, 15)
    assert rc == 0
    span = hi - lo
    assert np.all(tr[:, c].min(axis=1) >= lo - 1e-12 * span)
    assert np.all(tr[:, c].max(axis=1) <= hi + 1e-12 * span)
