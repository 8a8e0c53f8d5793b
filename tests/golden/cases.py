"""Golden-fixture cases: small seeded windows run through the reference build.

Each entry: name -> (workload, overrides, nsteps).  The same definitions are
used by make_golden.py (writes the fixtures with the reference's own
tracers.c, oracle/_ref) and by the tests (check the oracle and the CUDA path
against them).
"""
import hashlib

import numpy as np

from ems_b200 import _abi

MOVING = dict(layers=np.linspace(-30, 2.0, 8))
# layer faces at -1.0 and 0.6 m, inside the range of eta and oldeta: the
# surface cell of most columns changes during the step (general path; with a
# thin surface layer, tr_bounds' thin-surface cursor)
CROSS = dict(layers=np.array([-30.0, -22.0, -14.0, -8.0, -3.0, -1.0, 0.6, 2.5]))

CASES = {
    "small_quickest_ultimate": ("small", {}, 10),
    "small_vanleer": ("small", dict(trasc=_abi.VANLEER, ultimate=0), 10),
    "small_vanleer_ultimate": ("small", dict(trasc=_abi.VANLEER, ultimate=1), 10),
    "small_substeps": ("small", dict(dt=2000.0), 2),
    "small_moving_surface": ("small", dict(eta_offset=(1.9, -1.7), **MOVING), 6),
    "small_moving_substeps": ("small", dict(eta_offset=(1.9, -1.7), dt=1500.0, **MOVING), 3),
    "small_clip": ("small", dict(ultimate=0, tracers="step", mintr=[0.0, 0.0, 0.0],
                                 maxtr=[1.0, 2.0, 2.5]), 20),
    "small_thin_surface": ("small", dict(eta_offset=(1.9, -1.7), hmin=1.5,
                                         maxtr=[0.5, 0.5, 0.5], **MOVING), 4),
    "small_crossing": ("small", dict(eta_offset=(1.9, -1.7), **CROSS), 6),
    "small_crossing_substeps": ("small", dict(eta_offset=(1.9, -1.7), dt=1500.0, **CROSS), 3),
    "small_crossing_thin": ("small", dict(eta_offset=(1.9, -1.7), hmin=1.2,
                                          maxtr=[0.5, 0.5, 0.5], **CROSS), 4),
    "small_hdiff": ("small", dict(hdiff=(40.0, [1, 1, 1])), 10),
    "small_hdiff_mixed": ("small", dict(hdiff=(40.0, [1, 0, 1])), 10),
    "small_vanleer_hdiff": ("small", dict(trasc=_abi.VANLEER, ultimate=0,
                                          hdiff=(40.0, [0, 1, 1])), 10),
    "basin64": ("basin64", {}, 100),
}


# The other advection schemes (advect's dispatch, tracers.c:1509-1527),
# pinned directly against the reference build (the C restatement in
# oracle/shoc_oracle.c covers QUICKEST and Van Leer only).
O1, O2, O4, QCO, O2UW = 0x2, 0x4, 0x10, 0x40, 0x2000
SCHEME_CASES = {
    "small_order1": ("small", dict(trasc=O1, ultimate=0), 10),
    "small_order1_substeps": ("small", dict(trasc=O1, ultimate=1, dt=2000.0), 2),
    "small_order2": ("small", dict(trasc=O2, ultimate=0), 10),
    "small_order2_ultimate": ("small", dict(trasc=O2, ultimate=1), 10),
    "small_order4": ("small", dict(trasc=O4, ultimate=0), 10),
    "small_order4_ultimate_moving": ("small", dict(trasc=O4, ultimate=1,
                                                   eta_offset=(1.9, -1.7), **MOVING), 6),
    "small_quickest_co": ("small", dict(trasc=QCO, ultimate=0), 10),
    "small_quickest_co_ultimate_hdiff": ("small", dict(trasc=QCO, ultimate=1,
                                                       hdiff=(40.0, [1, 0, 1])), 10),
    "small_order2_uw": ("small", dict(trasc=O2UW, ultimate=0), 10),
    "small_order2_uw_ultimate_substeps": ("small", dict(trasc=O2UW, ultimate=1, dt=2000.0), 2),
}
ALL_CASES = dict(CASES, **SCHEME_CASES)


def build(name):
    from ems_b200 import synth
    wl, kw, nsteps = ALL_CASES[name]
    return synth.make(wl, **kw), nsteps


def input_digest(case):
    """sha256 over every array the step reads, to tell whether a fixture's
    inputs were regenerated bit for bit on this machine."""
    h = hashlib.sha256()
    w = case.win
    for a in (w.xp1, w.xm1, w.yp1, w.ym1, w.zp1, w.zm1, w.m2d, w.gridz, w.h1au1, w.h2au2,
              w.h1acell, w.h2acell, w.cellarea, w.botz, case.u1, case.u2, case.w,
              case.u1flux3d, case.u2flux3d, case.Kz, case.eta, case.oldeta, case.tr):
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()
