"""The SHOC-style window builder and the synthetic flow (CPU only)."""
import numpy as np

from ems_b200 import synth


def test_window_layout_and_maps():
    case = synth.make("small", seed=21)
    w = case.win
    g = w.geom
    c = w.wet_cells()
    # wet cells numbered surface layer first, i fastest within a layer
    k = w.s2k[c]
    assert np.all(np.diff(k) <= 0)
    # neighbour maps are symmetric between wet cells
    for fwd, back in ((w.xp1, w.xm1), (w.yp1, w.ym1)):
        nb = fwd[c]
        wet_nb = w.is_wet[nb].astype(bool)
        assert np.all(back[nb[wet_nb]] == c[wet_nb])
    # every ghost copies a wet neighbour; sediment cells self-map downward
    assert np.all(w.is_wet[w.bin[1:]] == 1)
    assert np.all(w.is_wet[w.bpt[1:]] == 0)
    bots = w.bot_t[1:]
    sed = w.zm1[bots]
    assert np.all(w.zm1[sed] == sed) and np.all(w.zp1[sed] == bots)
    # surface-layer cells double as the 2D index
    assert np.all(w.m2d[c] == w.map_top[w.s2j[c], w.s2i[c]])
    assert g.a3_t == w.nwet and g.b2_t == w.ncol


def test_flow_is_column_divergence_free():
    case = synth.make("small", seed=23)
    w = case.win
    c = w.wet_cells()
    div = (case.u1flux3d[w.xp1[c]] - case.u1flux3d[c] +
           case.u2flux3d[w.yp1[c]] - case.u2flux3d[c])
    col = np.zeros(w.sgsizS)
    np.add.at(col, w.m2d[c], div)
    scale = np.abs(case.u1flux3d).max()
    assert np.abs(col).max() <= 1e-9 * scale
    # w from continuity is ~0 at the free surface: the surface cell's inflow
    # from below balances its horizontal divergence
    top = w.w2_t[1:w.geom.b2_t + 1]
    fctop = (case.w[top] * w.cellarea[top] + case.u1flux3d[top] - case.u1flux3d[w.xp1[top]] +
             case.u2flux3d[top] - case.u2flux3d[w.yp1[top]])
    assert np.abs(fctop).max() <= 1e-9 * scale
    assert np.abs(case.u1).max() > 0 and np.abs(case.w[c]).max() > 0


def test_workload_sizes():
    case = synth.make("basin64")
    assert case.win.nx == 64 and case.win.nz == 20 and case.ntr == 1
    assert case.win.ncol == 64 * 64  # no land


def test_batch_window_basins_and_tracer_counts():
    """batch8small: eight basins side by side; every wet column carries its
    basin's tracer count (4, 8, ... 32) and no basin touches another."""
    import numpy as np
    from ems_b200 import synth
    case = synth.make("batch8small")
    w = case.win.wet_cells()
    cols = np.unique(case.win.m2d[w])
    counts = sorted(set(case.ntr2d[cols].tolist()))
    assert counts == [4, 8, 12, 16, 20, 24, 28, 32]
    # no wet column's x-neighbour column belongs to another basin
    i = case.win.s2i[w]
    nt = case.ntr2d[case.win.m2d[w]]
    xp = case.win.xp1[w]
    wet = np.zeros(case.win.sgsiz, bool)
    wet[w] = True
    nb = xp[wet[xp]]
    assert np.all(case.ntr2d[case.win.m2d[nb]] == nt[wet[xp]])
