"""The transport-mode flow preamble restated in plain Python (TEST
INFRASTRUCTURE ONLY: tests check the device preamble against it and against
the reference's own functions, oracle.ref_preamble).

What SHOC's transport mode computes before the tracer step (transport_step,
model/hd/tracers/transport.c:436-462), for a z-level window without open
boundaries, a linear free surface, no point sources and mdx = mdy = 1:

  set_dz_at_u1 / set_dz_at_u2   model/hd/momentum/vel3d.c:720-853 / :2718-2850
  set_flux_3d (VEL3D)           vel3d.c:4041-4175
  set_dz (surfaces, membership) model/hd/tracers/tracers.c:5731-5800
  vel_w_update (CONS_W)         vel3d.c:4609-4760, wtop = detadt (vel_w_bounds,
                                vel3d.c:5144-5215), set_w_dry (vel3d.c:5116-5135)

The face columns (SHOC's w2_e1 / bot_e1 / botzu1) are read off w3_e1: one
per surface-layer cell of it, down the run of w3_e1 cells below it, with the
higher of the two floors beside the face (hd_init.c:1443).  Every value is
the reference's expression in the reference's order (Python floats are IEEE
doubles and fuse nothing), so the results are bitwise comparable.
"""
import numpy as np

DRY_FRAC = 0.05  # SHOC's DRY_FRAC (hd_params.h)


def _gt_max(a, b):
    """SHOC's max(a, b): (a) > (b) ? (a) : (b)."""
    return a if a > b else b


def _lt_min(a, b):
    return a if a < b else b


def _faces(win, w3, ne, bm):
    zm1, zp1, botz = win.zm1, win.zp1, win.botz
    run = set(int(c) for c in w3[1:ne + 1])
    out = []
    for i in range(1, ne + 1):
        c2 = int(w3[i])
        if zp1[c2] != c2:
            continue
        c, cb = c2, c2
        while zm1[c] != c and c in run:
            cb = c
            c = int(zm1[c])
        out.append((c2, cb, _gt_max(botz[bm[c2]], botz[c2])))
    return out


def preamble(case, detadt, sur=None, nsur=None):
    """dict of dzu1, dzu2, u1flux3d, u2flux3d, w [sgsiz] after the preamble,
    from case's velocities and surface; sur / nsur: the window's sur_t /
    nsur_t before the step (default: the case's)."""
    win = case.win
    g = win.geom
    S = win.sgsiz
    zm1, zp1, xm1, ym1, xp1, yp1, m2d = (win.zm1, win.zp1, win.xm1, win.ym1, win.xp1, win.yp1,
                                         win.m2d)
    gridz, botz, cellarea = win.gridz, win.botz, win.cellarea
    eta, oldeta = case.eta, case.oldeta
    out = {k: np.zeros(S) for k in ("dzu1", "dzu2", "u1flux3d", "u2flux3d", "w")}
    w3_e1 = np.ctypeslib.as_array(g.w3_e1, shape=(g.v3_e1 + 1,))
    w3_e2 = np.ctypeslib.as_array(g.w3_e2, shape=(g.v3_e2 + 1,))

    # set_dz_at_u1 / _u2 and set_flux_3d
    for w3, ne, bm, u, h, dzu, flux in (
            (w3_e1, g.v3_e1, xm1, case.u1, win.h2au1, out["dzu1"], out["u1flux3d"]),
            (w3_e2, g.v3_e2, ym1, case.u2, win.h1au2, out["dzu2"], out["u2flux3d"])):
        for c2, cb, fl in _faces(win, w3, ne, bm):
            top = _gt_max(eta[c2], eta[bm[c2]])
            top = _gt_max(top, fl)
            c = c2
            while zm1[c] != c and gridz[c] > top:
                c = int(zm1[c])
            s = c
            t = top
            while c != cb:
                bot = gridz[c]
                dzu[c] = t - bot
                t = bot
                c = int(zm1[c])
            dzu[cb] = t - fl
            c = s
            while c != c2:
                c = int(zp1[c])
                dzu[c] = dzu[s]
            # the flux of every face cell, then zero above the surface
            c = c2
            while True:
                flux[c] = u[c] * dzu[c] * h[c2] * 1.0
                if c == cb:
                    break
                c = int(zm1[c])
            c = c2
            while c < s:
                flux[c] = 0.0
                c = int(zm1[c])

    # set_dz: old and new surfaces, the columns processed; vel_w_update
    sur = case.sur_t if sur is None else sur
    nsur_old = case.nsur_t if nsur is None else nsur
    w = out["w"]
    f1, f2 = out["u1flux3d"], out["u2flux3d"]
    nsur_new = np.zeros(g.b2_t + 1, np.int64)
    for cc in range(1, g.b2_t + 1):
        cs = int(win.w2_t[cc])
        so = int(nsur_old[cc])         # set_dz: sur_t = the previous nsur_t
        c = cs
        while zm1[c] != c and gridz[c] >= eta[cs]:
            c = int(zm1[c])
        sn = c
        s = _gt_max(so, sn)
        c2 = int(m2d[s])
        top = _lt_min(eta[c2], oldeta[c2])
        bot = DRY_FRAC * case.hmin + botz[c2]
        nsur_new[cc] = sn
        if not (top > bot and s != zm1[s]):
            continue
        c = int(win.bot_t[cc])
        cs = int(m2d[c])
        w[c] = 0.0                     # wbot
        fcbot = w[c] * cellarea[cs]
        while c > so:
            xp, yp, zp = int(xp1[c]), int(yp1[c]), int(zp1[c])
            fctop = fcbot + f1[c] - f1[xp] + f2[c] - f2[yp] + 0.0
            w[zp] = fctop / cellarea[cs]
            fcbot = fctop
            c = zp
        while c > sn:
            zp = int(zp1[c])
            w[zp] = detadt[cs]
            c = zp
    # set_w_dry: wtop above the new surface cell of every column
    for cc in range(1, g.b2_t + 1):
        c = int(nsur_new[cc])
        cs = int(m2d[c])
        zp = int(zp1[c])
        while c != zp:
            w[zp] = detadt[cs]
            c = zp
            zp = int(zp1[c])
    return out
