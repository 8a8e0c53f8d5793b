"""One basin decomposed over several GPUs (or processes): strips of columns.

SHOC runs a multi-window model by giving each window its own cells plus the
cells of its neighbours that its stencils read, refreshed by the window
transfers (model/hd/slaves/windows.c:152 builds the windows;
slaves/transfers.c:349,769 and the MPI buffers of slaves/TransferBuffer.cpp:
282-443 move the data).  Here a basin of nx x ny columns is cut along i into
strips, one per rank.  A strip's window holds its own columns plus `halo`
columns on each side taken from its neighbours, and is an ordinary window
of the library (it is stepped whole).  QUICKEST and ULTIMATE read two cells
across a face (tracers.c:1854-1855, :3528-3530), so a value that is wrong at
the strip's outer edge moves two columns inwards per sub-step: with halos of
2 x (sub-steps per step) columns, refreshed from their owners after every
step, every owned column steps bit for bit as in the undivided basin.  The
vertical solve, surf_conc and tr_bounds are local to each column.

  Strip(case, nparts, rank, halo=2)  the strip's Case (window, flow, tracers
                                     copied by (i, j, k) from the basin's),
                                     its owned-column map and the exchange
                                     plan with each neighbour
  exchange_host(...)                 one halo exchange of host arrays over a
                                     torch.distributed group (gloo)
  exchange_device(...)               the same on device buffers through the
                                     library's halo pack / unpack (NCCL)

All ranks must take the same number of sub-steps per step (the sub-step
length is the minimum over the whole basin in the undivided run); callers
check the step diagnostics.
"""
import numpy as np

from . import synth


def split(n, parts):
    """[(a, b)) ranges of n columns in `parts` nearly equal strips."""
    edges = np.linspace(0, n, parts + 1).round().astype(int)
    return [(int(edges[p]), int(edges[p + 1])) for p in range(parts)]


def _cell_index(win):
    """(nz, ny, nx) array: the sparse cell at (k, j, i) for the window's wet
    cells (0 elsewhere)."""
    idx = np.zeros((win.nz, win.ny, win.nx), np.int64)
    c = win.wet_cells()
    idx[win.s2k[c], win.s2j[c], win.s2i[c]] = c
    return idx


def _column_index(win):
    """(ny, nx) array: the 2D (surface-layer) cell of each wet column."""
    idx = np.zeros((win.ny, win.nx), np.int64)
    c2 = win.w2_t[1:win.geom.b2_t + 1]
    idx[win.s2j[c2], win.s2i[c2]] = c2
    return idx


def strip_case(case, lo, hi):
    """The window of columns lo <= i < hi of `case`'s basin, with every field
    copied from the basin's cells at the same (i, j, k)."""
    gw = case.win
    K = gw._keep
    cols = slice(lo, hi)
    faces = slice(lo, hi + 1)
    win = synth.Window(hi - lo, gw.ny, gw.nz, K["layers"], K["bathy"][:, cols],
                       K["land"][:, cols], K["h1acell"][:, faces], K["h2acell"][:, faces],
                       K["h1au1"][:, faces], K["h2au1"][:, faces], K["h1au2"][:, faces],
                       K["h2au2"][:, faces])
    g3, g2 = _cell_index(gw), _column_index(gw)
    lw = win.wet_cells()
    gi = g3[win.s2k[lw], win.s2j[lw], win.s2i[lw] + lo]
    if np.any(gi == 0):
        raise ValueError("strip cells missing from the basin")
    S, S2 = win.sgsiz, win.sgsizS
    c2 = win.w2_t[1:win.geom.b2_t + 1]
    g2i = g2[win.s2j[c2], win.s2i[c2] + lo]

    def f3(a):
        out = np.zeros(S)
        out[lw] = a[gi]
        return out

    def f2(a):
        out = np.zeros(S2)
        out[c2] = a[g2i]
        return out

    tr = np.zeros((case.ntr, S))
    tr[:, lw] = case.tr[:, gi]
    sub = synth.Case(case.name + "@%d:%d" % (lo, hi), win, case.ntr, case.dt, f3(case.u1),
                     f3(case.u2), f3(case.w), f3(case.u1flux3d), f3(case.u2flux3d), f3(case.Kz),
                     f2(case.eta), f2(case.oldeta), tr, trasc=case.trasc,
                     ultimate=case.ultimate, stab=case.stab, hmin=case.hmin,
                     mintr=case.mintr, maxtr=case.maxtr, seed=case.seed, nsteps=case.nsteps,
                     dzu1=f3(case.dzu1), dzu2=f3(case.dzu2), u1kh=f3(case.u1kh),
                     u2kh=f3(case.u2kh), diffuse=case.diffuse)
    sub.global_cells = gi        # basin cell of each of the strip's wet cells
    sub.local_cells = lw
    return sub


class Strip:
    """Rank `rank`'s strip of `case`'s basin cut into `nparts` strips along i,
    with `halo` columns on each side (2 x the sub-steps per step)."""

    def __init__(self, case, nparts, rank, halo=2):
        self.parts = split(case.win.nx, nparts)
        self.rank, self.nparts, self.halo = rank, nparts, halo
        a, b = self.parts[rank]
        if b - a < halo:
            raise ValueError("strips narrower than the halo")
        self.lo, self.hi = max(0, a - halo), min(case.win.nx, b + halo)
        self.a, self.b = a, b
        self.case = strip_case(case, self.lo, self.hi)
        w = self.case.win
        # 1 on the strip's own columns (2D cells), 0 on the halo
        self.owned2d = np.zeros(w.sgsizS, np.int32)
        c2 = w.w2_t[1:w.geom.b2_t + 1]
        gi2 = w.s2i[c2] + self.lo
        self.owned2d[c2[(gi2 >= a) & (gi2 < b)]] = 1
        # the strip's own wet cells (local) and their basin cells
        lw = self.case.local_cells
        gi = w.s2i[lw] + self.lo
        own = (gi >= a) & (gi < b)
        self.own_local = lw[own]
        self.own_global = self.case.global_cells[own]
        # exchange plan: per neighbour q, the cells sent to q (own cells in
        # q's window) and received from q (halo cells q owns), both in
        # basin-cell order, so the two sides list the same cells alike
        self.plan = {}
        for q in (rank - 1, rank + 1):
            if q < 0 or q >= nparts:
                continue
            qa, qb = self.parts[q]
            qlo, qhi = max(0, qa - halo), min(case.win.nx, qb + halo)
            send = own & (gi >= qlo) & (gi < qhi)
            recv = (gi >= qa) & (gi < qb)
            s_loc, s_glob = lw[send], self.case.global_cells[send]
            r_loc, r_glob = lw[recv], self.case.global_cells[recv]
            self.plan[q] = (s_loc[np.argsort(s_glob)].astype(np.int32),
                            r_loc[np.argsort(r_glob)].astype(np.int32))

    def send_cells(self):
        return np.concatenate([self.plan[q][0] for q in sorted(self.plan)] or [np.zeros(0, np.int32)])

    def recv_cells(self):
        return np.concatenate([self.plan[q][1] for q in sorted(self.plan)] or [np.zeros(0, np.int32)])


def exchange_host(pg, strip, tr):
    """One halo exchange of the host tracer array tr [ntr][sgsiz] of the
    strip's window with its neighbours over the torch.distributed group pg
    (every rank calls it, in step)."""
    import torch
    reqs, recvs = [], []
    for q in sorted(strip.plan):
        send, recv = strip.plan[q]
        sbuf = torch.from_numpy(np.ascontiguousarray(tr[:, send]))
        rbuf = torch.empty((tr.shape[0], len(recv)), dtype=torch.float64)
        reqs.append(pg.isend(sbuf, q))
        reqs.append(pg.irecv(rbuf, q))
        recvs.append((recv, rbuf))
    for r in reqs:
        r.wait()
    for recv, rbuf in recvs:
        tr[:, recv] = rbuf.numpy()


def exchange_device(pg, strip, step, dtype, device):
    """One halo exchange of a strip stepped by the library (handle `step`,
    whose plan was set with step.halo_plan(strip.send_cells(),
    strip.recv_cells())): the send cells are packed on the device, moved to
    the neighbours with NCCL send / recv of device tensors, and unpacked."""
    import torch
    ntr = step.case.ntr
    ns = sum(len(strip.plan[q][0]) for q in strip.plan)
    nr = sum(len(strip.plan[q][1]) for q in strip.plan)
    sbuf = torch.empty((ntr, ns), dtype=dtype, device=device)
    rbuf = torch.empty((ntr, nr), dtype=dtype, device=device)
    step.halo_pack(sbuf.data_ptr())
    reqs, so, ro, parts = [], 0, 0, []
    for q in sorted(strip.plan):
        n_s, n_r = len(strip.plan[q][0]), len(strip.plan[q][1])
        s = sbuf[:, so:so + n_s].contiguous()
        r = torch.empty((ntr, n_r), dtype=dtype, device=device)
        reqs += [pg.isend(s, q), pg.irecv(r, q)]
        parts.append((ro, r, s))
        so += n_s
        ro += n_r
    for r in reqs:
        r.wait()
    for ro, r, _ in parts:
        rbuf[:, ro:ro + r.shape[1]] = r
    torch.cuda.synchronize(device)
    step.halo_unpack(rbuf.data_ptr())
