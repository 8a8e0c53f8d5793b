"""One basin decomposed into strips (ems_b200.decomp): halo exchange once per
step, halos 2 x (sub-steps per step) columns wide, and the basin-wide
sub-step length (each strip's minimum over its own columns, then the
smallest).  The owned columns must step bit for bit as in the undivided
basin.

On the CPU the strips are stepped by the oracle (the C restatement pinned to
the reference), in one process and over two gloo ranks; on the GPU by the
library itself, two strips as two handles on one device, exchanging through
the library's halo pack / unpack on device buffers.
"""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

import oracle
from ems_b200 import decomp, synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
STEPS = 5


def basin():
    # two sub-steps per step: halos of four columns
    return synth.make("drop512", nx=40, ny=24, seed=7), 4


def oracle_strip_step(strip, state, dmin):
    tr, sur, nsur = state
    oracle.set_strip(strip.owned2d, dmin)
    try:
        rc, _, _, _, d = oracle.run_oracle(strip.case, 1, tr, sur, nsur)
    finally:
        oracle.set_strip()
    assert rc == 0
    return d


def oracle_strip_min(strip, state):
    tr, sur, nsur = state
    oracle.set_strip(strip.owned2d, 0.0)
    try:
        d = oracle.run_oracle(strip.case, 1, tr.copy(), sur.copy(), nsur.copy())[4]
    finally:
        oracle.set_strip()
    return d.dtm


def test_split_and_plan_are_consistent():
    case, halo = basin()
    P = 3
    strips = [decomp.Strip(case, P, r, halo=halo) for r in range(P)]
    owned = np.concatenate([s.own_global for s in strips])
    assert np.array_equal(np.sort(owned), np.sort(case.win.wet_cells()))  # a partition
    for r, s in enumerate(strips):
        for q, (send, recv) in s.plan.items():
            qsend = strips[q].plan[r][0]
            assert len(recv) == len(qsend) > 0
            # the same basin cells on both sides, in the same order
            g_recv = s.case.global_cells[np.searchsorted(s.case.local_cells, recv)]
            g_send = strips[q].case.global_cells[np.searchsorted(strips[q].case.local_cells,
                                                                 qsend)]
            assert np.array_equal(g_recv, g_send)


def test_strips_step_like_the_basin_in_one_process():
    case, halo = basin()
    ref = oracle.run_oracle(case, STEPS)
    assert ref[0] == 0 and ref[4].nsub == 2
    P = 3
    strips = [decomp.Strip(case, P, r, halo=halo) for r in range(P)]
    states = [s.case.copy_state() for s in strips]
    for _ in range(STEPS):
        dmin = min(oracle_strip_min(s, st) for s, st in zip(strips, states))
        for s, st in zip(strips, states):
            assert oracle_strip_step(s, st, dmin).nsub == 2
        for r, s in enumerate(strips):
            for q, (send, recv) in s.plan.items():
                states[r][0][:, recv] = states[q][0][:, strips[q].plan[r][0]]
    out = np.zeros_like(ref[1])
    for s, st in zip(strips, states):
        out[:, s.own_global] = st[0][:, s.own_local]
    w = case.win.wet_cells()
    np.testing.assert_array_equal(out[:, w], ref[1][:, w])


def _port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import datetime

    import torch
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    try:
        case, halo = basin()
        strip = decomp.Strip(case, world, rank, halo=halo)
        state = strip.case.copy_state()
        for _ in range(STEPS):
            t = torch.tensor([oracle_strip_min(strip, state)], dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MIN)
            oracle_strip_step(strip, state, float(t.item()))
            decomp.exchange_host(dist, strip, state[0])
        vals = torch.from_numpy(np.ascontiguousarray(state[0][:, strip.own_local]))
        cells = torch.from_numpy(strip.own_global.astype(np.int64))
        if rank == 0:
            out = np.zeros_like(case.tr)
            out[:, strip.own_global] = vals.numpy()
            for r in range(1, world):
                n = torch.zeros(1, dtype=torch.int64)
                dist.recv(n, r)
                c = torch.zeros(int(n.item()), dtype=torch.int64)
                v = torch.zeros((case.ntr, int(n.item())), dtype=torch.float64)
                dist.recv(c, r)
                dist.recv(v, r)
                out[:, c.numpy()] = v.numpy()
            ref = oracle.run_oracle(case, STEPS)[1]
            w = case.win.wet_cells()
            q.put(bool(np.array_equal(out[:, w], ref[:, w])))
        else:
            dist.send(torch.tensor([len(cells)], dtype=torch.int64), 0)
            dist.send(cells, 0)
            dist.send(vals, 0)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_step_like_the_basin():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    same = q.get(timeout=300)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert same


@pytest.mark.gpu
@pytest.mark.usefixtures("need_gpu")
def test_two_strips_on_one_gpu_step_like_the_basin():
    """Two handles (two strips) on one device, exchanging through the
    library's halo pack / unpack on device tensors between steps, against
    the undivided basin on the GPU: owned columns bitwise equal, and the
    strips' owned-column masses add up to the basin's."""
    import torch
    from ems_b200 import gpu
    case, halo = basin()
    whole = gpu.TracerStep(case)
    whole.start()
    whole.run(STEPS)
    whole.sync()
    ref = whole.download()
    mref = whole.mass()
    whole.close()
    P = 2
    strips = [decomp.Strip(case, P, r, halo=halo) for r in range(P)]
    steps = []
    for s in strips:
        t = gpu.TracerStep(s.case)
        t.start()
        t.set_owned(s.owned2d)
        t.halo_plan(s.send_cells(), s.recv_cells())
        steps.append(t)
    dev = torch.device("cuda", 0)
    for _ in range(STEPS):
        dmin = min(t.substep_min() for t in steps)
        for t in steps:
            t.set_substep_min(dmin)
            t.run(1)
            assert t.sync().nsub == 2
        # strip 0 sends to 1 and receives from 1 (and the other way round)
        bufs = []
        for s, t in zip(strips, steps):
            b = torch.empty((case.ntr, len(s.send_cells())), dtype=torch.float64, device=dev)
            t.halo_pack(b.data_ptr())
            bufs.append(b)
        for r, t in enumerate(steps):
            q = 1 - r
            b = bufs[q].contiguous()
            assert b.shape[1] == len(strips[r].recv_cells())
            t.halo_unpack(b.data_ptr())
            t.sync()
    out = np.zeros_like(ref)
    m = np.zeros(case.ntr)
    for s, t in zip(strips, steps):
        tr = t.download()
        out[:, s.own_global] = tr[:, s.own_local]
        m += t.mass_region(s.owned2d, 1)
        t.close()
    w = case.win.wet_cells()
    np.testing.assert_array_equal(out[:, w], ref[:, w])
    assert np.all(np.abs(m - mref) <= 1e-12 * np.abs(mref))
