"""The multi-rank plumbing of bench.py on CPU: two gloo ranks.

bench.py --gpus N runs one process per GPU under torchrun; each rank steps
its own differently seeded basin (weak scaling, no collective on the data
path) and the timing is the maximum over ranks.  These tests run the same
helpers with the gloo backend on two CPU processes.
"""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank), BENCH_BACKEND="gloo")
    sys.path.insert(0, ROOT)
    import argparse

    import bench
    from ems_b200 import synth
    w, r, local, pg = bench.dist_init()
    # the slowest rank's time is the job's time
    t = bench.max_over_ranks(pg, 10.0 + rank, "cpu")
    case = synth.make("small", seed=2048 + r)
    # the reference arm: rank 0 alone times the reference, the others exit
    ref = bench.run_reference(argparse.Namespace(workload="small", cpu_sample="20x14",
                                                 size="", steps=1, warmup=0), r, w)
    # whole-job mass: per-rank masses gathered and summed in rank order
    m = bench.mass_over_ranks(pg, [0.1 * (r + 1), 2.0 * (r + 1)], "cpu")
    # the whole job's work: every rank's units summed
    u = bench.sum_over_ranks(pg, 10.0 * (r + 1), "cpu")
    q.put((r, w, t, case.nwet, float(case.tr.sum()), ref is None, m.tolist(), u))
    pg.barrier()
    pg.destroy_process_group()


def test_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=300) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, w0, t0, n0, s0, none0, m0, u0), (r1, w1, t1, n1, s1, none1, m1, u1) = out
    assert (r0, r1, w0, w1) == (0, 1, 2, 2)
    assert t0 == t1 == 11.0            # max over ranks
    assert s0 != s1                    # each rank its own seeded basin
    assert none1 and (none0 is False)  # only rank 0 runs the reference arm
    assert m0 == m1 == [0.1 + 0.2, 6.0]   # the same bits on every rank
    assert u0 == u1 == 30.0


def test_compensated_sum_of_rank_masses():
    """The rank-order sum is compensated: 1e16 + 1 - 1e16 keeps the 1 that a
    plain sum loses."""
    sys.path.insert(0, ROOT)
    import bench
    got = bench.compensated_sum([[1e16, 3.0], [1.0, 4.0], [-1e16, 5.0]])
    assert got.tolist() == [1.0, 12.0]


def test_batch_basins_shared_out():
    """--workload batch8 over N ranks: every basin on exactly one rank,
    largest first to the least-loaded rank; a rank's subset keeps each
    basin's bathymetry and land as in the whole batch."""
    sys.path.insert(0, ROOT)
    import numpy as np
    from ems_b200 import synth
    for n in (1, 2, 3, 4, 8):
        parts = synth.batch_partition(synth.BATCH8, n)
        got = sorted(b for p in parts for b in p)
        assert got == list(range(8))
        loads = [sum(float(np.prod(synth.BATCH8[b])) for b in p) for p in parts]
        assert max(loads) <= max(float(np.prod(b)) for b in synth.BATCH8) + min(loads) + 1e-9
    whole = synth.make("batch8small", seed=5)
    sub = synth.make("batch8small", seed=5, which=[1, 6])
    assert sub.basins == [whole.basins[1], whole.basins[6]]
    assert sub.cell_tracers() < whole.cell_tracers()
