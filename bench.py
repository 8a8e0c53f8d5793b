"""Tracer-transport throughput on B200: tracer cell-steps per second.

One step = one SHOC tracer step (lateral ghost fill, set_dz, advection with
sub-stepping, surf_conc, tr_bounds, implicit vertical diffusion) over every
wet cell and tracer of the workload window.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--workload stiff2048] [--precision fp32mixed|fp64] [--no-fp64]

The headline is the FP32-mixed path; the same line carries the plain FP64
path run on the same inputs (its throughput, the speed-up, and the largest
per-tracer error max|x32 - x64| / max|x64| after the same steps) and the
FP64 mass drift of both over the run.

Multi-GPU (torchrun, one process per GPU): every rank steps its own
independent basin (a differently seeded copy of the workload), with no
collective on the data path -- weak scaling; the timing is the max over
ranks.  With --workload batch8 the eight basins of the multi-basin
configuration are shared out instead, largest first to the rank with the
least work (strong scaling: the job is the same eight basins at every N).
Rank 0 prints one JSON line.

The reference arm (--impl reference) times the reference's own
model/hd/tracers/tracers.c (compiled unmodified into oracle/_ref, OpenMP
tracer loop over all host cores) on the same workload window: one untimed
step, then --steps steps in one call, timed around the step loop alone.  It
builds the window with the oracle's own build of the window builder
(oracle/_lib), so that process loads no library of this package.  The
cpu_baseline of the GPU arm's line is the same reference build on a bounded
sample (a 512x256 window of the workload, one step).
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Tracer cell-steps/s, 1 B200: batched FP32-mixed vs plain FP64, at <=1e-5 error"
UNIT = "tracer cell-steps/s"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--workload", default="stiff2048")
    p.add_argument("--precision", default="fp32mixed", choices=["fp64", "fp32mixed", "fp32comp"])
    p.add_argument("--no-fp64", action="store_true",
                   help="skip the plain FP64 arm that the mixed-precision line compares with")
    p.add_argument("--size", default="",
                   help="NXxNY: the workload's grid at another horizontal size (profiling)")
    p.add_argument("--e2e-steps", type=int, default=3)
    p.add_argument("--cpu-sample", default="512x256")
    p.add_argument("--no-cpu", action="store_true")
    p.add_argument("--no-autotune", action="store_true",
                   help="keep the library's default launch configuration")
    return p.parse_args()


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.idx), "--query-gpu=" + self.Q,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm = [float(r[1]) for r in self.rows if len(r) >= 9 and r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in self.rows if len(r) >= 9 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            if len(r) >= 9:
                for nm, v in zip(names, r[5:9]):
                    if v.strip().lower() == "active":
                        reasons.add(nm)
        sm_sorted = sorted(sm)
        med = sm_sorted[len(sm_sorted) // 2] if sm_sorted else None
        return {"sm_mhz": med, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_init():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        backend = "nccl" if os.environ.get("BENCH_BACKEND", "nccl") == "nccl" else "gloo"
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
        pg = dist
    return world, rank, local, pg


def sum_over_ranks(pg, x, device):
    """Sum of one number over the ranks (the whole job's work)."""
    if pg is None:
        return x
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    pg.all_reduce(t, op=pg.ReduceOp.SUM)
    return float(t.item())


def max_over_ranks(pg, x, device):
    if pg is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def mass_over_ranks(pg, mass, device):
    """Whole-job mass per tracer: every rank's per-tracer masses are gathered
    and summed in rank order with Neumaier compensation, so every rank holds
    the same bits.  The one collective of the multi-GPU path (outside the
    timed steps); each rank's basin needs no exchange while it steps."""
    m = np.asarray(mass, np.float64)
    if pg is None:
        return m
    import torch
    t = torch.tensor(m, dtype=torch.float64, device=device)
    parts = [torch.empty_like(t) for _ in range(pg.get_world_size())]
    pg.all_gather(parts, t)
    return compensated_sum([p.cpu().numpy() for p in parts])


def compensated_sum(rows):
    """Element-wise Neumaier sum of equal-length rows, in row order."""
    s = np.zeros_like(np.asarray(rows[0], np.float64))
    c = np.zeros_like(s)
    for v in rows:
        v = np.asarray(v, np.float64)
        u = s + v
        c += np.where(np.abs(s) >= np.abs(v), (s - u) + v, (v - u) + s)
        s = u
    return s + c


def cpu_threads():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def workload_case(args, seed, sample=False, which=None):
    """The arm's window (sample: the bounded CPU sample of it; which: the
    basins of a multi-basin workload this rank steps)."""
    from ems_b200 import synth
    kw = {} if which is None else {"which": which}
    if sample:
        if args.workload in ("batch8", "batch8small"):
            # the eight basins at 1/16 of their horizontal size
            return synth.make(args.workload, seed=seed, scale=1.0 / 16)
        kw["nx"], kw["ny"] = (int(v) for v in args.cpu_sample.split("x"))
    elif args.size:
        kw["nx"], kw["ny"] = (int(v) for v in args.size.split("x"))
    return synth.make(args.workload, seed=seed, **kw)


def reference_time(case, steps, warmup, nthr):
    """(status, seconds per step) of the reference's tracers.c: `warmup`
    untimed steps, then `steps` steps in one call timed around its step
    loop."""
    import oracle
    tr, sur, nsur = case.copy_state()
    if warmup > 0:
        rc = oracle.run_ref(case, warmup, tr, sur, nsur, nthreads=nthr)[0]
        if rc:
            return rc, None
    rc = oracle.run_ref(case, steps, tr, sur, nsur, nthreads=nthr)[0]
    return rc, oracle.ref_loop_seconds(nthr) / max(steps, 1)


# full-window steps the reference arm times at most (about 32 s each on 16
# host cores at stiff2048), so that the arm ends within a few minutes
REF_MAX_STEPS = 3


def run_reference(args, rank, world, sample=False):
    """The reference's tracers.c (oracle/_ref) on the workload window, or on
    its bounded sample for the cpu_baseline of the GPU arm.  On the full
    window at most REF_MAX_STEPS of the requested steps are timed: the
    per-step cost of the CPU path is the same every step."""
    import oracle
    if rank != 0:
        return None
    if not oracle.ref_available(omp=True):
        return {"impl": "reference",
                "unavailable": "reference build oracle/_ref/libshoc_ref_omp.so not present"}
    from ems_b200 import synth
    if not sample and synth._lib is None:
        # this process (the reference arm) builds its window with the
        # oracle's copy of the window builder and loads nothing of the
        # package's native code
        from oracle import build as obuild
        synth.use_grid_lib(obuild.grid_lib())
    case = workload_case(args, seed=2048, sample=sample)
    nthr = cpu_threads()
    warm = 1 if args.warmup > 0 else 0  # the CPU path has no caches or clocks to warm
    nsteps = args.steps if sample else max(1, min(args.steps, REF_MAX_STEPS))
    rc, sec = reference_time(case, nsteps, warm, nthr)
    if rc:
        return {"impl": "reference", "unavailable": "reference step failed: status %d" % rc}
    ms = 1000.0 * sec
    units = case.cell_tracers()
    value = units / sec
    if sample:
        size = ("basins at 1/16 size" if args.workload.startswith("batch8") else
                "%s cells" % args.cpu_sample)
        desc = ("%s window, %s x %d layers, %d wet cells x %d tracers, %d step(s) timed" %
                (args.workload, size, case.win.nz, case.nwet, case.ntr, nsteps))
    else:
        desc = ("the full %s window (%dx%dx%d, %d wet cells x %d tracers), %d untimed + %d "
                "timed steps in one call (of %d requested), step loop timed" %
                (args.workload, case.win.nx, case.win.ny, case.win.nz, case.nwet, case.ntr,
                 warm, nsteps, args.steps))
    return {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": nsteps, "steps_requested": args.steps, "warmup": warm,
            "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "impl": "reference",
            "config": {"workload": args.workload + ("@" + args.size if args.size else ""),
                       "nx": case.win.nx, "ny": case.win.ny, "nz": case.win.nz,
                       "tracers": case.ntr, "wet_cells": case.nwet, "cell_tracers": units,
                       "seed": case.seed, "sample": args.cpu_sample if sample else None},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": nthr, "kind": "reference",
                             "sample": desc},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}


def kernel_bytes(case, kernel, fp64, comp=False):
    """Algorithmic HBM bytes of one launch of a transport kernel: every tracer
    value read once and written once (8 bytes FP64, 4 FP32, 6 FP32 with its
    16-bit compensation), plus its per-cell fields (advection: u1flux3d,
    u2flux3d, w, dz; column kernel: the four LU factors; the fused sub-step
    kernel: the five fields of a step, u1flux3d, u2flux3d, w, Kz through the
    LU factors, dz)."""
    s = 8 if fp64 else 4
    st = 6 if comp else s
    fields = 5 if kernel == "k_step32" else 4
    return case.cell_tracers() * 2 * st + case.nwet * fields * s


# device bytes per cell of a plain FP64 window besides its two tracer
# buffers: flow fields, work arrays, LU factors and tile tables (an upper
# estimate)
FP64_CELL_BYTES = 480


def host_room(case):
    """Whether the host can hold two FP64 copies of every tracer besides
    what it holds now (the sequential comparison of host_compare)."""
    import psutil
    need = 2 * case.ntr * case.win.sgsiz * 8
    return psutil.virtual_memory().available > 1.5 * need


def host_compare(case, x32, x64, basins):
    """compare() on the host for two [ntr][sgsiz] tracer arrays: per region
    (basin, or the whole window) and tracer, over the region's wet cells."""
    c = case.win.wet_cells()
    if basins:
        reg = case.basin2d[case.win.m2d[c]]
        groups = [c[reg == b] for b in range(len(basins))]
    else:
        groups = [c]
    shape = (len(groups), case.ntr)
    d = {k: np.zeros(shape) for k in ("max_abs", "max_ref", "sumsq_diff", "sumsq_ref")}
    for g, cells in enumerate(groups):
        for n in range(case.ntr):
            a, r = x32[n, cells], x64[n, cells]
            e = a - r
            d["max_abs"][g, n] = np.abs(e).max() if e.size else 0.0
            d["max_ref"][g, n] = np.abs(r).max() if r.size else 0.0
            d["sumsq_diff"][g, n] = float(np.dot(e, e))
            d["sumsq_ref"][g, n] = float(np.dot(r, r))
    with np.errstate(divide="ignore", invalid="ignore"):
        d["max_rel"] = np.where(d["max_ref"] > 0, d["max_abs"] / d["max_ref"], np.nan)
        d["rms_rel"] = np.where(d["sumsq_ref"] > 0, np.sqrt(d["sumsq_diff"] / d["sumsq_ref"]),
                                np.nan)
    return d


def time_arm(case, prec, local, args, pg, dev, clocks=None):
    """Warm up, then time args.steps graph-replayed steps on the library's
    stream (CUDA events, barrier + synchronize on both sides, max over
    ranks); then one profiled pass for the per-kernel split."""
    import torch
    from ems_b200 import _abi, gpu
    step = gpu.TracerStep(case, precision=prec, device=local)
    step.start()
    tuning, cached = None, None
    if not args.no_autotune:
        # the autotuner's trial steps start from a device copy of the state
        # and put it back (untimed); its choice is cached per GPU and window
        try:
            tuning, cached = step.autotune_ex(2)
        except _abi.StatusError as e:
            if e.code != 8:  # SHOC_TR_ENOMEM
                raise
            # no device memory left for the copy: the default configuration
            tuning, cached = dict(step.get_tuning(), autotune="skipped: no room for the "
                                  "state copy"), False
    own0 = step.mass()
    m0 = mass_over_ranks(pg, own0, dev)
    stream = torch.cuda.ExternalStream(step.stream(), device=dev)
    step.run(max(args.warmup, 3))
    step.sync()
    if pg is not None:
        pg.barrier()
    torch.cuda.synchronize()
    if clocks:
        clocks.start()
    l0 = step.launches()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    step.run(args.steps)
    e1.record(stream)
    diag = step.sync()
    torch.cuda.synchronize()
    clk = clocks.stop() if clocks else None
    launches = step.launches() - l0
    ms_step = max_over_ranks(pg, e0.elapsed_time(e1), dev) / args.steps
    # per-kernel times (profile mode launches the same kernels with events)
    step.profile(True)
    step.run(args.steps)
    step.sync()
    parts = [step.kernel_time(p)[0] for p in range(3)]
    step.profile(False)
    own1 = step.mass()
    m1 = mass_over_ranks(pg, own1, dev)
    drift = float(np.max(np.abs(m1 - m0) / np.maximum(np.abs(m0), 1e-300)))
    # the largest drift of any one rank's basin (a gain on one rank and a
    # loss on another could cancel in the whole-job figure)
    own = float(np.max(np.abs(own1 - own0) / np.maximum(np.abs(own0), 1e-300)))
    return dict(step=step, ms_step=ms_step, launches=launches, clocks=clk, diag=diag,
                parts=parts, mass_drift=drift, mass_drift_rank_max=max_over_ranks(pg, own, dev),
                nsteps=max(args.warmup, 3) + 2 * args.steps,
                tuning=dict(tuning, cached=cached) if tuning else None)


def main():
    args = parse()
    world, rank, local, pg = dist_init()
    if args.impl == "reference":
        out = run_reference(args, rank, world)
        if out is not None:
            print(json.dumps(out))
        if pg is not None:
            pg.destroy_process_group()
        return

    import torch

    from ems_b200 import gpu, synth

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    mixed = args.precision in ("fp32mixed", "fp32comp")
    comp = args.precision == "fp32comp"
    shared = args.workload in ("batch8", "batch8small") and world > 1
    if shared:
        # the eight basins shared out over the ranks (strong scaling)
        which = synth.batch_partition(synth.BATCH8, world)[rank]
        case = workload_case(args, seed=2048, which=which)
    else:
        which = None
        case = workload_case(args, seed=2048 + rank)
    units = case.cell_tracers()
    job_units = sum_over_ranks(pg, units, dev)  # every rank's work
    host_gb = case.ntr * case.win.sgsiz * 8 / 1e9  # one FP64 copy of all tracers

    # the headline arm (timed with clocks sampled), then the plain FP64 arm on
    # the same inputs for the speed-up and the error of the mixed precision
    arm = time_arm(case, gpu.FP32_COMP if comp else gpu.FP32_MIXED if mixed else gpu.FP64,
                   local, args, pg, dev,
                   ClockSampler(local))
    step = arm["step"]
    fp64 = None
    basins = getattr(case, "basins", None)
    both_fit = case.win.sgsiz * (2 * case.ntr * 8 + FP64_CELL_BYTES) < torch.cuda.mem_get_info(dev)[0]
    if mixed and not args.no_fp64 and not both_fit and not host_room(case):
        fp64 = {"skipped": "the FP64 window fits neither beside the mixed one on the device "
                           "nor, sequentially, in host memory"}
    elif mixed and not args.no_fp64:
        d = None
        if not both_fit:
            # the FP64 window does not fit beside the mixed one: the mixed
            # run's tracers go to the host, its window is freed, and the two
            # are compared on the host after the FP64 run
            x32 = step.download()
            step.close()
            step = arm["step"] = None
        ref = time_arm(case, gpu.FP64, local, args, pg, dev)
        if not both_fit:
            d = host_compare(case, x32, ref["step"].download(), basins)
            del x32
        # both precisions have stepped the same inputs the same number of
        # steps: per tracer (and basin) max |x32 - x64| / max |x64|
        if basins:
            if d is None:
                d = step.compare(ref["step"], region=case.basin2d, nregion=len(basins))
            per = [[float(v) for v in d["max_rel"][b, :T]] for b, (_, _, _, T) in
                   enumerate(basins)]
            err = max(max(r) for r in per)
            rms = max(float(v) for b, (_, _, _, T) in enumerate(basins)
                      for v in d["rms_rel"][b, :T])
        else:
            if d is None:
                d = step.compare(ref["step"])
            per = [float(v) for v in d["max_rel"][0]]
            err = max(per)
            rms = float(np.nanmax(d["rms_rel"][0]))
        err = max_over_ranks(pg, err, dev)
        fp64 = {"value": job_units / (ref["ms_step"] / 1000.0), "tuning": ref["tuning"],
                "ms_per_step": ref["ms_step"], "transport_ms": ref["parts"][0],
                "kernels_ms": {"k_adv64": ref["parts"][1], "k_vd64": ref["parts"][2]},
                "mass_rel_drift": ref["mass_drift"],
                "speedup_fp32mixed": ref["ms_step"] / arm["ms_step"],
                "max_rel_err_fp32mixed": err, "max_rms_rel_err_fp32mixed": rms,
                ("max_rel_err_per_basin" if basins else "max_rel_err_per_tracer"): per,
                "steps_compared": arm["nsteps"],
                "compared_on": "device" if both_fit else "host (windows run one after the other)"}
        ref["step"].close()

    value = job_units / (arm["ms_step"] / 1000.0)
    hbm, peak_kind = peaks()
    f64b = not mixed
    # the dominant transport kernel and its roofline
    if mixed and arm["parts"][2] == 0.0:  # one fused launch per sub-step
        kern = {"k_step32": arm["parts"][1]}
    elif mixed:
        kern = {"k_adv32": arm["parts"][1], "k_vd32": arm["parts"][2]}
    else:
        kern = {"k_adv64": arm["parts"][1], "k_vd64": arm["parts"][2]}
    kname = max(kern, key=kern.get)
    kms = kern[kname]
    kb = kernel_bytes(case, kname, f64b, comp)
    achieved = kb / (kms / 1000.0) / 1e9 if kms > 0 else 0.0
    traffic = None
    try:
        if args.size:  # the recorded traffic is of the workload's own size
            raise KeyError(args.size)
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            t = json.load(f).get("%s/%s/%s" % (kname, args.workload, args.precision))
        if t:
            traffic = t
    except Exception:
        pass
    step_bytes = case.bytes_per_step(fp64=f64b)

    # end to end through the drop-in C-ABI call on pinned host buffers
    S = case.win.sgsiz
    e2e_s = float("nan")
    if args.e2e_steps > 0 and host_gb <= 16.0 and step is not None:
        tr_host = case.tr.copy()
        sur, nsur = case.sur_t.copy(), case.nsur_t.copy()
        # every array the call copies is page-locked once, as a host model
        # keeping its window arrays for the run would do
        names = ["u1", "u2", "w", "u1flux3d", "u2flux3d", "Kz", "eta", "oldeta"]
        if case.diffuse.any():
            names += ["dzu1", "dzu2", "u1kh", "u2kh"]
        flow = [getattr(case, k) for k in names]
        with gpu.HostPinned([tr_host] + flow):
            step.step(tr_host, sur, nsur)  # warm: the drop-in call re-uploads everything
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            for _ in range(args.e2e_steps):
                step.step(tr_host, sur, nsur)
            e2e_s = (time.perf_counter() - t0) / args.e2e_steps
        del tr_host
    e2e_s = max_over_ranks(pg, e2e_s, dev)
    h2d = (case.ntr * S * 8 + (10 if case.diffuse.any() else 6) * S * 8 +
           2 * case.win.sgsizS * 8 + 2 * case.win.geom.b2_t * 4)
    d2h = case.ntr * S * 8 + 2 * case.win.geom.b2_t * 4

    cpu = None
    if rank == 0 and not args.no_cpu:
        rr = run_reference(argparse.Namespace(**dict(vars(args), steps=1, warmup=0)), 0, 1,
                           sample=True)
        if rr and "value" in rr:
            cpu = rr["cpu_baseline"]

    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": arm["ms_step"],
        "higher_is_better": True, "scaling": "strong" if shared else "weak",
        "vs_baseline": None,
        "dtype": "f32-comp" if comp else "f32-mixed" if mixed else "f64", "data": "synthetic",
        "config": {
            "workload": args.workload + ("@" + args.size if args.size else ""), "nx": case.win.nx, "ny": case.win.ny,
            "nz": case.win.nz, "tracers": case.ntr, "wet_cells": case.nwet,
            "cell_tracers": units,
            "basins": [list(b) for b in getattr(case, "basins", [])] or None,
            "columns": case.win.ncol, "precision": args.precision, "dt": case.dt,
            "substeps": arm["diag"].nsub, "seed": case.seed,
            "tuning": arm["tuning"],
            "l2": "inputs larger than L2 (%.1f GB of tracers and fields per step)" % (
                step_bytes / 1e9),
            "parallelism": ("basins shared out over GPUs: %s" % synth.batch_partition(
                synth.BATCH8, world) if shared else
                "independent basin per GPU" if world > 1 else "single GPU"),
        },
        "fp64": fp64,
        "mass_rel_drift": arm["mass_drift"],
        "mass_rel_drift_rank_max": arm["mass_drift_rank_max"],
        "clocks": arm["clocks"],
        "e2e": {"value": job_units / e2e_s if e2e_s == e2e_s else None, "unit": UNIT,
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "path": "shoc_tr_gpu_step on page-locked host arrays (copies inside the timing)"},
        "gpu_launches": arm["launches"],
        "kernels_ms": dict(kern, transport=arm["parts"][0]),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": achieved / hbm, "traffic": traffic, "kernel": kname,
                     "kernel_ms": kms, "algorithmic_bytes_per_launch": kb,
                     "peak_source": peak_kind,
                     "step_achieved": step_bytes / (arm["ms_step"] / 1000.0) / 1e9,
                     "step_frac": step_bytes / (arm["ms_step"] / 1000.0) / 1e9 / hbm},
        "cpu_baseline": cpu,
    }
    if rank == 0:
        print(json.dumps(out))
    if step is not None:
        step.close()
    if pg is not None:
        pg.barrier()
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
