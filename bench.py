"""Tracer-transport throughput on B200: tracer cell-steps per second.

One step = one SHOC tracer step (lateral ghost fill, set_dz, advection with
sub-stepping, surf_conc, tr_bounds, implicit vertical diffusion) over every
wet cell and tracer of the workload window.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--workload stiff2048] [--precision fp32mixed|fp64]

Multi-GPU (torchrun, one process per GPU): every rank steps its own
independent basin (a differently seeded copy of the workload), with no
collective on the data path -- weak scaling; the timing is the max over
ranks.  Rank 0 prints one JSON line.

The reference arm (--impl reference) times the reference's own
model/hd/tracers/tracers.c (compiled unmodified into oracle/_ref, OpenMP
tracer loop over all host cores) on a bounded sample of the same workload.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

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
    p.add_argument("--precision", default="fp64", choices=["fp64", "fp32mixed"])
    p.add_argument("--e2e-steps", type=int, default=3)
    p.add_argument("--cpu-sample", default="512x256")
    p.add_argument("--no-cpu", action="store_true")
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


def max_over_ranks(pg, x, device):
    if pg is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def cpu_threads():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def cpu_sample_case(args, seed):
    from ems_b200 import synth
    nx, ny = (int(v) for v in args.cpu_sample.split("x"))
    return synth.make(args.workload, seed=seed, nx=nx, ny=ny)


def run_reference(args, rank, world):
    """The reference's tracers.c (oracle/_ref) on a bounded sample."""
    import oracle
    if rank != 0:
        return None
    if not oracle.ref_available(omp=True):
        return {"impl": "reference",
                "unavailable": "reference build oracle/_ref/libshoc_ref_omp.so not present"}
    case = cpu_sample_case(args, seed=2048)
    nthr = cpu_threads()
    tr, sur, nsur = case.copy_state()
    for _ in range(max(args.warmup, 0) and 1):
        oracle.run_ref(case, 1, tr, sur, nsur, nthreads=nthr)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        rc = oracle.run_ref(case, 1, tr, sur, nsur, nthreads=nthr)[0]
        times.append(time.perf_counter() - t0)
        if rc:
            return {"impl": "reference", "unavailable": "reference step failed: status %d" % rc}
    ms = 1000.0 * sum(times) / len(times)
    value = case.nwet * case.ntr / (ms / 1000.0)
    sample = ("%s window, %s cells x %d layers, %d wet cells x %d tracers, 1 step per "
              "measured step" % (args.workload, args.cpu_sample, case.win.nz, case.nwet, case.ntr))
    return {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "impl": "reference",
            "config": {"workload": args.workload, "sample": args.cpu_sample},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": nthr, "kind": "reference",
                             "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}


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

    import numpy as np
    import torch

    from ems_b200 import gpu, synth

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    prec = gpu.FP32_MIXED if args.precision == "fp32mixed" else gpu.FP64
    case = synth.make(args.workload, seed=2048 + rank)
    step = gpu.TracerStep(case, precision=prec, device=local)
    step.start()
    stream = torch.cuda.ExternalStream(step.stream(), device=dev)

    # warm-up (also learns the sub-step schedule and captures the step graph)
    step.run(max(args.warmup, 3))
    step.sync()

    # timed region: per-step transport kernels are bracketed by CUDA events on
    # the library's stream (profile mode launches the same kernels directly)
    step.profile(True)
    if pg is not None:
        pg.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    l0 = step.launches()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    step.run(args.steps)
    e1.record(stream)
    diag = step.sync()
    torch.cuda.synchronize()
    clk = clocks.stop()
    launches = step.launches() - l0
    ms_total = e0.elapsed_time(e1)
    kern_ms, kern_n = step.kernel_time()
    step.profile(False)
    ms_total = max_over_ranks(pg, ms_total, dev)
    ms_step = ms_total / args.steps

    # graph-replay timing of the same steps (no per-kernel events)
    g0 = torch.cuda.Event(enable_timing=True)
    g1 = torch.cuda.Event(enable_timing=True)
    g0.record(stream)
    step.run(args.steps)
    g1.record(stream)
    step.sync()
    graph_ms_step = max_over_ranks(pg, g0.elapsed_time(g1), dev) / args.steps

    units = case.nwet * case.ntr
    value = units * world / (ms_step / 1000.0)
    fp64 = prec == gpu.FP64
    bytes_step = case.bytes_per_step(fp64=fp64)
    hbm, peak_kind = peaks()
    achieved = bytes_step / (kern_ms / 1000.0) / 1e9 if kern_ms > 0 else 0.0

    # end to end through the drop-in C-ABI call on pinned host buffers
    S = case.win.sgsiz
    pin = torch.empty((case.ntr, S), dtype=torch.float64, pin_memory=True)
    tr_host = pin.numpy()
    tr_host[:] = case.tr
    sur, nsur = case.sur_t.copy(), case.nsur_t.copy()
    e2e_s = float("nan")
    if args.e2e_steps > 0:
        step.step(tr_host, sur, nsur)  # warm: the drop-in call re-uploads everything
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(args.e2e_steps):
            step.step(tr_host, sur, nsur)
        e2e_s = (time.perf_counter() - t0) / args.e2e_steps
    e2e_s = max_over_ranks(pg, e2e_s, dev)
    h2d = (case.ntr * S * 8 + 6 * S * 8 + 2 * case.win.sgsizS * 8 +
           2 * case.win.geom.b2_t * 4)
    d2h = case.ntr * S * 8 + 2 * case.win.geom.b2_t * 4

    cpu = None
    if rank == 0 and not args.no_cpu:
        ref = run_reference(argparse.Namespace(**dict(vars(args), steps=1, warmup=0)), 0, 1)
        if ref and "value" in ref:
            cpu = ref["cpu_baseline"]

    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if fp64 else "f32-mixed", "data": "synthetic",
        "config": {
            "workload": args.workload, "nx": case.win.nx, "ny": case.win.ny,
            "nz": case.win.nz, "tracers": case.ntr, "wet_cells": case.nwet,
            "columns": case.win.ncol, "precision": args.precision, "dt": case.dt,
            "substeps": diag.nsub, "seed": case.seed,
            "l2": "inputs larger than L2 (%.1f GB of tracers per step)" % (bytes_step / 1e9),
            "parallelism": "independent basin per GPU" if world > 1 else "single GPU",
        },
        "graph_ms_per_step": graph_ms_step,
        "clocks": clk,
        "e2e": {"value": units / e2e_s if e2e_s == e2e_s else None, "unit": UNIT, "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h,
                "path": "shoc_tr_gpu_step on pinned host arrays (copies inside the timing)"},
        "gpu_launches": launches,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": achieved / hbm, "traffic": None,
                     "kernel": "k_transport<LAST>", "kernel_ms": kern_ms,
                     "kernel_launches": kern_n, "peak_source": peak_kind,
                     "algorithmic_bytes_per_launch": bytes_step},
        "cpu_baseline": cpu,
    }
    if rank == 0:
        print(json.dumps(out))
    step.close()
    if pg is not None:
        pg.barrier()
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
