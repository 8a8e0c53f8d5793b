"""Accuracy of the FP32-mixed step (or FP32_COMP, --precision fp32comp)
against the plain FP64 step.

Both precisions step the same window from the same state on the GPU; every
`every` steps the tracers are compared cell by cell over the wet cells:

  max relative error  = max |x32 - x64| / max |x64|          (per tracer)
  RMS relative error  = sqrt(sum (x32 - x64)^2 / sum x64^2)    (per tracer)

and each path's tracer mass (FP64 compensated sum over the water columns) is
compared with its initial value.  The FP64 path is bitwise equal to the
reference's tracers.c on the parity cases, so it stands in for the FP64
oracle at sizes the CPU cannot run for many steps.

  python -m ems_b200.accuracy --workload stiff2048 --steps 1000 --every 100

--worst also reports, per tracer, where its largest difference is (layer,
column, the column's bottom layer, the cell's velocities and Kz): the two
paths' tracers are copied to the host once, at the end.
"""
import argparse
import json
import time

import numpy as np

from . import gpu, synth


def worst_cells(case, x64, x32):
    """Per tracer: the wet cell of the largest |x32 - x64| and what is there."""
    win = case.win
    c = win.wet_cells()
    col = {int(v): i for i, v in enumerate(win.w2_t[1:win.geom.b2_t + 1], 1)}
    out = []
    for n in range(case.ntr):
        e = np.abs(x32[n, c] - x64[n, c])
        i = int(np.argmax(e))
        cell = int(c[i])
        cc = col[int(win.m2d[cell])]
        out.append({"tracer": n, "max_rel": float(e[i] / np.abs(x64[n, c]).max()),
                    "k": int(win.s2k[cell]), "i": int(win.s2i[cell]), "j": int(win.s2j[cell]),
                    "k_bottom": int(win.s2k[win.bot_t[cc]]), "x64": float(x64[n, cell]),
                    "u1": float(case.u1[cell]), "u2": float(case.u2[cell]),
                    "w": float(case.w[cell]), "Kz": float(case.Kz[cell])})
    return out


PRECISIONS = {"fp32mixed": gpu.FP32_MIXED, "fp32comp": gpu.FP32_COMP}


def compare(case, steps, every, device=0, log=None, worst=None, precision=gpu.FP32_MIXED):
    """Per-tracer errors of FP32-mixed (or FP32_COMP) vs FP64 after every
    `every` steps (compared on the device, shoc_tr_gpu_compare: no tracer
    leaves HBM).  worst: a list that receives worst_cells() after the last
    step."""
    s64 = gpu.TracerStep(case, precision=gpu.FP64, device=device)
    s32 = gpu.TracerStep(case, precision=precision, device=device)
    s64.start()
    s32.start()
    m64_0, m32_0 = s64.mass(), s32.mass()
    rows = []
    done = 0
    while done < steps:
        k = min(every, steps - done)
        s64.run(k)
        s32.run(k)
        s64.sync()
        s32.sync()
        done += k
        d = s32.compare(s64)
        mx = d["max_abs"][0] / np.maximum(d["max_ref"][0], 1e-300)
        rms = np.sqrt(d["sumsq_diff"][0] / np.maximum(d["sumsq_ref"][0], 1e-300))
        m64, m32 = s64.mass(), s32.mass()
        row = {"step": done,
               "max_rel": mx.tolist(), "rms_rel": rms.tolist(),
               "mass_drift_fp64": (np.abs(m64 - m64_0) / np.abs(m64_0)).tolist(),
               "mass_drift_fp32mixed": (np.abs(m32 - m32_0) / np.abs(m32_0)).tolist()}
        rows.append(row)
        if log:
            log("step %d: max rel %.3g, RMS rel %.3g, mass drift fp64 %.3g, fp32-mixed %.3g" % (
                done, mx.max(), rms.max(), max(row["mass_drift_fp64"]),
                max(row["mass_drift_fp32mixed"])))
    if worst is not None:
        worst.extend(worst_cells(case, s64.download(), s32.download()))
    s64.close()
    s32.close()
    return rows


def main():
    p = argparse.ArgumentParser()
    p.add_argument("--workload", default="stiff2048")
    p.add_argument("--steps", type=int, default=1000)
    p.add_argument("--every", type=int, default=100)
    p.add_argument("--seed", type=int, default=2048)
    p.add_argument("--size", default="", help="NXxNY: the workload at another size")
    p.add_argument("--json", default="")
    p.add_argument("--worst", action="store_true",
                   help="report where each tracer's largest difference is")
    p.add_argument("--precision", default="fp32mixed", choices=sorted(PRECISIONS))
    a = p.parse_args()
    kw = {}
    if a.size:
        kw["nx"], kw["ny"] = (int(v) for v in a.size.split("x"))
    case = synth.make(a.workload, seed=a.seed, **kw)
    t0 = time.time()
    worst = [] if a.worst else None
    rows = compare(case, a.steps, a.every, log=lambda s: print(s, flush=True), worst=worst,
                   precision=PRECISIONS[a.precision])
    out = {"workload": a.workload + ("@" + a.size if a.size else ""), "seed": a.seed,
           "precision": a.precision,
           "steps": a.steps, "tracers": case.ntr, "wet_cells": case.nwet,
           "seconds": time.time() - t0, "checkpoints": rows}
    if worst is not None:
        out["worst"] = worst
        for w in worst:
            print("worst", json.dumps(w))
    if a.json:
        with open(a.json, "w") as f:
            json.dump(out, f)
    last = rows[-1]
    print("per tracer after %d steps (max rel / RMS rel):" % last["step"])
    for n in range(case.ntr):
        print("  %2d  %.3e  %.3e" % (n, last["max_rel"][n], last["rms_rel"][n]))


if __name__ == "__main__":
    main()
