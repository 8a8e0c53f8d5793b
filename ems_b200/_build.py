"""Compiles the native libraries of the package in-tree.

  ems_b200/_lib/libshoc_grid.so    host C: SHOC-style sparse window builder
  ems_b200/_lib/libshoc_tr_gpu.so  CUDA sm_100a: the tracer step + C-ABI

Each library is rebuilt only when a source is newer than it.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "_lib")
INCLUDE = os.path.join(ROOT, "include")

GRID_SRC = ["shoc_grid.c"]
# (source, FMA contraction): the FP64 reference path must not contract
GPU_SRC = [("shoc_tr_gpu.cu", False), ("shoc_tr_f32.cu", True)]
GPU_HDR = ["shoc_tr_kernels.cuh", "shoc_tr_stage.cuh", "shoc_tr_tile.cuh", "shoc_tr_tile64.cuh",
           "shoc_tr_fused.cuh", "shoc_tr_launch.h"]

NVCC_ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.sep not in cand or os.path.exists(cand)):
            return cand
    return "nvcc"


def _stale(out, srcs):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(s) > t for s in srcs if os.path.exists(s))


def _run(cmd):
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout)
        raise RuntimeError("build failed: %s" % " ".join(cmd))
    return r.stdout


def grid_lib(force=False):
    os.makedirs(LIBDIR, exist_ok=True)
    out = os.path.join(LIBDIR, "libshoc_grid.so")
    srcs = [os.path.join(CSRC, s) for s in GRID_SRC]
    deps = srcs + [os.path.join(CSRC, "shoc_grid.h"), os.path.join(INCLUDE, "shoc_tr.h")]
    if force or _stale(out, deps):
        _run(["gcc", "-O2", "-fPIC", "-shared", "-std=gnu99", "-fopenmp", "-I", INCLUDE, "-I", CSRC,
              "-o", out] + srcs)
    return out


def gpu_lib(force=False, verbose=False):
    os.makedirs(LIBDIR, exist_ok=True)
    out = os.path.join(LIBDIR, "libshoc_tr_gpu.so")
    srcs = [os.path.join(CSRC, s) for s, _ in GPU_SRC]
    deps = srcs + [os.path.join(CSRC, h) for h in GPU_HDR] + [
        os.path.join(INCLUDE, "shoc_tr.h"), os.path.join(INCLUDE, "shoc_tr_gpu.h")]
    if force or _stale(out, deps):
        objs = []
        log = ""
        for (name, fmad), src in zip(GPU_SRC, srcs):
            obj = os.path.join(LIBDIR, os.path.splitext(name)[0] + ".o")
            cmd = [_nvcc()] + NVCC_ARCH + [
                "-O3", "-lineinfo", "-std=c++17", "--fmad=%s" % ("true" if fmad else "false"),
                "-Xcompiler", "-fPIC", "-I", INCLUDE, "-I", CSRC, "-c", "-o", obj, src]
            if verbose:
                cmd.insert(1, "-Xptxas=-v")
            log += _run(cmd)
            objs.append(obj)
        log += _run([_nvcc()] + NVCC_ARCH + ["-shared", "-o", out] + objs)
        for o in objs:
            os.remove(o)
        if verbose:
            sys.stdout.write(log)
    return out


def build_all(force=False):
    return [grid_lib(force), gpu_lib(force)]


if __name__ == "__main__":
    for p in build_all(force="--force" in sys.argv):
        print(p)
