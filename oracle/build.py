"""Builds the CPU checkers (TEST INFRASTRUCTURE ONLY).

  oracle/_lib/liboracle.so          the C restatement in oracle/shoc_oracle.c
  oracle/_lib/libshoc_grid.so       the window builder (ems_b200/csrc/shoc_grid.c)
                                    compiled for the reference arm of bench.py,
                                    so that arm loads no library of the product
  oracle/_ref/libshoc_ref.so        the reference's own model/hd/tracers/tracers.c
                                    and model/hd/closure/MY2-5.c (its tridiagonal),
                                    compiled unmodified, single thread
  oracle/_ref/libshoc_ref_omp.so    the same with -fopenmp -DHAVE_OMP (the
                                    reference's OpenMP tracer loop)
  oracle/_ref/libshoc_shim.so       include/shoc_tr_shim.h (the SHOC-side binding)
                                    compiled against the reference's headers,
                                    linked with the product library
  oracle/_ref/libshoc_ref_vel.so    the reference's transport-mode preamble:
                                    model/hd/momentum/vel3d.c with tracers.c and
                                    MY2-5.c, unmodified, driven by
                                    oracle/ref/ref_preamble.c (no-op link stubs
                                    for vel3d.c's other callees in
                                    oracle/ref/vel_stubs.c)

The reference libraries are built only where the reference source tree is
present: the directory named by the REF_ROOT environment variable or the
--ref-root argument, else a tree named `reference` beside this repository's
directory; elsewhere (a machine without the reference) the prebuilt files
are used as they are.  The reference build uses three stub headers
(oracle/ref/stub) for netcdf.h / ems_conf.h / svn_rev.h and the no-op link
stubs in oracle/ref/ref_harness.c.  Flags: -O3 -march=x86-64-v3
-ffp-contract=off, so no product or sum is fused and results are bitwise
comparable with the restatement.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
REF_ROOT = os.environ.get("REF_ROOT") or os.path.join(os.path.dirname(ROOT), "reference")
LIB = os.path.join(HERE, "_lib")
REF_OUT = os.path.join(HERE, "_ref")

CFLAGS = ["-O3", "-march=x86-64-v3", "-ffp-contract=off", "-fPIC", "-shared"]


def _stale(out, deps):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _run(cmd):
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout)
        raise RuntimeError("oracle build failed: " + " ".join(cmd))


def oracle_lib(force=False):
    os.makedirs(LIB, exist_ok=True)
    out = os.path.join(LIB, "liboracle.so")
    src = os.path.join(HERE, "shoc_oracle.c")
    deps = [src, os.path.join(HERE, "shoc_oracle.h"), os.path.join(ROOT, "include", "shoc_tr.h")]
    if force or _stale(out, deps):
        _run(["gcc", "-std=c99"] + CFLAGS + ["-I", os.path.join(ROOT, "include"), "-o", out,
                                             src, "-lm"])
    return out


def grid_lib(force=False):
    """The synthetic-window builder for the CPU checkers' own use."""
    os.makedirs(LIB, exist_ok=True)
    out = os.path.join(LIB, "libshoc_grid.so")
    csrc = os.path.join(ROOT, "ems_b200", "csrc")
    src = os.path.join(csrc, "shoc_grid.c")
    deps = [src, os.path.join(csrc, "shoc_grid.h"), os.path.join(ROOT, "include", "shoc_tr.h")]
    if force or _stale(out, deps):
        _run(["gcc", "-O2", "-fPIC", "-shared", "-std=gnu99", "-fopenmp", "-I",
              os.path.join(ROOT, "include"), "-I", csrc, "-o", out, src])
    return out


def ref_available():
    return os.path.exists(os.path.join(REF_ROOT, "model", "hd", "tracers", "tracers.c"))


def ref_libs(force=False):
    """Compile the reference tracer step (only where its sources exist)."""
    outs = [os.path.join(REF_OUT, "libshoc_ref.so"), os.path.join(REF_OUT, "libshoc_ref_omp.so")]
    if not ref_available():
        return [o for o in outs if os.path.exists(o)]
    os.makedirs(REF_OUT, exist_ok=True)
    R = REF_ROOT
    inc = ["-I", os.path.join(HERE, "ref", "stub"), "-I", os.path.join(ROOT, "include"),
           "-I", os.path.join(R, "lib", "include"), "-I", os.path.join(R, "model", "hd", "include")]
    for sub in ("sediments", "tracerstats", "waves", "ecology", "da"):
        inc += ["-I", os.path.join(R, "model", "lib", sub, "include")]
    srcs = [os.path.join(R, "model", "hd", "tracers", "tracers.c"),
            os.path.join(R, "model", "hd", "closure", "MY2-5.c"),
            os.path.join(HERE, "ref", "ref_harness.c")]
    deps = srcs + [os.path.join(ROOT, "include", "shoc_tr.h")]
    for out, extra in ((outs[0], []), (outs[1], ["-fopenmp", "-DHAVE_OMP"])):
        if force or _stale(out, deps):
            _run(["gcc", "-w"] + CFLAGS + extra + inc + ["-o", out] + srcs + ["-lm"])
    return outs


def ref_vel_lib(force=False):
    """set_dz_at_u1 / _u2, set_flux_3d, set_dz and vel_w_update compiled from
    the reference (only where its sources exist)."""
    out = os.path.join(REF_OUT, "libshoc_ref_vel.so")
    if not ref_available():
        return out if os.path.exists(out) else None
    R = REF_ROOT
    inc = ["-I", os.path.join(HERE, "ref", "stub"), "-I", os.path.join(ROOT, "include"),
           "-I", os.path.join(R, "lib", "include"), "-I", os.path.join(R, "model", "hd", "include")]
    for sub in ("sediments", "tracerstats", "waves", "ecology", "da"):
        inc += ["-I", os.path.join(R, "model", "lib", sub, "include")]
    srcs = [os.path.join(R, "model", "hd", "tracers", "tracers.c"),
            os.path.join(R, "model", "hd", "closure", "MY2-5.c"),
            os.path.join(R, "model", "hd", "momentum", "vel3d.c"),
            os.path.join(HERE, "ref", "ref_harness.c"), os.path.join(HERE, "ref", "ref_preamble.c"),
            os.path.join(HERE, "ref", "vel_stubs.c")]
    deps = srcs + [os.path.join(ROOT, "include", "shoc_tr.h")]
    if force or _stale(out, deps):
        os.makedirs(REF_OUT, exist_ok=True)
        _run(["gcc", "-w"] + CFLAGS + ["-DREF_WITH_VEL3D"] + inc + ["-o", out] + srcs + ["-lm"])
    return out


def shim_lib(force=False):
    """include/shoc_tr_shim.h compiled against the reference's headers and
    linked with the product library it binds (oracle/_ref/libshoc_shim.so);
    only where the reference sources exist."""
    out = os.path.join(REF_OUT, "libshoc_shim.so")
    if not ref_available():
        return out if os.path.exists(out) else None
    R = REF_ROOT
    gpulib = os.path.join(ROOT, "ems_b200", "_lib")
    inc = ["-I", os.path.join(HERE, "ref", "stub"), "-I", os.path.join(ROOT, "include"),
           "-I", os.path.join(R, "lib", "include"), "-I", os.path.join(R, "model", "hd", "include")]
    for sub in ("sediments", "tracerstats", "waves", "ecology", "da"):
        inc += ["-I", os.path.join(R, "model", "lib", sub, "include")]
    srcs = [os.path.join(R, "model", "hd", "tracers", "tracers.c"),
            os.path.join(R, "model", "hd", "closure", "MY2-5.c"),
            os.path.join(HERE, "ref", "ref_harness.c"), os.path.join(HERE, "ref", "shim_check.c")]
    deps = srcs + [os.path.join(ROOT, "include", n) for n in
                   ("shoc_tr.h", "shoc_tr_gpu.h", "shoc_tr_shim.h")]
    if force or _stale(out, deps):
        os.makedirs(REF_OUT, exist_ok=True)
        _run(["gcc", "-w"] + CFLAGS + inc + ["-o", out] + srcs +
             ["-L", gpulib, "-lshoc_tr_gpu", "-Wl,-rpath,$ORIGIN/../../ems_b200/_lib", "-lm"])
    return out


def build_all(force=False):
    out = [oracle_lib(force), grid_lib(force)]
    out += ref_libs(force)
    for extra in (shim_lib(force), ref_vel_lib(force)):
        if extra:
            out.append(extra)
    return out


if __name__ == "__main__":
    if "--ref-root" in sys.argv:
        REF_ROOT = sys.argv[sys.argv.index("--ref-root") + 1]
    for p in build_all(force="--force" in sys.argv):
        print(p)
