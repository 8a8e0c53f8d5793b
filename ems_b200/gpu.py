"""Python binding of the C-ABI in include/shoc_tr_gpu.h (libshoc_tr_gpu.so).

This is a thin ctypes layer: every call goes straight to the sm_100a library.
There is no CPU path -- if the library or a CUDA device is missing, the
constructor raises.
"""
import ctypes as C
import os

import numpy as np

from . import _abi

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libshoc_tr_gpu.so")

FP64 = 0
FP32_MIXED = 1
FP32_COMP = 2

# every entry point include/shoc_tr_gpu.h declares
EXPORTS = (
    "shoc_tr_gpu_create", "shoc_tr_gpu_destroy", "shoc_tr_gpu_step",
    "shoc_tr_gpu_upload_tracers", "shoc_tr_gpu_download_tracers", "shoc_tr_gpu_set_flow",
    "shoc_tr_gpu_get_surface", "shoc_tr_gpu_run", "shoc_tr_gpu_sync", "shoc_tr_gpu_mass",
    "shoc_tr_gpu_mass_noalloc", "shoc_tr_gpu_compare", "shoc_tr_gpu_state_size",
    "shoc_tr_gpu_save_state", "shoc_tr_gpu_load_state", "shoc_tr_gpu_tridiag",
    "shoc_tr_gpu_vdiff_cols", "shoc_tr_gpu_halo_plan", "shoc_tr_gpu_halo_pack",
    "shoc_tr_gpu_halo_unpack", "shoc_tr_gpu_mass_region", "shoc_tr_gpu_set_owned",
    "shoc_tr_gpu_substep_min", "shoc_tr_gpu_set_substep_min", "shoc_tr_gpu_host_register", "shoc_tr_gpu_host_unregister",
    "shoc_tr_gpu_stream", "shoc_tr_gpu_set_tiling", "shoc_tr_gpu_autotune", "shoc_tr_gpu_profile",
    "shoc_tr_gpu_kernel_time", "shoc_tr_gpu_kernel_time_part", "shoc_tr_gpu_launch_count",
    "shoc_tr_gpu_strerror", "shoc_tr_gpu_set_preamble", "shoc_tr_gpu_set_detadt",
    "shoc_tr_gpu_get_flow", "shoc_tr_gpu_get_tuning", "shoc_tr_gpu_set_tuning",
    "shoc_tr_gpu_autotune_ex",
)


class Tuning(C.Structure):
    """shoc_tr_tuning: the transport kernels' launch configuration."""
    _fields_ = [("fused", C.c_int), ("tracers_per_block", C.c_int), ("tile_x", C.c_int),
                ("phase_b_warps", C.c_int), ("prefetch", C.c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}

_lib = None


def lib(path=None):
    """Load the library (built in-tree by __graft_entry__.build())."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise FileNotFoundError(
            "libshoc_tr_gpu.so not built (%s); run __graft_entry__.build()" % p)
    L = C.CDLL(p)
    H = C.c_void_p
    L.shoc_tr_gpu_create.argtypes = [C.POINTER(_abi.Geom), C.POINTER(_abi.Opts), C.c_int,
                                     C.c_int, C.c_int, C.POINTER(H)]
    L.shoc_tr_gpu_destroy.argtypes = [H]
    L.shoc_tr_gpu_destroy.restype = None
    L.shoc_tr_gpu_step.argtypes = [H, C.POINTER(_abi.State), C.POINTER(_abi.Diag)]
    L.shoc_tr_gpu_upload_tracers.argtypes = [H, C.POINTER(_abi.DP)]
    L.shoc_tr_gpu_download_tracers.argtypes = [H, C.POINTER(_abi.DP)]
    L.shoc_tr_gpu_set_flow.argtypes = [H, C.POINTER(_abi.State)]
    L.shoc_tr_gpu_get_surface.argtypes = [H, _abi.IP, _abi.IP]
    L.shoc_tr_gpu_run.argtypes = [H, C.c_int]
    L.shoc_tr_gpu_sync.argtypes = [H, C.POINTER(_abi.Diag)]
    L.shoc_tr_gpu_mass.argtypes = [H, _abi.DP]
    L.shoc_tr_gpu_mass_noalloc.argtypes = [H, _abi.DP]
    L.shoc_tr_gpu_compare.argtypes = [H, H, _abi.IP, C.c_int] + [_abi.DP] * 4
    L.shoc_tr_gpu_state_size.argtypes = [H, C.POINTER(C.c_size_t)]
    L.shoc_tr_gpu_halo_plan.argtypes = [H, C.c_int, _abi.IP, C.c_int, _abi.IP]
    L.shoc_tr_gpu_halo_pack.argtypes = [H, C.c_void_p]
    L.shoc_tr_gpu_halo_unpack.argtypes = [H, C.c_void_p]
    L.shoc_tr_gpu_mass_region.argtypes = [H, _abi.IP, C.c_int, _abi.DP]
    L.shoc_tr_gpu_set_owned.argtypes = [H, _abi.IP]
    L.shoc_tr_gpu_substep_min.argtypes = [H, _abi.DP]
    L.shoc_tr_gpu_set_substep_min.argtypes = [H, C.c_double]
    L.shoc_tr_gpu_tridiag.argtypes = [H] + [_abi.DP] * 5 + [C.c_double]
    L.shoc_tr_gpu_vdiff_cols.argtypes = [H] + [_abi.DP] * 10 + [C.c_double]
    L.shoc_tr_gpu_save_state.argtypes = [H, C.c_void_p, C.c_size_t]
    L.shoc_tr_gpu_load_state.argtypes = [H, C.c_void_p, C.c_size_t]
    L.shoc_tr_gpu_host_register.argtypes = [C.c_void_p, C.c_size_t]
    L.shoc_tr_gpu_host_unregister.argtypes = [C.c_void_p]
    L.shoc_tr_gpu_stream.argtypes = [H]
    L.shoc_tr_gpu_stream.restype = C.c_void_p
    L.shoc_tr_gpu_set_tiling.argtypes = [H, C.c_int, C.c_int]
    L.shoc_tr_gpu_autotune.argtypes = [H, C.c_int, C.POINTER(C.c_int)]
    L.shoc_tr_gpu_profile.argtypes = [H, C.c_int]
    L.shoc_tr_gpu_kernel_time.argtypes = [H, C.POINTER(C.c_double), C.POINTER(C.c_int)]
    L.shoc_tr_gpu_kernel_time_part.argtypes = [H, C.c_int, C.POINTER(C.c_double),
                                               C.POINTER(C.c_int)]
    L.shoc_tr_gpu_launch_count.argtypes = [H]
    L.shoc_tr_gpu_launch_count.restype = C.c_longlong
    L.shoc_tr_gpu_get_tuning.argtypes = [H, C.POINTER(Tuning)]
    L.shoc_tr_gpu_set_tuning.argtypes = [H, C.POINTER(Tuning)]
    L.shoc_tr_gpu_autotune_ex.argtypes = [H, C.c_int, C.c_int, C.POINTER(Tuning),
                                          C.POINTER(C.c_int)]
    L.shoc_tr_gpu_set_preamble.argtypes = [H, C.c_int]
    L.shoc_tr_gpu_set_detadt.argtypes = [H, _abi.DP]
    L.shoc_tr_gpu_get_flow.argtypes = [H] + [_abi.DP] * 5
    L.shoc_tr_gpu_strerror.argtypes = [C.c_int]
    L.shoc_tr_gpu_strerror.restype = C.c_char_p
    for name in EXPORTS:
        if name not in ("shoc_tr_gpu_destroy", "shoc_tr_gpu_stream", "shoc_tr_gpu_launch_count",
                        "shoc_tr_gpu_strerror"):
            getattr(L, name).restype = C.c_int
    if path is None:
        _lib = L
    return L


def _check(where, rc):
    if rc != 0:
        raise _abi.StatusError(where, rc)


class HostPinned:
    """Page-locks numpy arrays the drop-in step copies every step
    (shoc_tr_gpu_host_register) for as long as the context is open."""

    def __init__(self, arrays):
        self.L = lib()
        self.arrays = []
        for a in arrays:
            assert a.flags.c_contiguous
            _check("host_register", self.L.shoc_tr_gpu_host_register(a.ctypes.data, a.nbytes))
            self.arrays.append(a)

    def close(self):
        while self.arrays:
            a = self.arrays.pop()
            _check("host_unregister", self.L.shoc_tr_gpu_host_unregister(a.ctypes.data))

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


class TracerStep:
    """One SHOC window's tracer step on a B200 (device-resident tracers).

    Mirrors the reference calls it replaces: ``step()`` is one
    set_lateral_BC_tr + set_dz + advect_diffuse + vert_diffuse_3d on host
    arrays (the drop-in), ``run()`` the same on tracers kept in HBM.
    Failures raise _abi.StatusError with the reference's error meaning
    (status 1: sub-step limit, tracers.c:664; status 2: zero pivot,
    tracers.c:4190).
    """

    def __init__(self, case, precision=FP64, device=0):
        self.case = case
        self._keep = []
        self.L = lib()
        opts = case.make_opts(self._keep)
        h = C.c_void_p()
        _check("shoc_tr_gpu_create",
               self.L.shoc_tr_gpu_create(C.byref(case.win.geom), C.byref(opts), case.ntr,
                                         precision, device, C.byref(h)))
        self.h = h
        self.precision = precision

    def close(self):
        if getattr(self, "h", None):
            self.L.shoc_tr_gpu_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- drop-in (host arrays) ------------------------------------------
    def step(self, tr, sur_t, nsur_t):
        """One step on host arrays, updated in place; returns the diag."""
        keep = []
        st = self.case.make_state(tr, sur_t, nsur_t, keep)
        d = _abi.Diag()
        _check("shoc_tr_gpu_step", self.L.shoc_tr_gpu_step(self.h, C.byref(st), C.byref(d)))
        return d

    # -- device-resident -------------------------------------------------
    def _rows(self, tr):
        rows = (_abi.DP * self.case.ntr)(*[tr[n].ctypes.data_as(_abi.DP)
                                           for n in range(self.case.ntr)])
        return rows

    def upload(self, tr):
        assert tr.dtype == np.float64 and tr.flags.c_contiguous
        _check("upload", self.L.shoc_tr_gpu_upload_tracers(self.h, self._rows(tr)))

    def download(self, out=None):
        if out is None:
            out = np.empty((self.case.ntr, self.case.win.sgsiz))
        _check("download", self.L.shoc_tr_gpu_download_tracers(self.h, self._rows(out)))
        return out

    def set_flow(self, sur_t=None, nsur_t=None):
        keep = []
        c = self.case
        tr_dummy = np.zeros((c.ntr, 1))
        st = _abi.State(c.ntr, C.POINTER(_abi.DP)(), _abi.iptr(sur_t), _abi.iptr(nsur_t),
                        _abi.dptr(c.u1), _abi.dptr(c.u2), _abi.dptr(c.w), _abi.dptr(c.u1flux3d),
                        _abi.dptr(c.u2flux3d), _abi.dptr(c.Kz), _abi.dptr(c.dzu1),
                        _abi.dptr(c.dzu2), _abi.dptr(c.u1kh), _abi.dptr(c.u2kh),
                        _abi.dptr(c.eta), _abi.dptr(c.oldeta), c.dt)
        keep.append(tr_dummy)
        _check("set_flow", self.L.shoc_tr_gpu_set_flow(self.h, C.byref(st)))

    def run(self, nsteps):
        _check("run", self.L.shoc_tr_gpu_run(self.h, int(nsteps)))

    def set_preamble(self, on=True, detadt=None):
        """Transport-mode flow preamble on the device (shoc_tr_gpu_set_preamble),
        with the surface velocity detadt [sgsizS] (default 0)."""
        _check("set_preamble", self.L.shoc_tr_gpu_set_preamble(self.h, 1 if on else 0))
        if on:
            d = np.zeros(self.case.win.sgsizS) if detadt is None else detadt
            d = np.ascontiguousarray(d, np.float64)
            _check("set_detadt", self.L.shoc_tr_gpu_set_detadt(self.h, _abi.dptr(d)))

    def get_flow(self):
        """dict of the device's u1flux3d, u2flux3d, w, dzu1, dzu2 [sgsiz]
        (dzu1 / dzu2 only where the handle holds them)."""
        S = self.case.win.sgsiz
        out = {k: np.zeros(S) for k in ("u1flux3d", "u2flux3d", "w")}
        _check("get_flow", self.L.shoc_tr_gpu_get_flow(
            self.h, _abi.dptr(out["u1flux3d"]), _abi.dptr(out["u2flux3d"]), _abi.dptr(out["w"]),
            None, None))
        d1, d2 = np.zeros(S), np.zeros(S)
        if self.L.shoc_tr_gpu_get_flow(self.h, None, None, None, _abi.dptr(d1),
                                       _abi.dptr(d2)) == 0:
            out["dzu1"], out["dzu2"] = d1, d2
        return out

    def sync(self):
        d = _abi.Diag()
        _check("sync", self.L.shoc_tr_gpu_sync(self.h, C.byref(d)))
        return d

    def surface(self):
        g = self.case.win.geom
        sur = np.zeros(g.b2_t + 1, np.int32)
        nsur = np.zeros(g.a2_t + 1, np.int32)
        _check("get_surface", self.L.shoc_tr_gpu_get_surface(self.h, _abi.iptr(sur),
                                                             _abi.iptr(nsur)))
        return sur, nsur

    def mass(self):
        m = np.zeros(self.case.ntr)
        _check("mass", self.L.shoc_tr_gpu_mass(self.h, _abi.dptr(m)))
        return m

    def mass_noalloc(self):
        """mass() through the entry point that allocates no device memory."""
        m = np.zeros(self.case.ntr)
        _check("mass_noalloc", self.L.shoc_tr_gpu_mass_noalloc(self.h, _abi.dptr(m)))
        return m

    def compare(self, ref, region=None, nregion=1):
        """Differences to another handle of the same window (on the device):
        dict of per-(region, tracer) arrays max_abs, max_ref, sumsq_diff,
        sumsq_ref, and the derived max_rel = max_abs / max_ref and rms_rel =
        sqrt(sumsq_diff / sumsq_ref).  region: int32 [sgsizS] 2D cell ->
        region id (None: the whole window)."""
        if region is not None:
            region = np.ascontiguousarray(region, np.int32)
        shape = (nregion, self.case.ntr)
        out = [np.zeros(shape) for _ in range(4)]
        _check("compare", self.L.shoc_tr_gpu_compare(self.h, ref.h, _abi.iptr(region), nregion,
                                                     *[_abi.dptr(o) for o in out]))
        d = dict(zip(("max_abs", "max_ref", "sumsq_diff", "sumsq_ref"), out))
        with np.errstate(divide="ignore", invalid="ignore"):
            d["max_rel"] = np.where(d["max_ref"] > 0, d["max_abs"] / d["max_ref"], np.nan)
            d["rms_rel"] = np.where(d["sumsq_ref"] > 0, np.sqrt(d["sumsq_diff"] / d["sumsq_ref"]),
                                    np.nan)
        return d

    def tridiag(self, Cd, Cm1, Cp1, rhs, var, minvar):
        """shoc_tr_gpu_tridiag on host arrays [sgsiz]; var updated in place."""
        _check("tridiag", self.L.shoc_tr_gpu_tridiag(
            self.h, _abi.dptr(Cd), _abi.dptr(Cm1), _abi.dptr(Cp1), _abi.dptr(rhs),
            _abi.dptr(var), float(minvar)))

    def vdiff_cols(self, var, dzcell, Cd, Cm1, Cp1, fb, ft, scale, dt, Splus=None, Sminus=None):
        """shoc_tr_gpu_vdiff_cols on host arrays; var updated in place."""
        _check("vdiff_cols", self.L.shoc_tr_gpu_vdiff_cols(
            self.h, _abi.dptr(var), _abi.dptr(dzcell), _abi.dptr(Cd), _abi.dptr(Cm1),
            _abi.dptr(Cp1), _abi.dptr(fb), _abi.dptr(ft), _abi.dptr(Splus), _abi.dptr(Sminus),
            _abi.dptr(scale), float(dt)))

    def halo_plan(self, send_cells, recv_cells):
        s = np.ascontiguousarray(send_cells, np.int32)
        r = np.ascontiguousarray(recv_cells, np.int32)
        _check("halo_plan", self.L.shoc_tr_gpu_halo_plan(self.h, len(s), _abi.iptr(s), len(r),
                                                         _abi.iptr(r)))

    def halo_pack(self, dev_ptr):
        """Send-cell values of every tracer into device memory at dev_ptr."""
        _check("halo_pack", self.L.shoc_tr_gpu_halo_pack(self.h, C.c_void_p(dev_ptr)))

    def halo_unpack(self, dev_ptr):
        _check("halo_unpack", self.L.shoc_tr_gpu_halo_unpack(self.h, C.c_void_p(dev_ptr)))

    def mass_region(self, region, reg):
        m = np.zeros(self.case.ntr)
        region = np.ascontiguousarray(region, np.int32)
        _check("mass_region", self.L.shoc_tr_gpu_mass_region(self.h, _abi.iptr(region), int(reg),
                                                             _abi.dptr(m)))
        return m

    def set_owned(self, owned2d):
        o = None if owned2d is None else np.ascontiguousarray(owned2d, np.int32)
        _check("set_owned", self.L.shoc_tr_gpu_set_owned(self.h, _abi.iptr(o)))

    def substep_min(self):
        d = np.zeros(1)
        _check("substep_min", self.L.shoc_tr_gpu_substep_min(self.h, _abi.dptr(d)))
        return float(d[0])

    def set_substep_min(self, dmin):
        _check("set_substep_min", self.L.shoc_tr_gpu_set_substep_min(self.h, float(dmin)))

    def save_state(self):
        """The resident state as bytes (shoc_tr_gpu_save_state)."""
        n = C.c_size_t()
        _check("state_size", self.L.shoc_tr_gpu_state_size(self.h, C.byref(n)))
        buf = np.empty(n.value, np.uint8)
        _check("save_state", self.L.shoc_tr_gpu_save_state(self.h, buf.ctypes.data, n.value))
        return buf

    def load_state(self, buf):
        buf = np.ascontiguousarray(buf, np.uint8)
        _check("load_state", self.L.shoc_tr_gpu_load_state(self.h, buf.ctypes.data, buf.nbytes))

    def checkpoint(self, path, **meta):
        """Writes the resident state to `path`: a one-line JSON header (the
        window, precision, sizes and `meta`, e.g. the step count), then the
        raw image of shoc_tr_gpu_save_state."""
        import json
        img = self.save_state()
        c = self.case
        head = dict(meta, format="shoc_tr_gpu state v1", precision=self.precision,
                    ntr=c.ntr, sgsiz=c.win.sgsiz, columns=c.win.ncol, nwet=c.nwet,
                    bytes=int(img.nbytes))
        with open(path, "wb") as f:
            f.write((json.dumps(head) + "\n").encode())
            f.write(img.tobytes())
        return head

    def resume(self, path):
        """Loads a checkpoint written by checkpoint(); returns its header."""
        import json
        with open(path, "rb") as f:
            head = json.loads(f.readline().decode())
            img = np.frombuffer(f.read(), np.uint8)
        if head.get("format") != "shoc_tr_gpu state v1" or img.nbytes != head["bytes"]:
            raise ValueError("%s: not a shoc_tr_gpu checkpoint" % path)
        self.load_state(img)
        return head

    def stream(self):
        return self.L.shoc_tr_gpu_stream(self.h)

    def set_tiling(self, cols=0, tracers=0):
        _check("set_tiling", self.L.shoc_tr_gpu_set_tiling(self.h, cols, tracers))

    def autotune(self, steps=2):
        """Pick the fastest launch configuration (`steps` trial steps per
        candidate from the current state, which is put back); returns the
        tracers per block (shoc_tr_gpu_autotune, no cache)."""
        tw = C.c_int()
        _check("autotune", self.L.shoc_tr_gpu_autotune(self.h, int(steps), C.byref(tw)))
        return tw.value

    def autotune_ex(self, steps=2, use_cache=True):
        """shoc_tr_gpu_autotune_ex: (tuning dict, from_cache)."""
        t, fc = Tuning(), C.c_int()
        _check("autotune_ex", self.L.shoc_tr_gpu_autotune_ex(
            self.h, int(steps), 1 if use_cache else 0, C.byref(t), C.byref(fc)))
        return t.as_dict(), bool(fc.value)

    def get_tuning(self):
        t = Tuning()
        _check("get_tuning", self.L.shoc_tr_gpu_get_tuning(self.h, C.byref(t)))
        return t.as_dict()

    def set_tuning(self, **kw):
        """Change fields of the current tuning (fused, tracers_per_block,
        tile_x, phase_b_warps)."""
        t = Tuning()
        _check("get_tuning", self.L.shoc_tr_gpu_get_tuning(self.h, C.byref(t)))
        for k, v in kw.items():
            setattr(t, k, int(v))
        _check("set_tuning", self.L.shoc_tr_gpu_set_tuning(self.h, C.byref(t)))

    def profile(self, on=True):
        _check("profile", self.L.shoc_tr_gpu_profile(self.h, 1 if on else 0))

    def kernel_time(self, part=0):
        """(ms per step, steps) of the last sub-step's transport (part 0), the
        advection kernel (1) or the column kernel (2) since the last call."""
        ms = C.c_double()
        n = C.c_int()
        _check("kernel_time", self.L.shoc_tr_gpu_kernel_time_part(self.h, part, C.byref(ms),
                                                                   C.byref(n)))
        return ms.value, n.value

    def launches(self):
        return int(self.L.shoc_tr_gpu_launch_count(self.h))

    # convenience: the resident path from a case's initial state
    def start(self, tr=None, sur_t=None, nsur_t=None):
        c = self.case
        if tr is None:
            tr, sur_t, nsur_t = c.copy_state()
        self.upload(tr)
        self.set_flow(sur_t, nsur_t)
