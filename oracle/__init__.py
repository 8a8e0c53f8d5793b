"""CPU checkers for the tracer step (TEST INFRASTRUCTURE ONLY).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference
arm may import this package, and only as the thing results are checked
against or timed beside -- never as part of the product path.

  run_oracle(case, nsteps, ...)  the C restatement (oracle/shoc_oracle.c)
  run_ref(case, nsteps, ...)     the reference's own tracers.c, compiled
                                 unmodified (oracle/_ref, built by
                                 oracle/build.py where the reference exists)
  ref_preamble(case, detadt)     the reference's transport-mode flow preamble
                                 (vel3d.c compiled unmodified)
  preamble(case, detadt)         its restatement (oracle/flow_preamble.py)
"""
import ctypes as C
import os

import numpy as np

from ems_b200 import _abi

HERE = os.path.dirname(os.path.abspath(__file__))
_libs = {}


def _load(name):
    if name in _libs:
        return _libs[name]
    from . import build
    if name == "ref_vel":
        path = os.path.join(HERE, "_ref", "libshoc_ref_vel.so")
        if not os.path.exists(path):
            build.ref_vel_lib()
        if not os.path.exists(path):
            return None
        L = C.CDLL(path)
        L.ref_preamble.argtypes = [C.POINTER(_abi.Geom), C.POINTER(_abi.State),
                                   C.POINTER(_abi.Opts)] + [_abi.DP] * 6
        L.ref_preamble.restype = C.c_int
        _libs[name] = L
        return L
    if name == "oracle":
        path = build.oracle_lib()
        L = C.CDLL(path)
        L.oracle_run.argtypes = [C.POINTER(_abi.Geom), C.POINTER(_abi.State),
                                 C.POINTER(_abi.Opts), C.c_int, C.POINTER(_abi.Diag)]
        L.oracle_run.restype = C.c_int
        L.oracle_set_owned.argtypes = [_abi.IP]
        L.oracle_set_owned.restype = None
        L.oracle_set_substep_min.argtypes = [C.c_double]
        L.oracle_set_substep_min.restype = None
    else:
        fname = "libshoc_ref_omp.so" if name == "ref_omp" else "libshoc_ref.so"
        path = os.path.join(HERE, "_ref", fname)
        if not os.path.exists(path):
            build.ref_libs()
        if not os.path.exists(path):
            return None
        L = C.CDLL(path)
        L.ref_run.argtypes = [C.POINTER(_abi.Geom), C.POINTER(_abi.State),
                              C.POINTER(_abi.Opts), C.c_int, C.c_int, C.POINTER(_abi.Diag)]
        L.ref_run.restype = C.c_int
        L.ref_last_message.restype = C.c_char_p
        L.ref_last_loop_seconds.restype = C.c_double
        G, S, O, D = C.POINTER(_abi.Geom), C.POINTER(_abi.State), C.POINTER(_abi.Opts), _abi.DP
        L.ref_tridiag.argtypes = [G, S, O, D, D, D, D, D, C.c_double]
        L.ref_tridiag.restype = C.c_int
        L.ref_vdiff_cols.argtypes = [G, S, O] + [D] * 10 + [C.c_double]
        L.ref_vdiff_cols.restype = C.c_int
    _libs[name] = L
    return L


def ref_available(omp=False):
    return _load("ref_omp" if omp else "ref") is not None


def _call(fn, case, nsteps, tr, sur, nsur, *extra):
    keep = []
    if tr is None:
        tr, sur, nsur = case.copy_state()
    st = case.make_state(tr, sur, nsur, keep)
    op = case.make_opts(keep)
    d = _abi.Diag()
    rc = fn(C.byref(case.win.geom), C.byref(st), C.byref(op), int(nsteps), *extra, C.byref(d))
    return rc, tr, sur, nsur, d


def run_oracle(case, nsteps, tr=None, sur=None, nsur=None):
    """nsteps of the restatement; returns (status, tr, sur_t, nsur_t, diag)."""
    return _call(_load("oracle").oracle_run, case, nsteps, tr, sur, nsur)


def run_ref(case, nsteps, tr=None, sur=None, nsur=None, nthreads=1):
    """nsteps of the reference build; nthreads > 1 uses its OpenMP loop."""
    L = _load("ref_omp" if nthreads > 1 else "ref")
    if L is None:
        raise FileNotFoundError("reference build oracle/_ref not available")
    return _call(L.ref_run, case, nsteps, tr, sur, nsur, C.c_int(int(nthreads)))


def ref_loop_seconds(nthreads=1):
    """Wall time of the step loop of the last run_ref (its window set-up,
    the copy of the caller's arrays into SHOC's structs, excluded)."""
    L = _load("ref_omp" if nthreads > 1 else "ref")
    return float(L.ref_last_loop_seconds())


def max_rel_err(a, b, cells, floor=1e-300):
    """max over cells of |a-b| / max(|b|, floor), per tracer row."""
    a = np.asarray(a)[..., cells]
    b = np.asarray(b)[..., cells]
    return (np.abs(a - b) / np.maximum(np.abs(b), floor)).max(axis=-1)


def _ref_call(fn_name, case, sur, nsur, *args):
    L = _load("ref")
    if L is None:
        raise FileNotFoundError("reference build oracle/_ref not available")
    keep = []
    tr = case.tr.copy()
    st = case.make_state(tr, sur, nsur, keep)
    op = case.make_opts(keep)
    return getattr(L, fn_name)(C.byref(case.win.geom), C.byref(st), C.byref(op), *args)


def ref_tridiag(case, Cd, Cm1, Cp1, rhs, var, minvar, sur=None, nsur=None):
    """The reference's closure tridiagonal (closure/MY2-5.c:499) on every
    water column (surface cells nsur_t); var updated in place; status."""
    sur = case.sur_t.copy() if sur is None else sur
    nsur = case.nsur_t.copy() if nsur is None else nsur
    P = _abi.dptr
    return _ref_call("ref_tridiag", case, sur, nsur, P(Cd), P(Cm1), P(Cp1), P(rhs), P(var),
                     C.c_double(minvar))


def ref_vdiff_cols(case, var, dzcell, Cd, Cm1, Cp1, fb, ft, scale, dt, Splus=None,
                   Sminus=None, sur=None, nsur=None):
    """The reference's implicit_vdiff_at_cc (tracers.c:7407) on every water
    column; var updated in place; status."""
    sur = case.sur_t.copy() if sur is None else sur
    nsur = case.nsur_t.copy() if nsur is None else nsur
    P = _abi.dptr
    return _ref_call("ref_vdiff_cols", case, sur, nsur, P(var), P(dzcell), P(Cd), P(Cm1),
                     P(Cp1), P(fb), P(ft), P(Splus), P(Sminus), P(scale), C.c_double(dt))


def ref_preamble(case, detadt, sur=None, nsur=None):
    """The reference's set_dz_at_u1 / _u2, set_flux_3d (VEL3D), set_dz and
    vel_w_update on case's window, velocities and surface (transport.c:
    436-462), wtop = detadt [sgsizS]; returns dict of dzu1, dzu2, u1flux3d,
    u2flux3d, w (each [sgsiz])."""
    L = _load("ref_vel")
    if L is None:
        raise FileNotFoundError("reference build oracle/_ref/libshoc_ref_vel.so not available")
    # the reference's set_dz moves the surface vectors it is given: copies
    sur = np.array(case.sur_t if sur is None else sur, np.int32)
    nsur = np.array(case.nsur_t if nsur is None else nsur, np.int32)
    keep = []
    tr = case.tr.copy()
    st = case.make_state(tr, sur, nsur, keep)
    op = case.make_opts(keep)
    S = case.win.sgsiz
    out = {k: np.zeros(S) for k in ("dzu1", "dzu2", "u1flux3d", "u2flux3d", "w")}
    det = np.ascontiguousarray(detadt, np.float64)
    P = _abi.dptr
    rc = L.ref_preamble(C.byref(case.win.geom), C.byref(st), C.byref(op), P(det),
                        P(out["dzu1"]), P(out["dzu2"]), P(out["u1flux3d"]), P(out["u2flux3d"]),
                        P(out["w"]))
    if rc:
        raise RuntimeError("ref_preamble: status %d" % rc)
    return out


def preamble(case, detadt, sur=None, nsur=None):
    """The restatement of the same preamble (oracle/flow_preamble.py)."""
    from . import flow_preamble
    return flow_preamble.preamble(case, detadt, sur, nsur)


def set_strip(owned2d=None, dmin=0.0):
    """The oracle steps a strip of a decomposed basin: only owned2d's columns
    count in its sub-step minimum, and dmin (> 0) is the basin-wide minimum
    it uses.  set_strip() goes back to whole windows."""
    L = _load("oracle")
    global _owned_keep
    _owned_keep = None if owned2d is None else np.ascontiguousarray(owned2d, np.int32)
    L.oracle_set_owned(_abi.iptr(_owned_keep))
    L.oracle_set_substep_min(float(dmin))


_owned_keep = None
