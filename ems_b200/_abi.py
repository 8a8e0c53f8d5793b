"""ctypes mirror of include/shoc_tr.h (the plain-C window description).

The same structs are handed to the CUDA library, to the CPU oracle and to the
reference build, so every path sees one and the same SHOC window.
"""
import ctypes as C

import numpy as np

QUICKEST = 0x20
VANLEER = 0x80
ORIGINAL = 1
SUB_STEP = 2
SUB_STEP_NOSURF = 4
SUB_STEP_TRACER = 16

STATUS = {
    0: "ok",
    1: "maximum number of tracer sub-steps exceeded",
    2: "zero pivot in the implicit vertical diffusion solve",
    3: "NaN in a tracer after the step",
    4: "geometry fails the layout checks",
    5: "unsupported option",
    6: "CUDA runtime error",
    7: "bad argument",
    8: "allocation failed",
    9: "problem larger than the fixed scratch area",
}

IP = C.POINTER(C.c_int)
DP = C.POINTER(C.c_double)


class Geom(C.Structure):
    _fields_ = [
        ("nz", C.c_int), ("sgsiz", C.c_int), ("sgsizS", C.c_int),
        ("n3_t", C.c_int), ("a3_t", C.c_int), ("b3_t", C.c_int), ("v3_t", C.c_int),
        ("w3_t", IP),
        ("n2_t", C.c_int), ("a2_t", C.c_int), ("b2_t", C.c_int), ("v2_t", C.c_int),
        ("w2_t", IP), ("bot_t", IP),
        ("v3_e1", C.c_int), ("v3_e2", C.c_int), ("w3_e1", IP), ("w3_e2", IP),
        ("xp1", IP), ("xm1", IP), ("yp1", IP), ("ym1", IP), ("zp1", IP), ("zm1", IP),
        ("m2d", IP), ("s2i", IP), ("s2j", IP), ("s2k", IP),
        ("nbpt", C.c_int), ("bpt", IP), ("bin", IP),
        ("h1au1", DP), ("h2au2", DP), ("h1au2", DP), ("h2au1", DP),
        ("h1acell", DP), ("h2acell", DP), ("cellarea", DP), ("botz", DP),
        ("gridz", DP),
    ]


class State(C.Structure):
    _fields_ = [
        ("ntr", C.c_int), ("tr_wc", C.POINTER(DP)),
        ("sur_t", IP), ("nsur_t", IP),
        ("u1", DP), ("u2", DP), ("w", DP), ("u1flux3d", DP), ("u2flux3d", DP),
        ("Kz", DP), ("dzu1", DP), ("dzu2", DP), ("u1kh", DP), ("u2kh", DP),
        ("eta", DP), ("oldeta", DP), ("dt", C.c_double),
    ]


class Opts(C.Structure):
    _fields_ = [
        ("trasc", C.c_int), ("ultimate", C.c_int), ("stab", C.c_int),
        ("hmin", C.c_double),
        ("ntbdy", C.c_int), ("tbdy", IP), ("ntdif_v", C.c_int), ("tdif_v", IP),
        ("advect", IP), ("diffuse", IP), ("mintr", DP), ("maxtr", DP),
        ("ntr2d", IP),
    ]


class Diag(C.Structure):
    _fields_ = [
        ("nsub", C.c_int), ("dtm", C.c_double), ("nwarn", C.c_longlong),
        ("vc", C.c_int), ("vcs", C.c_int),
    ]


def iptr(a):
    """Pointer to the data of an int32 numpy array (or NULL for None)."""
    if a is None:
        return IP()
    assert a.dtype == np.int32 and a.flags.c_contiguous
    return a.ctypes.data_as(IP)


def dptr(a):
    """Pointer to the data of a float64 numpy array (or NULL for None)."""
    if a is None:
        return DP()
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(DP)


def status_text(code):
    return STATUS.get(int(code), "unknown status %d" % int(code))


class StatusError(RuntimeError):
    def __init__(self, where, code):
        self.code = int(code)
        super().__init__("%s: %s (status %d)" % (where, status_text(code), self.code))
