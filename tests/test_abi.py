"""The C-ABI library loads and exports every entry point include/*.h declares
(no device work: this runs on machines without a GPU)."""
import ctypes as C
import os
import re

import pytest

from ems_b200 import _build, gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared(header):
    text = open(os.path.join(ROOT, "include", header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(shoc_tr_gpu_\w+)\s*\(", text)))


@pytest.fixture(scope="module")
def L():
    path = _build.gpu_lib()
    return gpu.lib(path)


def test_every_declared_symbol_is_exported(L):
    names = declared("shoc_tr_gpu.h")
    assert len(names) >= 15
    assert set(names) == set(gpu.EXPORTS)
    for n in names:
        assert hasattr(L, n), n


def test_strerror_covers_status_codes(L):
    for code in range(10):
        s = L.shoc_tr_gpu_strerror(code).decode()
        assert s and "unknown" not in s
    assert L.shoc_tr_gpu_strerror(99).decode() == "unknown status"


def test_create_rejects_bad_arguments_without_device_work(L):
    h = C.c_void_p()
    assert L.shoc_tr_gpu_create(None, None, 1, 0, 0, C.byref(h)) == 7  # SHOC_TR_EARG
    assert not h.value
