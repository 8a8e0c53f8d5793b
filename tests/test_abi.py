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


def test_precision_constants_match_header():
    """The binding's precision codes are the header's SHOC_TR_FP* values."""
    import re
    from ems_b200 import gpu
    with open(os.path.join(ROOT, "include", "shoc_tr_gpu.h")) as f:
        txt = f.read()
    want = {m.group(1): int(m.group(2))
            for m in re.finditer(r"#define SHOC_TR_(FP\w+)\s+(\d+)", txt)}
    assert want == {"FP64": gpu.FP64, "FP32_MIXED": gpu.FP32_MIXED, "FP32_COMP": gpu.FP32_COMP}
