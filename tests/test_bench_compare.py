"""bench.py's host-side comparison of the mixed and plain FP64 runs, used
when a window is too large for both to sit on the device at once (the
full-size eight-basin batch): per basin and tracer, over the basin's wet
cells, the same max / RMS measures as the device comparison."""
import importlib.util
import os

import numpy as np

from ems_b200 import synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location("bench_mod", os.path.join(ROOT, "bench.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def test_host_compare_per_basin():
    bench = _bench()
    case = synth.make("batch8small")
    rng = np.random.default_rng(5)
    x64 = case.tr.copy()
    x32 = x64 * (1.0 + 1e-6 * rng.standard_normal(x64.shape))
    d = bench.host_compare(case, x32, x64, case.basins)
    c = case.win.wet_cells()
    reg = case.basin2d[case.win.m2d[c]]
    for b in range(len(case.basins)):
        cells = c[reg == b]
        for n in (0, case.basins[b][3] - 1):
            e = np.abs(x32[n, cells] - x64[n, cells]).max() / np.abs(x64[n, cells]).max()
            assert abs(d["max_rel"][b, n] - e) <= 1e-15 * e
            r = np.sqrt(((x32[n, cells] - x64[n, cells]) ** 2).sum() /
                        (x64[n, cells] ** 2).sum())
            assert abs(d["rms_rel"][b, n] - r) <= 1e-12 * r
    whole = bench.host_compare(case, x32, x64, None)
    assert whole["max_rel"].shape == (1, case.ntr)
    # every wet cell is in one basin: the window's maxima are the basins'
    np.testing.assert_array_equal(whole["max_abs"][0], d["max_abs"].max(axis=0))
    np.testing.assert_array_equal(whole["max_ref"][0], d["max_ref"].max(axis=0))
