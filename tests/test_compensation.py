"""The 16-bit compensation of SHOC_TR_FP32_COMP, restated in numpy.

The device encodes an FP64 value v as v32 = (float)v (round to nearest) and
its compensation q: the residual v - v32 converted to FP32 toward zero, then
cut to its upper 16 bits (a bfloat16, again toward zero).  Decoding is
v32 + bf16(q).  These tests check the two properties the design relies on,
on the scheme itself (the device code is checked by the drop-in tests on a
GPU):

* accuracy: v32 + decoded is within 2^-31 of |v| relative (8 significant
  bits of a residual that is at most half an FP32 ulp);
* the trip through FP64 is exact: (float)(v32 + decoded) == v32 and encoding
  v32 + decoded again gives the same q.  This is what makes the drop-in step
  on FP64 host arrays equal the device-resident one bit for bit.
"""
import numpy as np


def f32_rz(x):
    """FP64 -> FP32 toward zero."""
    f = x.astype(np.float32)
    over = np.abs(f.astype(np.float64)) > np.abs(x)
    f[over] = np.nextafter(f[over], np.float32(0))
    return f


def encode(v):
    v32 = v.astype(np.float32)
    with np.errstate(invalid="ignore", over="ignore"):
        r = f32_rz(v - v32.astype(np.float64))
    q = (r.view(np.uint32) >> 16).astype(np.uint16)
    q[~np.isfinite(r)] = 0
    return v32, q


def decode(v32, q):
    return v32.astype(np.float64) + (q.astype(np.uint32) << 16).view(np.float32).astype(np.float64)


def values(n, seed):
    rng = np.random.default_rng(seed)
    v = rng.lognormal(0.0, 6.0, n) * rng.choice([-1.0, 1.0], n)
    # values on and next to FP32 rounding boundaries: ties, powers of two
    m = rng.integers(1, 1 << 23, n // 4).astype(np.float64)
    e = rng.integers(-40, 40, n // 4).astype(np.float64)
    tie = (m + 0.5) * 2.0 ** e
    p2 = 2.0 ** e * (1.0 - rng.uniform(0.0, 2.0 ** -24, n // 4))
    near = (m + 0.5 - rng.uniform(0.0, 2.0 ** -20, n // 4)) * 2.0 ** e
    return np.concatenate([v, tie, -tie, p2, near])


def test_compensation_accuracy():
    v = values(200000, 1)
    v32, q = encode(v)
    d = decode(v32, q)
    rel = np.abs(d - v) / np.abs(v)
    assert rel.max() <= 2.0 ** -31, rel.max()
    # without it the stored value is off by up to half an FP32 ulp
    assert (np.abs(v32.astype(np.float64) - v) / np.abs(v)).max() > 2.0 ** -26


def test_trip_through_fp64_is_exact():
    v = values(200000, 2)
    v32, q = encode(v)
    d = decode(v32, q)
    v32b, qb = encode(d)
    np.testing.assert_array_equal(v32b, v32)
    np.testing.assert_array_equal(qb, q)
    np.testing.assert_array_equal(decode(v32b, qb), d)


def test_zero_and_non_finite():
    v = np.array([0.0, -0.0, np.inf, -np.inf, np.nan, 1e-45, 3.4e38])
    v32, q = encode(v)
    assert q[0] == 0 and q[1] == 0
    assert np.all(q[2:5] == 0)  # no residual for an infinite or NaN value
    d = decode(v32, q)
    assert d[0] == 0.0 and np.isinf(d[2]) and np.isnan(d[4])
