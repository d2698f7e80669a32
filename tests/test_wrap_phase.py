"""The division-free form of wrap_phase (csrc/qhk_math.cuh) against the reference formula
p - 2 pi floor((p + pi) / 2 pi) (src/common.hpp:33), in IEEE float32 on the host: numpy's float32
add, multiply and divide round to nearest like the device's __fadd_rn, __fmul_rn, __fdiv_rn, so equal
bits here are equal bits there."""

from __future__ import annotations

import numpy as np

PI = np.float32(np.pi)
TWO_PI = np.float32(2.0) * PI


def reference(p):
    p = p.astype(np.float32)
    x = p + PI
    return p - TWO_PI * np.floor(x / TWO_PI)


def comparisons(p):
    p = p.astype(np.float32)
    x = p + PI
    inside = (x > np.float32(-3.0)) & (x < np.float32(12.0))
    f = np.where(x < 0, np.float32(-1.0), np.where(x >= TWO_PI, np.float32(1.0), np.float32(0.0)))
    f = np.where(inside, f, np.floor(x / TWO_PI)).astype(np.float32)
    return p - TWO_PI * f


def neighbours(v, k=4096):
    """The k floats on either side of float32 v."""
    v = np.float32(v)
    bits = v.view(np.int32)
    steps = np.arange(-k, k + 1, dtype=np.int64)
    if v > 0:
        b = bits + steps
    elif v < 0:
        b = bits - steps
    else:
        b = np.concatenate([np.arange(0, k, dtype=np.int64), -np.arange(1, k, dtype=np.int64)])
        return np.where(b >= 0, b, (np.int64(0x80000000) - b)).astype(np.uint32).view(np.float32)
    return b.astype(np.int32).view(np.float32)


def test_same_bits_on_dense_samples():
    rng = np.random.default_rng(7)
    for scale in (np.pi, 2 * np.pi, 4 * np.pi, 50.0):
        p = rng.uniform(-scale, scale, 2_000_000).astype(np.float32)
        assert np.array_equal(reference(p).view(np.int32), comparisons(p).view(np.int32))


def test_same_bits_around_every_threshold():
    # p where x = p + pi crosses 0, 2 pi, and the ends of the comparison range (-3, 12).
    for x in (0.0, float(TWO_PI), -3.0, 12.0, float(-TWO_PI), float(2 * TWO_PI)):
        p = neighbours(np.float32(x) - PI)
        p = p[np.isfinite(p)]
        assert np.array_equal(reference(p).view(np.int32), comparisons(p).view(np.int32)), x


def test_every_float_near_the_phase_range():
    # All floats p in [-pi - 3, 2 pi] step by step around the two inner thresholds, and a stride
    # through the whole range.
    lo, hi = np.float32(-np.pi - 3.0), np.float32(2.0 * np.pi)
    p = np.linspace(lo, hi, 5_000_001, dtype=np.float32)
    assert np.array_equal(reference(p).view(np.int32), comparisons(p).view(np.int32))


def test_special_values():
    p = np.array([np.inf, -np.inf, np.nan, 0.0, -0.0, np.float32(3.4e38), -np.float32(3.4e38), 1e-45, -1e-45],
                 np.float32)
    with np.errstate(invalid="ignore", over="ignore"):
        a, b = reference(p), comparisons(p)
    assert np.array_equal(np.isnan(a), np.isnan(b))
    keep = ~np.isnan(a)
    assert np.array_equal(a[keep].view(np.int32), b[keep].view(np.int32))
