"""The rounding argument behind the weighting kernels' weight_div, checked by
exact emulation on the CPU: numpy's FP64 reciprocal, FP64 product, floor and
f32 conversion round as the device's __drcp_rn, DMUL, floor and
__double2float_rn do, the near-midpoint residual (one exact FMA on the
device) is computed with rationals, and numpy's f32 division is the IEEE one.
Wherever the product is at least 2^-126 (1 + 2^-50) (the fast path) its f32
rounding must equal the correctly rounded quotient; below that exact
midpoints exist (shown here), and the quotient is rounded as an integer count
of 2^-149, which must match too."""
from fractions import Fraction

import numpy as np

FAST_MIN = np.float64(2.0 ** -126 * (1.0 + 2.0 ** -50))


def _fast_path(e, s):
    p = e.astype(np.float64) * (1.0 / s.astype(np.float64))
    return p, p >= FAST_MIN


def _weight_div(e, s):
    """weight_div of pf_internal.h for e >= 0 and 1 <= S <= 2^100."""
    e64, s64 = e.astype(np.float64), s.astype(np.float64)
    rs = 1.0 / s64
    p = e64 * rs
    fast = p >= FAST_MIN
    x = e64 * 2.0 ** 149
    y = x * rs
    fl = np.floor(y)
    dm = y - (fl + 0.5)
    k = np.where(dm > 0, fl + 1, fl)
    near = ~fast & (np.abs(dm) <= 2.0 ** -28)
    for i in np.flatnonzero(near):
        r = Fraction(float(x[i])) - (Fraction(float(fl[i])) + Fraction(1, 2)) * Fraction(float(s64[i]))
        odd = int(fl[i]) & 1
        k[i] = fl[i] + 1 if (r > 0 or (r == 0 and odd)) else fl[i]
    out = np.where(fast, p, k * 2.0 ** -149).astype(np.float32)
    return out, int(near.sum())


def _midpoints(rng, n):
    """Pairs whose quotient is an exact midpoint of the 2^-149 grid."""
    so = rng.integers(1, 1 << 12, n) * 2 + 1
    mm = rng.integers(0, 1 << 11, n) * 2 + 1
    t = rng.integers(0, 20, n)
    big = mm * so
    keep = big < (1 << 24)
    exact = big[keep] * np.exp2(t[keep] - 150.0)
    e = exact.astype(np.float32)
    s = (so[keep] * np.exp2(t[keep])).astype(np.float32)
    ok = e.astype(np.float64) == exact  # odd multiples of 2^-150 are not floats
    return e[ok], s[ok]


def test_fast_path_equals_ieee_division():
    rng = np.random.default_rng(3)
    for _ in range(4):
        n = 2_000_000
        e = rng.integers(0, 0x3F800001, n, dtype=np.int64).astype(np.uint32).view(np.float32)
        s = ((np.float32(1.0) + rng.random(n, dtype=np.float32))
             * np.exp2(rng.integers(0, 25, n)).astype(np.float32)).astype(np.float32)
        s = np.where(rng.random(n) < 0.1, np.round(s), s).astype(np.float32)
        s = np.maximum(s, np.float32(1.0))
        p, ok = _fast_path(e, s)
        assert ok.mean() > 0.5
        ref = (e / s).astype(np.float32)
        assert (p[ok].astype(np.float32).view(np.uint32) == ref[ok].view(np.uint32)).all()


def test_integer_significands():
    rng = np.random.default_rng(4)
    e = (rng.integers(1, 1 << 24, 2_000_000).astype(np.float32)
         * np.float32(2.0 ** -24)).astype(np.float32)
    s = np.maximum(rng.integers(1, 1 << 24, 2_000_000), 1).astype(np.float32)
    p, ok = _fast_path(e, s)
    assert ok.all()
    ref = (e / s).astype(np.float32)
    assert (p.astype(np.float32).view(np.uint32) == ref.view(np.uint32)).all()


def test_subnormal_quotients_need_the_division():
    """11000715 * 2^-149 / 13310 = 1653 * 2^-150 is an exact midpoint of the
    subnormal grid (between 826 and 827 * 2^-149): the IEEE quotient rounds to
    even (826), the product with RN(1/13310) lies just above the midpoint and
    rounds to 827 — so quotients below 2^-126 must not take the fast path."""
    e = np.array([11000715 * 2.0 ** -149], np.float32)
    s = np.array([13310.0], np.float32)
    assert float(e[0]) == 11000715 * 2.0 ** -149
    p, ok = _fast_path(e, s)
    assert not ok[0]
    assert (e / s).astype(np.float32)[0] == np.float32(826 * 2.0 ** -149)
    assert p.astype(np.float32)[0] == np.float32(827 * 2.0 ** -149)


def test_weight_div_equals_ieee_division_everywhere():
    rng = np.random.default_rng(6)
    for hi in (0x3F800001, 0x0D000000):  # all of [0, 1]; quotients mostly subnormal
        n = 1_000_000
        e = rng.integers(0, hi, n, dtype=np.int64).astype(np.uint32).view(np.float32)
        s = ((np.float32(1.0) + rng.random(n, dtype=np.float32))
             * np.exp2(rng.integers(0, 40, n)).astype(np.float32)).astype(np.float32)
        s = np.maximum(np.where(rng.random(n) < 0.2, np.round(s), s), 1).astype(np.float32)
        out, _ = _weight_div(e, s)
        ref = (e / s).astype(np.float32)
        assert (out.view(np.uint32) == ref.view(np.uint32)).all()


def test_weight_div_exact_midpoints():
    e, s = _midpoints(np.random.default_rng(7), 400_000)
    out, near = _weight_div(e, s)
    assert e.size > 100_000 and near == e.size
    ref = (e / s).astype(np.float32)
    assert (out.view(np.uint32) == ref.view(np.uint32)).all()
