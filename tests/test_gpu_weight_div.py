"""The weighting kernels form the normalised weight expf(ll - M) / S as the
FP64 product e * RN(1/S) rounded once to f32 (weight_div), round quotients
below 2^-126 as an integer count of 2^-149 (an exact FMA residual near
midpoints), and keep the IEEE f32 division for non-finite operands and
S < 1.  Bar: bit-identical to the IEEE division on the device and to
numpy's f32 division, over random pairs spanning every binade of e (subnormals
included) and S in [1, 2^24], integer-significand pairs, and special values."""

import numpy as np
import pytest

import cuda_pf_localization_b200 as pkg
from tests.test_weight_div_cpu import _midpoints

pytestmark = pytest.mark.gpu


def _pairs(rng, n, hi=0x3F800001):
    bits = rng.integers(0, hi, n, dtype=np.int64).astype(np.uint32)
    e = bits.view(np.float32)
    s = ((np.float32(1.0) + rng.random(n, dtype=np.float32))
         * np.exp2(rng.integers(0, 25, n)).astype(np.float32)).astype(np.float32)
    s = np.where(rng.random(n) < 0.1, np.round(s), s).astype(np.float32)
    return e, np.maximum(s, np.float32(1.0))


def _specials():
    tiny = np.float32(2.0 ** -149)
    vals = np.array([0.0, tiny, 3 * tiny, np.float32(2.0 ** -126), np.float32(2.0 ** -125),
                     0.5, 1.0, 2.0, np.inf, np.nan, 1e30, np.float32(3.4e38)], np.float32)
    svals = np.array([1.0, 2.0, 3.0, 6.0, 7.0, 1e-30, tiny, 0.0, np.inf, np.nan, 16777215.0,
                      -2.0], np.float32)
    e, s = np.meshgrid(vals, svals)
    # exact midpoints of the subnormal grid, where a single rounding of the
    # FP64 product would differ from the IEEE quotient
    mid_e = np.array([11000715 * 2.0 ** -149, 39021760 * 2.0 ** -149], np.float32)
    mid_s = np.array([13310.0, 79232.0], np.float32)
    return (np.r_[e.ravel(), mid_e].astype(np.float32),
            np.r_[s.ravel(), mid_s].astype(np.float32))


def _run(kernels, h, e, s):
    fast = np.zeros_like(e)
    ieee = np.zeros_like(e)
    assert kernels.pfc_weight_div_check(h, pkg.fptr(e), pkg.fptr(s), e.size, pkg.fptr(fast),
                                        pkg.fptr(ieee)) == 0
    return fast, ieee


def _same_bits(a, b):
    both_nan = np.isnan(a) & np.isnan(b)
    return both_nan | (a.view(np.uint32) == b.view(np.uint32))


def test_weight_div_matches_ieee_division(kernels):
    h = kernels.pfc_create(64)
    try:
        rng = np.random.default_rng(11)
        cases = [_pairs(rng, 4_000_000) for _ in range(4)]
        ei = (rng.integers(1, 1 << 24, 2_000_000).astype(np.float32)
              * np.float32(2.0 ** -24)).astype(np.float32)
        si = np.maximum(rng.integers(1, 1 << 24, 2_000_000), 1).astype(np.float32)
        # quotients mostly below 2^-126, and exact midpoints of the 2^-149 grid
        cases += [(ei, si), _specials(), _pairs(rng, 4_000_000, 0x0D000000),
                  _midpoints(rng, 2_000_000)]
        for e, s in cases:
            fast, ieee = _run(kernels, h, e, s)
            with np.errstate(all="ignore"):
                ref = (e / s).astype(np.float32)
            assert _same_bits(fast, ieee).all()
            assert _same_bits(ieee, ref).all()
    finally:
        kernels.pfc_destroy(h)
