"""GPU parity of the particle-filter path against the oracle and against the
reference library built from its own source (oracle/_ref), on identical
inputs, through the C-ABI.

Tolerances (the bar of the specification):
  * log-likelihoods: identical bits to the reference kernel is the target;
    the test bound is 2e-6 relative (a few f32 ulps of the 256-term sum);
  * weights: 1e-5 relative to the reference after both are renormalised in
    FP64 (the reference's own normaliser is an f32 atomic sum);
  * the 14 + 12 FP64 sums: 1e-9 relative to the FP64 oracle on the same f32
    state and weights, 1e-5 relative to the reference;
  * ancestors: bit-exact against the oracle's fixed-point specification, and
    bit-exact against the reference's pick rule fed the reference's own cum;
  * predict / reinit: 2e-5 absolute against the oracle driven by the same
    Philox noise (f32 vs f64 arithmetic).
"""
import ctypes as C

import numpy as np
import pytest

import cuda_pf_localization_b200 as pkg
import oracle
from tests.pf_helpers import (RawPF, cloud, f32p, f64p, i32p, ours_ll, ours_set_state,
                              ours_weights, ref_ll, ref_set_state, ref_weights, rel_close,
                              scale_obs)

pytestmark = pytest.mark.gpu

N = 50_000  # not a multiple of the 256-thread block nor of the 4096 scan tile
SR = 1.0    # range sigma of the comparison fixture


@pytest.fixture(scope="module")
def weighted_pair(kernels, ref):
    """Our library and the reference on the same state after one weighting
    of the at-scale observation set."""
    lm, obs, tp, tq = scale_obs()
    yaw = 2.0 * np.arctan2(tq[3], tq[0])
    pos, quat = cloud(N, 1, centre=tp, pos_std=0.3, rot_std=0.05, yaw=yaw)
    ours = RawPF(kernels, N, seed=9)
    theirs = RawPF(ref, N, seed=9)
    ours_set_state(ours, pos, quat)
    ref_set_state(ref, theirs, pos, quat)
    ours.landmarks(lm)
    theirs.landmarks(lm)
    # sigma_r = 1 m keeps many weights non-negligible (at 0.05 m the posterior
    # of 256 observations sits on one particle and the comparison is empty)
    assert ours.weight(obs, SR, 0.02, 3.0) == 0
    assert theirs.weight(obs, SR, 0.02, 3.0) == 0
    yield dict(ours=ours, theirs=theirs, pos=pos, quat=quat, lm=lm, obs=obs)
    ours.close()
    theirs.close()


def test_loglik_matches_reference_kernel(weighted_pair, ref):
    a = ours_ll(weighted_pair["ours"])
    b = ref_ll(ref, weighted_pair["theirs"])
    exact = np.mean(a == b)
    print(f"ll bit-identical fraction {exact:.6f}")
    assert np.all(rel_close(a, b, 2e-6, 1e-6)), np.max(np.abs(a - b))


def test_loglik_matches_fp64_oracle(weighted_pair):
    d = weighted_pair
    a = ours_ll(d["ours"]).astype(np.float64)
    o = oracle.loglik(d["pos"].astype(np.float64), d["quat"].astype(np.float64),
                      d["lm"].astype(np.float32).astype(np.float64),
                      [tuple(r[:2]) + tuple(np.float32(r[2:]).astype(np.float64)) for r in d["obs"]],
                      SR, 0.02, 3.0)
    # f32 evaluation of 256 gated terms against FP64
    assert np.all(np.abs(a - o) <= 1e-5 * np.abs(o) + 5e-3), np.max(np.abs(a - o))


def test_weights_match_reference(weighted_pair, ref):
    a = ours_weights(weighted_pair["ours"]).astype(np.float64)
    b = ref_weights(ref, weighted_pair["theirs"]).astype(np.float64)
    assert abs(a.sum() - 1.0) < 1e-5
    a /= a.sum()
    b /= b.sum()
    big = b > 1e-12 * b.max()
    rel = np.abs(a[big] - b[big]) / b[big]
    print(f"max weight rel diff {rel.max():.3e} over {big.sum()} weights")
    assert big.sum() > 100
    assert rel.max() <= 1e-5


def test_est_sums_fp64_vs_oracle_and_reference(weighted_pair, ref):
    d = weighted_pair
    ours, theirs = d["ours"], d["theirs"]
    w = ours_weights(ours)
    pos, quat = ours.snapshot()
    s = ours.est_sums()
    o = oracle.est_sums(pos, quat, w)
    assert np.all(rel_close(s, o, 1e-9, 1e-15)), np.max(np.abs(s - o))
    # the reference fed the same weights
    ref_set_state(ref, theirs, pos, quat, w)
    r = theirs.est_sums()
    assert np.all(rel_close(s, r, 1e-5, 1e-9)), np.max(np.abs(s - r) / (np.abs(r) + 1e-9))


def test_covs_fp64_vs_oracle_and_reference(weighted_pair, ref):
    d = weighted_pair
    ours, theirs = d["ours"], d["theirs"]
    w = ours_weights(ours)
    pos, quat = ours.snapshot()
    s = ours.est_sums()
    m10 = s[3:13]
    q = np.zeros(4)
    pkg.core().pfcore_quat_mean(pkg.dptr(np.ascontiguousarray(m10)), pkg.dptr(q))
    mp = s[:3].astype(np.float32)
    mq = q.astype(np.float32)
    c = ours.covs(mp, mq)
    o = oracle.covs(pos, quat, w, mp, mq)
    assert np.all(rel_close(c, o, 1e-9, 1e-15)), np.max(np.abs(c - o))
    ref_set_state(ref, theirs, pos, quat, w)
    theirs.est_sums()
    r = theirs.covs(mp, mq)
    # relative to the largest variance of each block (off-diagonals can be ~0)
    scale = np.r_[np.full(6, np.abs(r[[0, 3, 5]]).max()), np.full(6, np.abs(r[[6, 9, 11]]).max())]
    assert np.all(scale > 0)
    assert np.all(np.abs(c - r) <= 1e-5 * scale), np.max(np.abs(c - r) / scale)


def test_covs_speculation_hits_and_misses(weighted_pair):
    ours = weighted_pair["ours"]
    s = ours.est_sums()
    q = np.zeros(4)
    pkg.core().pfcore_quat_mean(pkg.dptr(np.ascontiguousarray(s[3:13])), pkg.dptr(q))
    hit = ours.covs(s[:3].astype(np.float32), q.astype(np.float32))
    # a different mean must be honoured (recomputed, not the speculative one)
    other = ours.covs((s[:3] + 0.25).astype(np.float32), q.astype(np.float32))
    assert other[0] > hit[0]
    again = ours.covs(s[:3].astype(np.float32), q.astype(np.float32))
    assert np.array_equal(again, hit)


def _weighted_state(kernels, n, seed, sr=1.0):
    lm, obs, tp, tq = scale_obs(seed=seed)
    yaw = 2.0 * np.arctan2(tq[3], tq[0])
    pos, quat = cloud(n, seed, centre=tp, pos_std=0.2, rot_std=0.03, yaw=yaw)
    pf = RawPF(kernels, n, seed=3)
    ours_set_state(pf, pos, quat)
    pf.landmarks(lm)
    assert pf.weight(obs, sr, 0.02, 3.0) == 0
    return pf


# sr = 0.05 m puts (nearly) all weight on one particle: one scan tile then owns
# every output, the load-imbalance case of the ancestor runs.  4M is the
# largest size of the at-scale workload; beyond 4096 * 1024 particles the
# weight pass forms its block prefixes without staging them in shared memory.
@pytest.mark.parametrize("n,sr", [(1, 1.0), (7, 1.0), (4096, 1.0), (4097, 1.0), (50_000, 1.0),
                                  (1_000_000, 1.0), (1_000_000, 0.05), (4_000_000, 1.0),
                                  (4_500_000, 0.05)])
def test_resample_ancestors_bit_exact_vs_spec(kernels, n, sr):
    pf = _weighted_state(kernels, n, 21, sr)
    try:
        w = ours_weights(pf)
        pos0, quat0 = pf.snapshot()
        assert kernels.pfc_record_ancestors(pf.h, 1) == 0
        assert kernels.pfc_resample_u01(pf.h, 0.37, 0.0) == 0
        anc = np.zeros(n, np.int32)
        assert kernels.pfc_get_ancestors(pf.h, i32p(anc)) == 0
        ref_anc, _ = oracle.resample_fixed(w, 0.37)
        assert ref_anc is not None
        assert np.array_equal(anc, ref_anc)
        pos1, quat1 = pf.snapshot()
        assert np.array_equal(pos1.reshape(-1, 3), pos0.reshape(-1, 3)[anc])
        assert np.array_equal(quat1.reshape(-1, 4), quat0.reshape(-1, 4)[anc])
        assert np.all(ours_weights(pf) == np.float32(1.0) / np.float32(n))
    finally:
        pf.close()


def test_resample_lcg_stream_and_injection(kernels):
    n = 100_000
    pf = _weighted_state(kernels, n, 5)
    try:
        lcg0 = 0x1234_5678_9ABC_DEF1
        assert kernels.pfc_set_lcg(pf.h, lcg0) == 0
        w = ours_weights(pf)
        pos0, quat0 = pf.snapshot()
        assert kernels.pfc_record_ancestors(pf.h, 1) == 0
        assert kernels.pfc_resample(pf.h, 0.01) == 0
        lcg1 = C.c_ulonglong()
        assert kernels.pfc_get_lcg(pf.h, C.byref(lcg1)) == 0
        assert lcg1.value == oracle.lcg_next(lcg0)
        anc, _ = oracle.resample_fixed(w, oracle.lcg_u01(lcg1.value))
        got = np.zeros(n, np.int32)
        assert kernels.pfc_get_ancestors(pf.h, i32p(got)) == 0
        assert np.array_equal(got, anc)
        expect = pos0.reshape(-1, 3)[anc].reshape(-1).copy()
        k = int(np.float32(0.01) * np.float32(n))
        expect = oracle.inject_apply(expect, k, lcg1.value, 0)  # gen: no predict yet
        pos1, quat1 = pf.snapshot()
        assert np.array_equal(pos1, expect)
        assert np.array_equal(quat1.reshape(-1, 4), quat0.reshape(-1, 4)[anc])
    finally:
        pf.close()


def test_pick_rule_bit_exact_vs_reference_cum(kernels, ref):
    n = 50_000
    lm, obs, tp, tq = scale_obs(seed=8)
    yaw = 2.0 * np.arctan2(tq[3], tq[0])
    pos, quat = cloud(n, 8, centre=tp, pos_std=0.2, rot_std=0.03, yaw=yaw)
    theirs = RawPF(ref, n, seed=3)
    ours = RawPF(kernels, n, seed=3)
    try:
        ref_set_state(ref, theirs, pos, quat)
        theirs.landmarks(lm)
        assert theirs.weight(obs) == 0
        lcg0 = ref.ref_get_lcg(theirs.h)
        theirs.resample(0.0)
        cum = np.zeros(n)
        assert ref.ref_get_cum(theirs.h, f64p(cum)) == 0
        total = cum[-1]
        u0 = oracle.lcg_u01(oracle.lcg_next(lcg0)) * (total / n)
        anc = np.zeros(n, np.int32)
        assert kernels.pfc_pick_from_cum(ours.h, f64p(cum), n, u0, total, i32p(anc)) == 0
        rpos, rquat = theirs.snapshot()
        assert np.array_equal(rpos.reshape(-1, 3), pos.reshape(-1, 3)[anc])
        assert np.array_equal(rquat.reshape(-1, 4), quat.reshape(-1, 4)[anc])
        assert np.array_equal(anc, oracle.pick_from_cum(cum, u0, total))
    finally:
        ours.close()
        theirs.close()


def test_reinit_and_predict_match_oracle_noise(kernels):
    n = 20_000
    seed = 17
    pf = RawPF(kernels, n, seed=seed)
    orc = oracle.OraclePF(n, seed=seed)
    try:
        pose = [1.0, -2.0, 0.5, 0.9238795, 0.0, 0.0, 0.3826834]
        pf.reinit(pose, [0.5, 1.0, 0.2], [0.05, 0.1, 0.2])
        orc.reinit(np.float32(pose).astype(np.float64), np.float32([0.5, 1.0, 0.2]),
                   np.float32([0.05, 0.1, 0.2]))
        pos, quat = pf.snapshot()
        op, oq, _ = orc.state()
        assert np.max(np.abs(pos.reshape(-1, 3) - op)) < 2e-5
        assert np.max(np.abs(quat.reshape(-1, 4) - oq)) < 2e-6
        # predict one step from the GPU's own f32 state
        orc.set_state(pos.astype(np.float64), quat.astype(np.float64))
        t, q = [0.3, 0.05, -0.02], [0.99875026, 0.0, 0.0, 0.04997917]
        tn, rn = [0.02, 0.02, 0.01], [0.01, 0.01, 0.02]
        pf.predict(t, q, tn, rn)
        orc.predict(np.float32(t), np.float32(q), np.float32(tn), np.float32(rn))
        pos2, quat2 = pf.snapshot()
        op2, oq2, _ = orc.state()
        assert np.max(np.abs(pos2.reshape(-1, 3) - op2)) < 2e-5
        assert np.max(np.abs(quat2.reshape(-1, 4) - oq2)) < 2e-6
    finally:
        pf.close()


def test_reinit_noise_statistics(kernels):
    n = 400_000
    pf = RawPF(kernels, n, seed=5)
    try:
        ps = np.array([1.0, 2.0, 0.5])
        pf.reinit([0, 0, 0, 1, 0, 0, 0], ps, [0.0, 0.0, 0.0])
        pos, _ = pf.snapshot()
        p = pos.reshape(-1, 3).astype(np.float64)
        assert np.all(np.abs(p.mean(0)) < 4 * ps / np.sqrt(n))
        assert np.all(np.abs(p.std(0) / ps - 1.0) < 0.01)
        z = np.sort(p[:, 0] / ps[0])
        from math import erf, sqrt
        cdf = 0.5 * (1 + np.vectorize(erf)(z[::40] / sqrt(2)))
        emp = (np.arange(z.size)[::40] + 1) / z.size
        assert np.max(np.abs(cdf - emp)) < 0.005
    finally:
        pf.close()


def test_weight_edge_cases(kernels):
    n = 3000
    lm = np.array([[5.0, 5.0, 1.0], [1.0, 2.0, 3.0]])
    pf = RawPF(kernels, n, seed=4)
    try:
        pf.reinit([5, 5, 1, 1, 0, 0, 0], [3.0] * 3, [0.1] * 3)
        pf.landmarks(lm)
        uni = np.float32(1.0) / np.float32(n)
        # informative observation collapses the weights (ungated, as in
        # crates/pf_core/tests/cuda_agreement.rs:82-131)
        assert pf.weight([(0, 0, 0.0, 0.0, 0.0, 0.0)], gate=0.0) == 0
        w = ours_weights(pf)
        assert 1.0 / np.sum(w.astype(np.float64) ** 2) < n / 2
        # no observations -> uniform
        assert kernels.pfc_weight(pf.h, None, 0, 0.05, 0.02, 0.0) == 0
        assert np.all(ours_weights(pf) == uni)
        # ids outside the table are skipped -> all ll = 0 -> uniform
        assert pf.weight([(7, 0, 1.0, 0.0, 0.0, 0.0), (-1, 1, 1.0, 0, 0, 2.0)]) == 0
        assert np.allclose(ours_weights(pf), uni, rtol=1e-6)
        assert np.all(ours_ll(pf) == 0.0)
        # more observations than the capacity are clamped (cap 256)
        rows = [(0, 0, 0.0, 0.0, 0.0, 0.0)] * 300
        assert pf.weight(rows) == 0
        ll300 = ours_ll(pf)
        assert pf.weight(rows[:256]) == 0
        assert np.array_equal(ll300, ours_ll(pf))
        # NaN weights make the resample invalid: uniform weights, no gather
        pos0, quat0 = pf.snapshot()
        wn = np.full(n, 1.0 / n, np.float32)
        wn[5] = np.nan
        ours_set_state(pf, pos0, quat0, wn)
        assert kernels.pfc_resample(pf.h, 0.0) == 0
        pos1, _ = pf.snapshot()
        assert np.array_equal(pos0, pos1)
        assert np.all(ours_weights(pf) == uni)
        assert abs(pf.est_sums()[13] * n - 1.0) < 1e-6
    finally:
        pf.close()


def test_range_bearing_loglik_matches_reference(kernels, ref):
    n = 20_000
    lm = np.random.default_rng(2).uniform(-10, 10, size=(16, 3))
    pos, quat = cloud(n, 4, centre=(0.5, -0.5, 0.2), pos_std=0.4, rot_std=0.1)
    rng = np.random.default_rng(6)
    rows = []
    for k in range(40):
        i = int(rng.integers(0, 16))
        d = lm[i] - np.array([0.5, -0.5, 0.2])
        r = float(np.linalg.norm(d))
        u = -d / r  # the model compares -pred_dir with the observed direction
        rows.append((i, 1, *(u + rng.normal(scale=0.01, size=3)), r + rng.normal(scale=0.05)))
    ours = RawPF(kernels, n, seed=1)
    theirs = RawPF(ref, n, seed=1)
    try:
        for gate in (0.0, 3.0):
            ours_set_state(ours, pos, quat)
            ref_set_state(ref, theirs, pos, quat)
            ours.landmarks(lm)
            theirs.landmarks(lm)
            assert ours.weight(rows, 0.05, 0.02, gate) == 0
            assert theirs.weight(rows, 0.05, 0.02, gate) == 0
            a, b = ours_ll(ours), ref_ll(ref, theirs)
            # the same rounded operations as the reference kernel: identical bits
            assert np.array_equal(a, b), np.mean(a == b)
    finally:
        ours.close()
        theirs.close()


@pytest.mark.parametrize("gate", [0.0, 3.0])
def test_weight_variants_bit_identical(kernels, ref, gate):
    """The packed f32x2 path and the scalar path perform the same rounded
    operations as the reference kernel: all three agree bit for bit."""
    lm, obs, tp, tq = scale_obs(seed=4)
    yaw = 2.0 * np.arctan2(tq[3], tq[0])
    n = 30_001
    pos, quat = cloud(n, 2, centre=tp, pos_std=0.5, rot_std=0.05, yaw=yaw)
    outs = []
    for variant in (0, 1):
        pf = RawPF(kernels, n, seed=1)
        try:
            assert kernels.pfc_set_weight_kernel(pf.h, variant) == 0
            ours_set_state(pf, pos, quat)
            pf.landmarks(lm)
            assert pf.weight(obs, 0.05, 0.02, gate) == 0
            outs.append(ours_ll(pf))
        finally:
            pf.close()
    theirs = RawPF(ref, n, seed=1)
    try:
        ref_set_state(ref, theirs, pos, quat)
        theirs.landmarks(lm)
        assert theirs.weight(obs, 0.05, 0.02, gate) == 0
        r = ref_ll(ref, theirs)
    finally:
        theirs.close()
    assert np.array_equal(outs[0], outs[1])
    assert np.array_equal(outs[0], r)
