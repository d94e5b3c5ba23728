"""Batched global localization: many queries scored in one launch.

Uniform batch (pfgl_localize_batch): each query's CAERs, bottom-k poses and
indices equal the single-query path's (its own dispersion, exhaustive
pfgl_score, pfgl_topk_ex) bit for bit, also when the batch is split into
chunks by the hypothesis capacity.

Learned batch (pfgl_learned_localize_batch): every query's bottom-k is the
stable CAER order of its own samples (checked against the CPU oracle's sort
and against pfgl_score of the same hypotheses), the batch localizes unseen
poses as well as the single-query path, and the fallback obeys the
threshold."""
import math

import numpy as np
import pytest

import cuda_pf_localization_b200 as pkg
import oracle
from cuda_pf_localization_b200 import sim

pytestmark = pytest.mark.gpu

SPAN, RMAX = 2 * math.pi, 10.0


def _gl(seed, cap):
    lib = pkg.kernels()
    g = np.ascontiguousarray(sim.rooms_grid(seed))
    h = lib.pfgl_create(200, 200, 0.05, 0.0, 0.0, pkg.u8ptr(g), cap)
    assert h
    return lib, g, h


def _scans(g, h, n, seed):
    rng = np.random.default_rng(seed)
    poses = np.array([sim.free_pose(g, rng) for _ in range(n)], np.float32)
    return poses, pkg.render_scans(h, poses, noise=0.01, seed=seed + 1)


@pytest.mark.parametrize("cap", [1 << 20, 40_000])
def test_uniform_batch_equals_single_queries(kernels, cap):
    lib, g, h = _gl(7, cap)
    try:
        _, scans = _scans(g, h, 5, 11)
        n_pos, n_yaw, k = 1000, 16, 64
        seeds = np.array([900 + 7 * q for q in range(5)], np.uint64)
        bp, bc, bi = pkg.localize_batch(h, scans, n_pos, n_yaw, seeds, k)
        for q in range(5):
            assert lib.pfgl_generate_yaws(h, n_pos, n_yaw, int(seeds[q])) == 0
            assert lib.pfgl_score(h, pkg.fptr(scans[q]), 360, RMAX, SPAN) == 0
            out = np.zeros(3 * k, np.float32)
            cs = np.zeros(k, np.float32)
            ids = np.zeros(k, np.int32)
            assert lib.pfgl_topk_ex(h, k, pkg.fptr(out), pkg.fptr(cs), pkg.iptr(ids)) == k
            np.testing.assert_array_equal(bi[q], ids)
            np.testing.assert_array_equal(bc[q], cs)
            np.testing.assert_array_equal(bp[q], out.reshape(k, 3))
    finally:
        lib.pfgl_destroy(h)


def test_uniform_batch_rejects_oversized_queries(kernels):
    lib, g, h = _gl(7, 1 << 20)
    try:
        _, scans = _scans(g, h, 2, 3)
        with pytest.raises(RuntimeError):
            pkg.localize_batch(h, scans, 5000, 16, [1, 2], 64)   # 80k > 65536 per query
        with pytest.raises(RuntimeError):
            pkg.localize_batch(h, scans, 100, 16, [1, 2], 129)   # k > 128
    finally:
        lib.pfgl_destroy(h)


@pytest.fixture(scope="module")
def trained():
    lib, g, h = _gl(21, 1 << 20)
    lp = pkg.LearnedProposal(h, batch=1024, seed=3)
    lp.make_data(524_288, seed=17)
    lp.train(2000, lr=1e-3)
    yield lib, g, h, lp
    lp.close()
    lib.pfgl_destroy(h)


def test_learned_batch_bottom_k_is_stable_caer_order(trained):
    lib, g, h, lp = trained
    _, scans = _scans(g, h, 40, 31)
    S, k = 700, 64
    out, cs, ids, info = lp.localize_batch(scans, n_samples=S, n_fallback=0, k=k)
    assert np.all(info == 0)
    # one chunk (40 * 700 <= capacity): the batch's samples and CAERs are on
    # the handle
    hyp = np.zeros(3 * 40 * S, np.float32)
    caer = np.zeros(40 * S, np.float32)
    assert lib.pfgl_get_hyps(h, pkg.fptr(hyp)) == 0
    assert lib.pfgl_get_caer(h, pkg.fptr(caer)) == 0
    hyp = hyp.reshape(40, S, 3)
    caer = caer.reshape(40, S)
    for q in range(40):
        order = oracle.topk_from_scores(caer[q], k)
        np.testing.assert_array_equal(ids[q], order)
        np.testing.assert_array_equal(cs[q], caer[q][order])
        np.testing.assert_array_equal(out[q], hyp[q][order])
    # the batched CAERs are the single-query scorer's, bit for bit
    for q in (0, 17, 39):
        flat = np.ascontiguousarray(hyp[q].reshape(-1))
        assert lib.pfgl_set_hyps(h, pkg.fptr(flat), S) == 0
        assert lib.pfgl_score(h, pkg.fptr(scans[q]), 360, RMAX, SPAN) == 0
        c1 = np.zeros(S, np.float32)
        assert lib.pfgl_get_caer(h, pkg.fptr(c1)) == 0
        np.testing.assert_array_equal(c1, caer[q])


def _success(top, poses):
    dp = np.hypot(top[:, 0] - poses[:, 0], top[:, 1] - poses[:, 1])
    dth = np.abs((top[:, 2] - poses[:, 2] + np.pi) % (2 * np.pi) - np.pi)
    return (dp <= 0.5) & (dth <= 0.1)


def test_learned_batch_localizes_like_single_queries(trained):
    lib, g, h, lp = trained
    poses, scans = _scans(g, h, 200, 41)
    out, _, _, _ = lp.localize_batch(scans, n_samples=2000, n_fallback=0, k=8)
    ok_b = _success(out[:, 0], poses)
    ok_s = np.array([_success(lp.localize(scans[q], n_samples=2000, n_fallback=0, k=1)[0],
                              poses[q:q + 1])[0] for q in range(len(poses))])
    print(f"\nbatch {ok_b.mean():.3f} single {ok_s.mean():.3f}")
    assert ok_b.mean() >= 0.85
    assert abs(ok_b.mean() - ok_s.mean()) <= 0.05


def test_learned_batch_fallback_follows_threshold(trained):
    lib, g, h, lp = trained
    poses, scans = _scans(g, h, 12, 51)
    lp.set_threshold(-1.0)                   # every query falls back
    _, cs, _, info = lp.localize_batch(scans, n_samples=500, n_fallback=16_000, k=8)
    assert np.all(info >= 1)
    assert np.all(np.isfinite(cs)) and np.all(np.diff(cs, axis=1) >= 0)
    lp.set_threshold(float("inf"))           # none does
    _, _, _, info = lp.localize_batch(scans, n_samples=500, n_fallback=16_000, k=8)
    assert np.all(info == 0)
    tau, held = lp.calibrate(n_queries=100, n_samples=1000, seed=5)
    assert np.isfinite(tau) and held >= 0.8
