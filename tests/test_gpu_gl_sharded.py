"""A CBGL query sharded by hypotheses: each rank generates its slice of the
global dispersion (pfgl_generate_yaws_range) and keeps its k best composite
keys; merging the ranks' candidates gives exactly the bottom-k of localizing
the whole set on one GPU.  The ranks run one after another on one GPU here
(independent launches, nothing waits on another rank); the all-gather itself
is covered by the gloo tests in test_multirank_cpu.py."""
import math

import numpy as np
import pytest

import cuda_pf_localization_b200 as pkg
from cuda_pf_localization_b200 import multi, sim

pytestmark = pytest.mark.gpu

SEED = 4242
N_YAW = 16


@pytest.fixture(scope="module")
def gl():
    g = np.ascontiguousarray(sim.rooms_grid(31))
    lib = pkg.kernels()
    h = lib.pfgl_create(200, 200, 0.05, 0.0, 0.0, pkg.u8ptr(g), 400_000)
    assert h
    rng = np.random.default_rng(2)
    truth = np.array([sim.free_pose(g, rng)], np.float32)
    scan = pkg.render_scans(h, truth, noise=0.01, seed=5)[0]
    yield h, scan
    lib.pfgl_destroy(h)


def test_range_dispersion_equals_rows_of_whole(gl):
    h, _ = gl
    lib = pkg.kernels()
    n_pos = 1000
    assert lib.pfgl_generate_yaws(h, n_pos, N_YAW, SEED) == 0
    whole = np.zeros(3 * n_pos * N_YAW, np.float32)
    assert lib.pfgl_get_hyps(h, pkg.fptr(whole)) == 0
    whole = whole.reshape(-1, 3)
    for p0, m in [(0, 1), (17, 100), (999, 1), (500, 500)]:
        assert lib.pfgl_generate_yaws_range(h, p0, m, N_YAW, SEED) == 0
        part = np.zeros(3 * m * N_YAW, np.float32)
        assert lib.pfgl_get_hyps(h, pkg.fptr(part)) == 0
        np.testing.assert_array_equal(part.reshape(-1, 3),
                                      whole[p0 * N_YAW:(p0 + m) * N_YAW])
    assert lib.pfgl_generate_yaws_range(h, -1, 10, N_YAW, SEED) == -1


@pytest.mark.parametrize("n_pos,world", [(12_500, 2), (12_500, 3), (20_000, 8), (5, 8)])
def test_sharded_bottom_k_equals_single_gpu(gl, n_pos, world):
    h, scan = gl
    lib = pkg.kernels()
    k = 64
    span, rmax = 2 * math.pi, 10.0
    # the whole set on one GPU
    assert lib.pfgl_generate_yaws(h, n_pos, N_YAW, SEED) == 0
    kf = min(k, n_pos * N_YAW)
    out = np.zeros(3 * kf, np.float32)
    cs = np.zeros(kf, np.float32)
    ids = np.zeros(kf, np.int32)
    assert lib.pfgl_localize(h, pkg.fptr(scan), 360, rmax, span, kf, pkg.fptr(out),
                             pkg.fptr(cs), pkg.iptr(ids)) == kf
    # the ranks' shards, one after another, merged
    keys, poses = [], []
    for rank in range(world):
        kk, pp = multi.local_bottom_k(h, scan, n_pos, N_YAW, SEED, k, world, rank)
        keys.append(kk)
        poses.append(pp)
    mk, mp = multi.merge_bottom_k(np.concatenate(keys), np.concatenate(poses), k, None)
    np.testing.assert_array_equal((mk & np.uint64(0xFFFFFFFF)).astype(np.int64), ids)
    np.testing.assert_array_equal(multi.key_caer(mk), cs)
    np.testing.assert_array_equal(mp, out.reshape(-1, 3))
