"""A particle filter sharded over ranks (pfc_shard_*, multi.ShardedFilter)
against the same filter on one handle (pfc_cycle): every rank predicts and
weights its slice, the exchange gives every rank the whole weighted cloud,
and every rank finishes the cycle on it.  The shards here are handles of one
process on one GPU with the in-process exchange (multi.update_in_process);
over several GPUs the exchange is an NCCL all-gather of the same chunks
(multi.exchange_views, whose plumbing the gloo test in
test_multirank_cpu.py covers).

Bar: every cycle's 24-value record and the final particles identical, bit
for bit, on every shard, over at-scale cycles that resample and inject
(softmax, ESS decision, ancestors, injection and estimates are computed from
the exchanged state by the same kernels)."""
import ctypes as C

import numpy as np
import pytest

import cuda_pf_localization_b200 as pkg
from cuda_pf_localization_b200 import multi, sim
from tests.pf_helpers import RawPF

pytestmark = pytest.mark.gpu


def _odom(st, sc):
    o = pkg.PfcOdom()
    o.t[:] = list(map(float, st.odom_t))
    o.q[:] = list(map(float, st.odom_q))
    o.tstd[:] = list(sc.trans_noise)
    o.rstd[:] = list(sc.rot_noise)
    return o


def _setup(lib, h, sc):
    lm = np.ascontiguousarray(sc.landmarks, np.float32).reshape(-1)
    assert lib.pfc_upload_landmarks(h, pkg.fptr(lm), lm.size // 3) == 0
    pri = np.r_[sc.prior_p, sc.prior_q]
    ps = np.full(3, 0.5, np.float32)
    rs = np.full(3, 0.2, np.float32)
    assert lib.pfc_reinit(h, *map(float, pri), pkg.fptr(ps), pkg.fptr(rs)) == 0


def _snapshot(lib, h, n):
    pos = np.zeros(3 * n, np.float32)
    quat = np.zeros(4 * n, np.float32)
    assert lib.pfc_snapshot(h, pkg.fptr(pos), pkg.fptr(quat)) == 0
    return pos, quat


@pytest.mark.parametrize("n,world", [(100_003, 2), (100_003, 3), (4097, 4), (1_000_000, 2)])
def test_sharded_filter_equals_single_filter(kernels, n, world):
    sc = sim.scale_config(cycles=6, seed=5)
    prm = pkg.PfcCycleParams(0.05, 0.02, 3.0, 0.5, 0.01, 0)
    single = RawPF(kernels, n, seed=9)
    shards = [multi.ShardedFilter(n, world, r, seed=9) for r in range(world)]
    try:
        for h in [single.h] + [s.h for s in shards]:
            _setup(kernels, h, sc)
        resampled = 0
        for st in sc.steps:
            odom = _odom(st, sc)
            cobs = pkg.make_cobs(st.obs)
            e1 = np.zeros(pkg.PFC_EST_LEN)
            assert kernels.pfc_cycle(single.h, C.byref(odom), cobs, len(st.obs), C.byref(prm),
                                     pkg.dptr(e1)) == 0
            for e in multi.update_in_process(shards, odom, st.obs, prm):
                np.testing.assert_array_equal(e, e1)
            resampled += int(e1[pkg.PFC_EST_RESAMPLED])
        assert resampled >= 3
        p1, q1 = _snapshot(kernels, single.h, n)
        for s in shards:
            p, q = _snapshot(kernels, s.h, n)
            np.testing.assert_array_equal(p, p1)
            np.testing.assert_array_equal(q, q1)
    finally:
        single.close()
        for s in shards:
            s.close()


def test_cycle_without_observations_matches(kernels):
    """A cycle with no observations keeps uniform weights on both forms."""
    n, world = 20_000, 2
    sc = sim.scale_config(cycles=2, seed=7)
    prm = pkg.PfcCycleParams(0.05, 0.02, 3.0, 0.5, 0.0, 0)
    single = RawPF(kernels, n, seed=3)
    shards = [multi.ShardedFilter(n, world, r, seed=3) for r in range(world)]
    try:
        for h in [single.h] + [s.h for s in shards]:
            _setup(kernels, h, sc)
        # the first cycle without observations, the second with them
        for st, rows in zip(sc.steps, ([], sc.steps[1].obs)):
            odom = _odom(st, sc)
            e1 = np.zeros(pkg.PFC_EST_LEN)
            cobs = pkg.make_cobs(rows) if len(rows) else None
            assert kernels.pfc_cycle(single.h, C.byref(odom), cobs, len(rows), C.byref(prm),
                                     pkg.dptr(e1)) == 0
            for e in multi.update_in_process(shards, odom, rows, prm):
                np.testing.assert_array_equal(e, e1)
        p1, q1 = _snapshot(kernels, single.h, n)
        p, q = _snapshot(kernels, shards[1].h, n)
        np.testing.assert_array_equal(p, p1)
        np.testing.assert_array_equal(q, q1)
    finally:
        single.close()
        for s in shards:
            s.close()


def test_shard_calls_checked(kernels):
    h = kernels.pfc_create(64)
    try:
        assert kernels.pfc_shard_init(h, 1000, 2, 2, 1) == -1
        assert kernels.pfc_shard_init(h, 0, 1, 0, 1) == -1
        assert kernels.pfc_init(h, 1000, 1) == 0
        odom = pkg.PfcOdom()
        prm = pkg.PfcCycleParams(0.05, 0.02, 3.0, 0.5, 0.0, 0)
        # a plain handle is not a shard
        assert kernels.pfc_shard_weight(h, C.byref(odom), None, 0, C.byref(prm)) == -1
        assert "not a shard handle" in pkg.last_error()
        assert kernels.pfc_shard_finish(h, C.byref(prm), None) == -1
        assert kernels.pfc_shard_init(h, 1000, 3, 1, 1) == 0
        chunk, n_pad = C.c_int(), C.c_int()
        assert kernels.pfc_shard_layout(h, C.byref(chunk), C.byref(n_pad)) == 0
        assert chunk.value == 2048 and n_pad.value == 3 * 2048
    finally:
        kernels.pfc_destroy(h)
