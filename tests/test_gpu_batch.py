"""Batched filters: every filter of a batch equals the same filter run alone
through the single-filter fused cycle (same seed, same inputs) — particles and
weights bit for bit, estimate records to FP64 rounding — with and without the
CUDA graph and for every estimate tile size.
"""
import ctypes as C

import numpy as np
import pytest

import cuda_pf_localization_b200 as pkg
from cuda_pf_localization_b200 import sim

pytestmark = pytest.mark.gpu

SIZES = [1000, 1537, 4096, 5000, 20000, 70001]
CYCLES = 6
PRM = dict(sigma_r=0.05, sigma_b=0.02, gate=3.0, ess_ratio=0.5, inject=0.01)


def _workload(seed=5):
    rng = np.random.default_rng(seed)
    scen, counts = [], []
    for f, n in enumerate(SIZES):
        sc = sim.helix_scenario(CYCLES, int(rng.integers(8, 65)), (20.0, 20.0, 5.0), 64, 0.1,
                                100 + f, phase=float(rng.uniform(0, 6.28)))
        c = rng.integers(4, 65, size=CYCLES)
        c[f % CYCLES] = 0 if f == 2 else c[f % CYCLES]  # one predict-only cycle
        for k, st in enumerate(sc.steps):
            st.obs = st.obs[: int(c[k])]
            if f == 3:  # range-bearing observations in one filter
                st.obs = st.obs.copy()
                v = st.obs[:, 2:5]
                r = np.linalg.norm(v, axis=1)
                st.obs[:, 1] = 1
                st.obs[:, 5] = r
                st.obs[:, 2:5] = v / np.maximum(r, 1e-9)[:, None]
        scen.append(sc)
        counts.append(c)
    return scen


def _odom(sc, st):
    o = pkg.PfcOdom()
    o.t[:] = list(map(float, st.odom_t))
    o.q[:] = list(map(float, st.odom_q))
    o.tstd[:] = list(sc.trans_noise)
    o.rstd[:] = list(sc.rot_noise)
    return o


def _run_singles(scen, seeds):
    lib = pkg.kernels()
    out = []
    prm = pkg.PfcCycleParams(PRM["sigma_r"], PRM["sigma_b"], PRM["gate"], PRM["ess_ratio"],
                             PRM["inject"], 0)
    for f, (n, sc) in enumerate(zip(SIZES, scen)):
        h = lib.pfc_create(256)
        try:
            assert lib.pfc_init(h, n, seeds[f]) == 0
            lm = np.ascontiguousarray(sc.landmarks, np.float32).reshape(-1)
            assert lib.pfc_upload_landmarks(h, pkg.fptr(lm), len(sc.landmarks)) == 0
            pri = np.r_[sc.prior_p, sc.prior_q].astype(np.float32)
            ps, rs = np.full(3, 0.5, np.float32), np.full(3, 0.2, np.float32)
            assert lib.pfc_reinit(h, *map(float, pri), pkg.fptr(ps), pkg.fptr(rs)) == 0
            ests = []
            for st in sc.steps:
                est = np.zeros(pkg.PFC_EST_LEN)
                obs = pkg.make_cobs(st.obs)
                assert lib.pfc_cycle(h, C.byref(_odom(sc, st)), obs, len(st.obs),
                                     C.byref(prm), pkg.dptr(est)) == 0
                ests.append(est)
            pos = np.zeros(3 * n, np.float32)
            quat = np.zeros(4 * n, np.float32)
            assert lib.pfc_snapshot(h, pkg.fptr(pos), pkg.fptr(quat)) == 0
            w = np.zeros(n, np.float32)
            assert lib.pfc_get_weights(h, pkg.fptr(w)) == 0
            out.append((np.array(ests), pos, quat, w))
        finally:
            lib.pfc_destroy(h)
    return out


def _run_batch(scen, seeds, graph=True, tiles=None):
    b = pkg.BatchPF(SIZES, seeds=seeds)
    try:
        b.set_params(**PRM)
        b.set_landmarks([sc.landmarks for sc in scen])
        if tiles is not None:
            b.set_tiles(tiles)
        b.use_graph(graph)
        pose7 = np.array([np.r_[sc.prior_p, sc.prior_q] for sc in scen], np.float32)
        b.reinit(pose7, np.full((len(SIZES), 3), 0.5), np.full((len(SIZES), 3), 0.2))
        ests = []
        for k in range(CYCLES):
            odoms = [_odom(sc, sc.steps[k]) for sc in scen]
            ests.append(b.cycle(odoms, [sc.steps[k].obs for sc in scen]))
        snaps = [b.snapshot(f) for f in range(len(SIZES))]
        ws = [b.weights(f) for f in range(len(SIZES))]
        launches = b.lib.pfc_batch_launches(b.handle)
        return np.array(ests), snaps, ws, launches
    finally:
        b.close()


@pytest.fixture(scope="module")
def reference_run(kernels):
    scen = _workload()
    seeds = [31 + 7 * f for f in range(len(SIZES))]
    return scen, seeds, _run_singles(scen, seeds)


def _compare(ref, ests, snaps, ws):
    resampled_any = False
    for f in range(len(SIZES)):
        r_est, r_pos, r_quat, r_w = ref[f]
        b_est = ests[:, f, :]
        # resampling decisions and every particle identical
        assert np.array_equal(b_est[:, pkg.PFC_EST_RESAMPLED], r_est[:, pkg.PFC_EST_RESAMPLED])
        resampled_any |= bool(r_est[:, pkg.PFC_EST_RESAMPLED].any())
        assert np.array_equal(snaps[f][0], r_pos), f
        assert np.array_equal(snaps[f][1], r_quat), f
        assert np.array_equal(ws[f], r_w), f
        # estimate records: FP64 sums over different tiles
        assert np.allclose(b_est[:, :22], r_est[:, :22], rtol=1e-9, atol=1e-12), f
    assert resampled_any


def test_batch_equals_single_filters(reference_run):
    scen, seeds, ref = reference_run
    ests, snaps, ws, launches = _run_batch(scen, seeds, graph=True)
    _compare(ref, ests, snaps, ws)
    assert launches > 0


def test_batch_without_graph_equal(reference_run):
    scen, seeds, ref = reference_run
    ests, snaps, ws, _ = _run_batch(scen, seeds, graph=False)
    _compare(ref, ests, snaps, ws)


@pytest.mark.parametrize("tiles", [[1024, 1024, 2048, 4096], [32768, 16384, 8192, 2048]])
def test_batch_tile_choices_equal(reference_run, tiles):
    scen, seeds, ref = reference_run
    ests, snaps, ws, _ = _run_batch(scen, seeds, tiles=tiles)
    _compare(ref, ests, snaps, ws)


def test_batch_autotune_keeps_results(reference_run):
    scen, seeds, ref = reference_run
    b = pkg.BatchPF(SIZES, seeds=seeds)
    try:
        b.set_params(**PRM)
        b.set_landmarks([sc.landmarks for sc in scen])
        pose7 = np.array([np.r_[sc.prior_p, sc.prior_q] for sc in scen], np.float32)
        b.reinit(pose7, np.full((len(SIZES), 3), 0.5), np.full((len(SIZES), 3), 0.2))
        ests = []
        for k in range(CYCLES):
            if k == 1:
                tiles, _ = b.autotune(reps=2)
                assert all(t in (2048, 4096, 8192, 16384, 32768) for t in tiles)
            odoms = [_odom(sc, sc.steps[k]) for sc in scen]
            ests.append(b.cycle(odoms, [sc.steps[k].obs for sc in scen]))
        snaps = [b.snapshot(f) for f in range(len(SIZES))]
        ws = [b.weights(f) for f in range(len(SIZES))]
    finally:
        b.close()
    _compare(ref, np.array(ests), snaps, ws)
