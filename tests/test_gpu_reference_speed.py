"""The library against the reference's own CUDA library (built from its source
for sm_100a) on the same B200 and the same inputs: the drop-in paths must not
be slower.  Prints both throughputs.
"""
import ctypes as C
import math
import time

import numpy as np
import pytest

import cuda_pf_localization_b200 as pkg
from cuda_pf_localization_b200 import sim

pytestmark = pytest.mark.gpu

N = 1_000_000
FILTER = dict(range_noise=0.05, bearing_noise=0.02, gate_sigma=3.0, resample_ess_ratio=0.5,
              random_inject_ratio=0.01)


def _ref_cycles(ref, sc, n, cycles):
    """Reference library in the Rust CudaBackend call order (predict, weight,
    est_sums -> host Markley mean -> covs, resample when ESS < N/2 and the
    second estimate); returns particle-updates/s."""
    f32 = lambda a: np.ascontiguousarray(a, np.float32)
    h = ref.pfc_create(256)
    try:
        assert ref.pfc_init(h, n, 42) == 0
        lm = f32(sc.landmarks).reshape(-1)
        ref.pfc_upload_landmarks(h, pkg.fptr(lm), len(sc.landmarks))
        pri = np.r_[sc.prior_p, sc.prior_q]
        ps, rs = f32([0.5] * 3), f32([0.2] * 3)
        ref.pfc_reinit(h, *map(float, pri), pkg.fptr(ps), pkg.fptr(rs))
        tn, rn = f32(sc.trans_noise), f32(sc.rot_noise)
        obs = [pkg.make_cobs(st.obs) for st in sc.steps]
        sums, cv = np.zeros(14), np.zeros(12)

        def estimate():
            ref.pfc_est_sums(h, pkg.dptr(sums))
            m = np.zeros((4, 4))
            e = 3
            for r in range(4):
                for c in range(r, 4):
                    m[r, c] = m[c, r] = sums[e]
                    e += 1
            vals, vecs = np.linalg.eigh(m)
            q = vecs[:, int(np.argmax(vals))]
            q = q if q[0] >= 0 else -q
            ref.pfc_covs(h, float(sums[0]), float(sums[1]), float(sums[2]), *map(float, q),
                         pkg.dptr(cv))
            return 1.0 / sums[13] if sums[13] > 0 else 0.0

        def cycle(k):
            st = sc.steps[k]
            ref.pfc_predict(h, *map(float, st.odom_t), *map(float, st.odom_q), pkg.fptr(tn),
                            pkg.fptr(rn))
            ref.pfc_weight(h, C.cast(obs[k], C.c_void_p), len(st.obs), 0.05, 0.02, 3.0)
            if estimate() < 0.5 * n:
                ref.pfc_resample(h, 0.01)
                estimate()

        for k in range(2):
            cycle(k)
        t0 = time.perf_counter()
        for k in range(2, 2 + cycles):
            cycle(k)
        return n * cycles / (time.perf_counter() - t0)
    finally:
        ref.pfc_destroy(h)


def _our_cycles(sc, n, cycles):
    core = pkg.core()
    pf = pkg.ParticleFilter(n, seed=42, trans_noise=sc.trans_noise, rot_noise=sc.rot_noise,
                            **FILTER)
    try:
        pf.set_map(sc.landmark_dict())
        pf.reinitialize(np.r_[sc.prior_p, sc.prior_q], [0.5] * 3, [0.2] * 3)
        odoms = [pkg.make_core_odom(st.odom_t, st.odom_q, sc.trans_noise, sc.rot_noise)
                 for st in sc.steps]
        obs = [pkg.make_core_obs(st.obs) for st in sc.steps]
        est = pkg.PfcoreEstimate()
        for k in range(2):
            assert core.pfcore_filter_update(pf._h, C.byref(odoms[k]), obs[k],
                                             len(sc.steps[k].obs), C.byref(est)) == 0
        t0 = time.perf_counter()
        for k in range(2, 2 + cycles):
            assert core.pfcore_filter_update(pf._h, C.byref(odoms[k]), obs[k],
                                             len(sc.steps[k].obs), C.byref(est)) == 0
        return n * cycles / (time.perf_counter() - t0)
    finally:
        pf.close()


def test_pf_cycle_not_slower_than_reference_library(kernels, ref):
    sc = sim.helix_scenario(24, 64, (50.0, 50.0, 10.0), 256, 0.10, 11)
    ours = _our_cycles(sc, N, 20)
    theirs = _ref_cycles(ref, sc, N, 20)
    print(f"\nPF cycle @1M (drop-in path): ours {ours:.3e} /s, reference {theirs:.3e} /s, "
          f"ratio {ours / theirs:.2f}")
    assert ours >= theirs


def test_gl_not_slower_than_reference_library(kernels, ref):
    lib = pkg.kernels()
    g = np.ascontiguousarray(sim.rooms_grid(11))
    nh, k = 1_000_000, 64
    rng = np.random.default_rng(12)
    h = lib.pfgl_create(200, 200, 0.05, 0.0, 0.0, pkg.u8ptr(g), nh)
    rh = ref.pfgl_create(200, 200, 0.05, 0.0, 0.0, pkg.u8ptr(g), nh)
    try:
        poses = np.array([sim.free_pose(g, rng) for _ in range(5)], np.float32)
        scans = pkg.render_scans(h, poses, noise=0.01, seed=3)
        out = np.zeros(3 * k, np.float32)

        def ours_solve(t):
            lib.pfgl_generate(h, nh, 100 + t)
            assert lib.pfgl_score(h, pkg.fptr(scans[t]), 360, 10.0, 2 * math.pi) == 0
            assert lib.pfgl_topk(h, k, pkg.fptr(out)) == k

        def ref_solve(t):
            ref.pfgl_generate(rh, nh, 100 + t)
            ref.pfgl_score(rh, pkg.fptr(scans[t]), 360, 10.0, 2 * math.pi)
            assert ref.pfgl_topk(rh, k, pkg.fptr(out)) == k

        rates = []
        for solve in (ours_solve, ref_solve):
            solve(0)
            t0 = time.perf_counter()
            for t in range(len(poses)):
                solve(t)
            rates.append(len(poses) / (time.perf_counter() - t0))
        print(f"\nCBGL @1M hypotheses (pfgl_generate/score/topk): ours {rates[0]:.1f} solves/s, "
              f"reference {rates[1]:.1f} solves/s")
        assert rates[0] >= rates[1]
    finally:
        lib.pfgl_destroy(h)
        ref.pfgl_destroy(rh)
