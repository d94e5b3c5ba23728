"""Pins the CPU oracle with the reference's own tests.

Each test restates one test of the reference (cited) against the oracle, with
the reference's thresholds: crates/pf_core/tests/integration.rs,
crates/pf_core/tests/global_loc.rs and, for the analytic-prior checks,
crates/pf_core/tests/cuda_agreement.rs (which holds the CPU backend to the
same bounds as the GPU).
"""
import math

import numpy as np
import pytest

import oracle
from cuda_pf_localization_b200 import sim

TAU = 2 * math.pi


def test_raycast_hits_walls_at_expected_distance():
    # crates/pf_core/tests/global_loc.rs:11-23
    g = sim.room_grid()
    d = oracle.cast_ray(g, 0.05, (0, 0), 5.0, 5.0, 1.0, 0.0, 20.0)
    assert abs(d - 4.95) < 0.15
    d2 = oracle.cast_ray(g, 0.05, (0, 0), 5.0, 5.0, 0.0, 1.0, 20.0)
    assert abs(d2 - 4.95) < 0.15


def test_raycast_hits_interior_pillar():
    # crates/pf_core/tests/global_loc.rs:25-34
    g = sim.room_grid()
    d = oracle.cast_ray(g, 0.05, (0, 0), 2.5, 5.0, 1.0, 0.0, 20.0)
    assert abs(d - 1.25) < 0.12


def test_raycast_respects_rmax():
    # crates/pf_core/tests/global_loc.rs:36-41
    g = sim.room_grid()
    assert oracle.cast_ray(g, 0.05, (0, 0), 5.0, 5.0, 1.0, 0.0, 2.0) == 2.0


def test_cpu_gl_recovers_pose_in_synthetic_room():
    # crates/pf_core/tests/global_loc.rs:43-67
    g = sim.room_grid()
    truth = (6.0, 7.0, 0.8)
    scan = oracle.map_scan(g, 0.05, (0, 0), *truth, 360, TAU, 10.0)
    top = oracle.gl_localize(g, 0.05, (0, 0), scan, TAU, 10.0, 20000, 10, 7)
    assert len(top) > 0
    best = top[0]
    assert math.hypot(best[0] - truth[0], best[1] - truth[1]) < 0.35
    assert np.all(np.diff(top[:, 3]) >= 0)


def _run_oracle_filter(sc, n, seed, pos_std, rot_std, ess_ratio=0.5, gate=0.0, inject=0.0):
    pf = oracle.OraclePF(n, seed=seed, range_noise=0.05, gate=gate, ess_ratio=ess_ratio,
                         inject=inject)
    pf.reinit(np.r_[sc.prior_p, sc.prior_q], pos_std, rot_std)
    errs = []
    for st in sc.steps:
        est, _ = pf.update(st.odom_t, st.odom_q, sc.trans_noise, sc.rot_noise, sc.landmarks,
                           st.obs)
        errs.append(float(np.linalg.norm(est["position"] - st.truth_p)))
    return np.array(errs), pf


def test_converges_on_3d_trajectory():
    # crates/pf_core/tests/integration.rs:11-38 (N=4096, seed 123,
    # circle_scenario(100, 777), prior spread 1 m / 0.5 rad, mean error < 0.25)
    sc = sim.circle_scenario(100, 777)
    assert all(len(s.obs) > 0 for s in sc.steps)
    errs, _ = _run_oracle_filter(sc, 4096, 123, [1.0] * 3, [0.5] * 3)
    assert errs.mean() < 0.25, errs.mean()


def test_coasts_without_observations():
    # crates/pf_core/tests/integration.rs:40-68
    pf = oracle.OraclePF(1024, seed=5)
    pf.reinit([1.0, 2.0, 3.0, 1.0, 0.0, 0.0, 0.0], [0.1] * 3, [0.01] * 3)
    for _ in range(20):
        est, _ = pf.update([1.0, 0.0, 0.0], [1.0, 0, 0, 0], [0.01] * 3, [0.005] * 3,
                           np.zeros((0, 3)), [])
    assert abs(est["position"][0] - 21.0) < 0.5
    assert abs(est["position"][1] - 2.0) < 0.2
    assert abs(est["position"][2] - 3.0) < 0.2


def test_ess_drops_on_informative_observation():
    # crates/pf_core/tests/integration.rs:70-101
    pf = oracle.OraclePF(2048, seed=77, ess_ratio=0.0)
    pf.reinit([5.0, 5.0, 1.0, 1.0, 0.0, 0.0, 0.0], [3.0] * 3, [0.1] * 3)
    lm = np.array([[5.0, 5.0, 1.0]])
    est, _ = pf.update([0, 0, 0], [1, 0, 0, 0], [0.05, 0.05, 0.05], [0.02, 0.02, 0.03], lm,
                       [(0, 0, 0.0, 0.0, 0.0, 0.0)])
    assert est["ess"] < 1024.0
    assert abs(est["position"][0] - 5.0) < 0.5


def test_quaternion_mean_handles_sign_flip():
    # crates/pf_core/tests/integration.rs:103-120
    pf = oracle.OraclePF(2, seed=42)
    pf.reinit([0, 0, 0, 1, 0, 0, 0], [1e-9] * 3, [0.0] * 3)
    est = pf.estimate()
    assert abs(abs(est["attitude"][0]) - 1.0) < 1e-6
    # antipodal quaternions describe the same rotation: the mean is unchanged
    p, q, w = pf.state()
    q[1] = -q[1]
    pf.set_state(p.reshape(-1), q.reshape(-1))
    assert abs(abs(pf.estimate()["attitude"][0]) - 1.0) < 1e-6


def test_covariances_match_gaussian_prior():
    # crates/pf_core/tests/cuda_agreement.rs:30-80 (CPU side of the check)
    n = 200_000
    pos_std = np.array([1.0, 2.0, 0.5])
    rot_std = np.array([0.05, 0.07, 0.02])
    pf = oracle.OraclePF(n, seed=7)
    pf.reinit([0, 0, 0, 1, 0, 0, 0], pos_std, rot_std)
    e = pf.estimate()
    for i in range(3):
        want = pos_std[i] ** 2
        assert abs(e["pos_cov"][i, i] - want) < 0.12 * want
        wrot = rot_std[i] ** 2
        assert abs(e["att_cov"][i, i] - wrot) < 0.15 * wrot
        for j in range(3):
            if i != j:
                assert abs(e["pos_cov"][i, j]) < 0.1 * want
                assert abs(e["att_cov"][i, j]) < 0.1 * wrot
    assert np.all(np.abs(e["position"]) < 0.05)


def test_tight_cloud_attitude_covariance():
    # crates/pf_core/tests/cuda_agreement.rs:177-219 (CPU side: att_cov within
    # 5 % of sigma^2, ESS of a uniform cloud = N)
    n = 100_000
    rot_std = np.array([1e-3, 2e-3, 3e-3])
    pf = oracle.OraclePF(n, seed=7)
    pf.reinit([0, 0, 0, 1, 0, 0, 0], [0.01] * 3, rot_std)
    e = pf.estimate()
    assert abs(e["ess"] - n) < 1e-6 * n
    for i in range(3):
        want = rot_std[i] ** 2
        assert abs(e["att_cov"][i, i] - want) < 0.05 * want


def test_random_injection_tracks_trajectory():
    # crates/pf_core/tests/cuda_agreement.rs:133-174 (inject 0.1, 20 coasting
    # steps of 0.5 m; the mean stays within 0.6 m of 0.5 (k+1))
    pf = oracle.OraclePF(4096, seed=13, ess_ratio=0.5, inject=0.1)
    pf.reinit([0, 0, 0, 1, 0, 0, 0], [0.5] * 3, [0.01] * 3)
    for k in range(20):
        est, _ = pf.update([0.5, 0, 0], [1, 0, 0, 0], [0.02] * 3, [0.005] * 3,
                           np.zeros((0, 3)), [])
        if k >= 1:
            assert abs(est["position"][0] - 0.5 * (k + 1)) < 0.6
