"""The reference's own filter tests, run on this library through the drop-in
path (the C++ mirror of pf_core's ParticleFilter over the pfc_* C-ABI), with
the reference's thresholds, plus tracking accuracy against the CPU oracle.

Restated: crates/pf_core/tests/cuda_agreement.rs (GPU against CPU and the
analytic prior) and crates/pf_core/tests/integration.rs (behaviour of the
filter), each cited below.
"""
import math

import numpy as np
import pytest

import cuda_pf_localization_b200 as pkg
import oracle
from cuda_pf_localization_b200 import sim

pytestmark = pytest.mark.gpu

ZERO_ODOM = pkg.make_core_odom([0, 0, 0], [1, 0, 0, 0], [0, 0, 0], [0, 0, 0])


def _estimate(pf):
    """Estimate of the current cloud: a cycle with no motion, no noise and no
    observations (weights stay uniform, no resample)."""
    return pf.update(ZERO_ODOM, [])


def test_cuda_covariances_match_gaussian_prior(kernels):
    # crates/pf_core/tests/cuda_agreement.rs:30-80: N = 200k, seed 7; CPU and
    # GPU means within 0.05; diagonal position variance within 12 % and
    # attitude variance within 15 % of the prior; off-diagonals below 10 %.
    n = 200_000
    pos_std = np.array([1.0, 2.0, 0.5])
    rot_std = np.array([0.05, 0.07, 0.02])
    pf = pkg.ParticleFilter(n, seed=7)
    try:
        pf.reinitialize([0, 0, 0, 1, 0, 0, 0], pos_std, rot_std)
        e = _estimate(pf)
    finally:
        pf.close()
    cpu = oracle.OraclePF(n, seed=7)
    cpu.reinit([0, 0, 0, 1, 0, 0, 0], pos_std, rot_std)
    c = cpu.estimate()
    assert np.all(np.abs(e["position"] - c["position"]) < 0.05)
    for i in range(3):
        want, wrot = pos_std[i] ** 2, rot_std[i] ** 2
        assert abs(e["pos_cov"][i, i] - want) < 0.12 * want
        assert abs(e["att_cov"][i, i] - wrot) < 0.15 * wrot
        for j in range(3):
            if i != j:
                assert abs(e["pos_cov"][i, j]) < 0.1 * want
                assert abs(e["att_cov"][i, j]) < 0.1 * wrot


def test_cuda_empty_obs_resets_weights_like_cpu(kernels):
    # crates/pf_core/tests/cuda_agreement.rs:82-131: an informative
    # observation drops the ESS below N/2; an empty observation set, or one
    # whose landmark is not in the map, leaves the weights uniform (> 0.95 N).
    n = 20_000
    pf = pkg.ParticleFilter(n, seed=77, resample_ess_ratio=0.0)
    try:
        pf.set_map({0: (5.0, 5.0, 1.0)})
        pf.reinitialize([5.0, 5.0, 1.0, 1, 0, 0, 0], [3.0] * 3, [0.1] * 3)
        e = pf.update(ZERO_ODOM, [(0, 0, 0.0, 0.0, 0.0, 0.0)])
        assert e["ess"] < n / 2
        e = pf.update(ZERO_ODOM, [])
        assert e["ess"] > 0.95 * n
        pf.update(ZERO_ODOM, [(0, 0, 0.0, 0.0, 0.0, 0.0)])
        e = pf.update(ZERO_ODOM, [(7, 0, 0.0, 0.0, 0.0, 0.0)])  # id 7 not in the map
        assert e["ess"] > 0.95 * n
    finally:
        pf.close()


def test_cuda_random_injection_tracks_trajectory(kernels):
    # crates/pf_core/tests/cuda_agreement.rs:133-174: inject 0.1, 20 steps of
    # 0.5 m without observations; the mean stays within 0.6 m of 0.5 (k + 1).
    pf = pkg.ParticleFilter(4096, seed=13, resample_ess_ratio=0.5, random_inject_ratio=0.1)
    try:
        pf.reinitialize([0, 0, 0, 1, 0, 0, 0], [0.5] * 3, [0.01] * 3)
        odom = pkg.make_core_odom([0.5, 0, 0], [1, 0, 0, 0], [0.02] * 3, [0.005] * 3)
        for k in range(20):
            e = pf.update(odom, [])
            if k >= 1:
                assert abs(e["position"][0] - 0.5 * (k + 1)) < 0.6
    finally:
        pf.close()


def test_cuda_tight_cloud_accuracy(kernels):
    # crates/pf_core/tests/cuda_agreement.rs:177-219: N = 100k tight cloud;
    # |ESS - N| small, attitude covariance within 5 % of sigma^2 and within
    # 2 % of the CPU's.
    n = 100_000
    rot_std = np.array([1e-3, 2e-3, 3e-3])
    pf = pkg.ParticleFilter(n, seed=7)
    try:
        pf.reinitialize([0, 0, 0, 1, 0, 0, 0], [0.01] * 3, rot_std)
        e = _estimate(pf)
    finally:
        pf.close()
    cpu = oracle.OraclePF(n, seed=7)
    cpu.reinit([0, 0, 0, 1, 0, 0, 0], [0.01] * 3, rot_std)
    c = cpu.estimate()
    assert abs(e["ess"] - n) < 0.05 * n
    for i in range(3):
        want = rot_std[i] ** 2
        assert abs(e["att_cov"][i, i] - want) < 0.05 * want
        assert abs(e["att_cov"][i, i] - c["att_cov"][i, i]) < 0.02 * c["att_cov"][i, i]


def test_converges_on_3d_trajectory(kernels):
    # crates/pf_core/tests/integration.rs:11-38 on the GPU backend: N = 4096,
    # seed 123, circle_scenario(100, 777), prior 1 m / 0.5 rad, mean error
    # below 0.25 m.
    sc = sim.circle_scenario(100, 777)
    pf = pkg.ParticleFilter(4096, seed=123, trans_noise=sc.trans_noise, rot_noise=sc.rot_noise)
    try:
        pf.set_map(sc.landmark_dict())
        pf.reinitialize(np.r_[sc.prior_p, sc.prior_q], [1.0] * 3, [0.5] * 3)
        errs = []
        for st in sc.steps:
            e = pf.update(pkg.make_core_odom(st.odom_t, st.odom_q, sc.trans_noise,
                                             sc.rot_noise), st.obs)
            errs.append(np.linalg.norm(e["position"] - st.truth_p))
    finally:
        pf.close()
    assert np.mean(errs) < 0.25, np.mean(errs)


def test_coasts_without_observations(kernels):
    # crates/pf_core/tests/integration.rs:40-68
    pf = pkg.ParticleFilter(1024, seed=5)
    try:
        pf.reinitialize([1.0, 2.0, 3.0, 1, 0, 0, 0], [0.1] * 3, [0.01] * 3)
        odom = pkg.make_core_odom([1.0, 0, 0], [1, 0, 0, 0], [0.01] * 3, [0.005] * 3)
        for _ in range(20):
            e = pf.update(odom, [])
    finally:
        pf.close()
    assert abs(e["position"][0] - 21.0) < 0.5
    assert abs(e["position"][1] - 2.0) < 0.2
    assert abs(e["position"][2] - 3.0) < 0.2


def _track(sc, n, seed, gate, inject, fused):
    pf = pkg.ParticleFilter(n, seed=seed, gate_sigma=gate, random_inject_ratio=inject,
                            trans_noise=sc.trans_noise, rot_noise=sc.rot_noise)
    try:
        pf.set_map(sc.landmark_dict())
        pf.reinitialize(np.r_[sc.prior_p, sc.prior_q], [0.5] * 3, [0.2] * 3)
        errs = []
        for st in sc.steps:
            e = pf.update(pkg.make_core_odom(st.odom_t, st.odom_q, sc.trans_noise,
                                             sc.rot_noise), st.obs, fused=fused)
            errs.append(np.linalg.norm(e["position"] - st.truth_p))
        return np.array(errs)
    finally:
        pf.close()


def _track_oracle(sc, n, seed, gate, inject):
    pf = oracle.OraclePF(n, seed=seed, range_noise=0.05, gate=gate, ess_ratio=0.5,
                         inject=inject)
    pf.reinit(np.r_[sc.prior_p, sc.prior_q], [0.5] * 3, [0.2] * 3)
    errs = []
    for st in sc.steps:
        e, _ = pf.update(st.odom_t, st.odom_q, sc.trans_noise, sc.rot_noise, sc.landmarks,
                         st.obs)
        errs.append(float(np.linalg.norm(e["position"] - st.truth_p)))
    return np.array(errs)


@pytest.mark.parametrize("fused", [False, True])
def test_tracking_config_matches_oracle_accuracy(kernels, fused):
    """Plain tracking workload (10k particles, 12 landmarks, 100 cycles,
    3-sigma gate): the mean tracking error of the GPU filter is within the
    CPU oracle's (different noise streams, same models)."""
    sc = sim.tracking_config(cycles=100, seed=7)
    gpu = _track(sc, 10_000, 3, 3.0, 0.0, fused)
    cpu = _track_oracle(sc, 10_000, 3, 3.0, 0.0)
    print(f"\ntracking config: GPU {gpu.mean():.4f} m, oracle {cpu.mean():.4f} m")
    assert gpu.mean() <= 1.5 * cpu.mean() + 0.01
    assert gpu[20:].mean() < 0.1


def test_scale_config_matches_oracle_accuracy(kernels):
    """At-scale workload (64 landmarks, 256 observations with 10 % outliers,
    injection 0.01) at 100k particles, 30 cycles."""
    sc = sim.scale_config(cycles=30, seed=11)
    gpu = _track(sc, 100_000, 3, 3.0, 0.01, True)
    cpu = _track_oracle(sc, 100_000, 3, 3.0, 0.01)
    print(f"\nscale config: GPU {gpu.mean():.4f} m, oracle {cpu.mean():.4f} m")
    assert gpu.mean() <= 1.5 * cpu.mean() + 0.01
