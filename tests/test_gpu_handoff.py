"""Global-localization -> particle-filter hand-off on the device: the PF is
reseeded around the CBGL bottom-k without copying the winners to the host.
"""
import ctypes as C
import math

import numpy as np
import pytest

import cuda_pf_localization_b200 as pkg
import oracle
from cuda_pf_localization_b200 import sim
from pf_helpers import RawPF

pytestmark = pytest.mark.gpu


def _localize(lib, g, truth, k):
    gh = lib.pfgl_create(200, 200, 0.05, 0.0, 0.0, pkg.u8ptr(np.ascontiguousarray(g)), 200_000)
    assert gh
    scan = pkg.render_scans(gh, np.array([truth], np.float32), noise=0.01, seed=4)[0]
    assert lib.pfgl_generate_yaws(gh, 12_500, 16, 3) == 0
    out = np.zeros(3 * k, np.float32)
    assert lib.pfgl_localize(gh, pkg.fptr(scan), 360, 10.0, 2 * math.pi, k, pkg.fptr(out),
                             None, None) == k
    return gh, out.reshape(k, 3)


def test_topk_device_pointer_holds_last_bottom_k(kernels):
    """The device poses equal the host bottom-k: a noise-free hand-off puts
    particle i exactly on winner i mod k."""
    lib = pkg.kernels()
    g = sim.rooms_grid(5)
    truth = sim.free_pose(g, np.random.default_rng(1))
    k = 8
    gh, top = _localize(lib, g, truth, k)
    pf = RawPF(kernels, 64, seed=3)
    try:
        kk = C.c_int(0)
        ptr = lib.pfgl_topk_device(gh, C.byref(kk))
        assert ptr and kk.value == k
        assert lib.pfgl_topk_device(gh, None) == ptr
        zero = np.zeros(3, np.float32)
        assert lib.pfc_reinit_poses(pf.h, C.c_void_p(ptr), k, 0.5, pkg.fptr(zero),
                                    pkg.fptr(zero)) == 0
        pos, quat = pf.snapshot()
        pos = pos.reshape(-1, 3)
        quat = quat.reshape(-1, 4)
        idx = np.arange(64) % k
        assert np.array_equal(pos[:, 0], top[idx, 0])
        assert np.array_equal(pos[:, 1], top[idx, 1])
        assert np.all(pos[:, 2] == np.float32(0.5))
        yaw = 2 * np.arctan2(quat[:, 3], quat[:, 0])
        dyaw = (yaw - top[idx, 2] + np.pi) % (2 * np.pi) - np.pi
        assert np.max(np.abs(dyaw)) < 1e-5
        assert math.hypot(top[0, 0] - truth[0], top[0, 1] - truth[1]) <= 0.5
    finally:
        pf.close()
        lib.pfgl_destroy(gh)


def test_reinit_from_gl_matches_oracle_prior(kernels):
    """Particle i starts from winner i mod k: identical to the oracle's
    Gaussian prior around that winner with the same Philox noise."""
    lib = pkg.kernels()
    g = sim.rooms_grid(6)
    truth = sim.free_pose(g, np.random.default_rng(2))
    k, n, seed, z = 8, 20_000, 13, 1.25
    gh, top = _localize(lib, g, truth, k)
    pf = RawPF(kernels, n, seed=seed)
    try:
        kk = C.c_int(0)
        ptr = lib.pfgl_topk_device(gh, C.byref(kk))
        assert kk.value == k
        ps = np.float32([0.05, 0.08, 0.02])
        rs = np.float32([0.01, 0.02, 0.05])
        assert lib.pfc_reinit_poses(pf.h, C.c_void_p(ptr), k, z, pkg.fptr(ps),
                                    pkg.fptr(rs)) == 0
        pos, quat = pf.snapshot()
        pos = pos.reshape(-1, 3)
        quat = quat.reshape(-1, 4)
        for j in range(k):
            x, y, yaw = (float(v) for v in top[j])
            h = np.float32(0.5) * np.float32(yaw)
            pose = np.array([x, y, z, math.cos(h), 0.0, 0.0, math.sin(h)])
            orc = oracle.OraclePF(n, seed=seed)
            orc.reinit(np.float32(pose).astype(np.float64), ps.astype(np.float64),
                       rs.astype(np.float64))
            op, oq, _ = orc.state()
            sel = np.arange(j, n, k)
            assert np.max(np.abs(pos[sel] - op[sel])) < 2e-5
            assert np.max(np.abs(quat[sel] - oq[sel])) < 2e-6
        # weights uniform after the hand-off
        w = np.zeros(n, np.float32)
        assert kernels.pfc_get_weights(pf.h, pkg.fptr(w)) == 0
        assert np.allclose(w, 1.0 / n)
    finally:
        pf.close()
        lib.pfgl_destroy(gh)


def test_handoff_then_tracking_converges(kernels):
    """GL on a room, hand-off, then Cartesian landmark updates: the filter
    tracks the true pose."""
    lib = pkg.kernels()
    g = sim.rooms_grid(7)
    rng = np.random.default_rng(3)
    truth = sim.free_pose(g, rng)
    k, n = 16, 50_000
    gh, _ = _localize(lib, g, truth, k)
    pf = RawPF(kernels, n, seed=21)
    try:
        ptr = lib.pfgl_topk_device(gh, None)
        ps = np.float32([0.1, 0.1, 0.05])
        rs = np.float32([0.01, 0.01, 0.05])
        assert lib.pfc_reinit_poses(pf.h, C.c_void_p(ptr), k, 0.0, pkg.fptr(ps),
                                    pkg.fptr(rs)) == 0
        lms = np.array([[1, 1, 0.5], [9, 1, 1.0], [1, 9, 0.3], [9, 9, 1.5], [5, 5, 2.0]],
                       np.float32)
        assert kernels.pfc_upload_landmarks(pf.h, pkg.fptr(lms.reshape(-1)), len(lms)) == 0
        x, y, yaw = truth
        c, s = math.cos(yaw), math.sin(yaw)
        for _ in range(10):
            pf.predict([0.0, 0.0, 0.0], [1.0, 0.0, 0.0, 0.0], [0.03, 0.03, 0.01],
                       [0.005, 0.005, 0.01])
            rows = []
            for i, l in enumerate(lms):
                d = l - np.array([x, y, 0.0])
                body = np.array([c * d[0] + s * d[1], -s * d[0] + c * d[1], d[2]])
                body = body + rng.normal(0, 0.05, 3)
                rows.append([i, 0, *body, 0.0])
            obs = pkg.make_cobs(np.array(rows))
            assert kernels.pfc_weight(pf.h, obs, len(rows), 0.05, 0.02, 3.0) == 0
            assert kernels.pfc_resample(pf.h, 0.0) == 0
        sums = np.zeros(14)
        assert kernels.pfc_est_sums(pf.h, pkg.dptr(sums)) == 0
        assert math.hypot(sums[0] - x, sums[1] - y) < 0.1
    finally:
        pf.close()
        lib.pfgl_destroy(gh)
