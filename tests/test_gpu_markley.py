"""The device Markley mean of the fused cycle against the host solve of the
same moments (crates/pf_core/src/types.rs:118-143 semantics), for a clustered
attitude cloud (the warp-parallel repeated-squaring path) and for uniformly
random attitudes (a near-degenerate spectrum, which the warp path hands to
the serial Jacobi fallback when its residual check fails).

The cycle runs with zero odometry and no observations, so the cloud it
estimates is the one set here with uniform weights 1/n (f32); the oracle's
FP64 sums of that cloud feed the host solve."""
import ctypes as C

import numpy as np
import pytest

import cuda_pf_localization_b200 as pkg
import oracle
from tests.pf_helpers import RawPF, cloud, ours_set_state

pytestmark = pytest.mark.gpu


def _random_quats(n, seed):
    q = np.random.default_rng(seed).normal(size=(n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    return q.astype(np.float32)


@pytest.mark.parametrize("kind", ["clustered", "isotropic"])
def test_device_markley_equals_host(kernels, kind):
    n = 200_003
    pos, quat = cloud(n, 5, centre=(1.0, -2.0, 0.5), pos_std=0.3, rot_std=0.1, yaw=0.7)
    if kind == "isotropic":
        quat = _random_quats(n, 6)
    pf = RawPF(kernels, n, seed=3)
    try:
        ours_set_state(pf, pos, quat)
        odom = pkg.PfcOdom()
        odom.t[:] = [0.0, 0.0, 0.0]
        odom.q[:] = [1.0, 0.0, 0.0, 0.0]
        odom.tstd[:] = [0.0] * 3
        odom.rstd[:] = [0.0] * 3
        prm = pkg.PfcCycleParams(0.05, 0.02, 3.0, 0.5, 0.0, 0)
        est = np.zeros(pkg.PFC_EST_LEN)
        assert kernels.pfc_cycle(pf.h, C.byref(odom), None, 0, C.byref(prm), pkg.dptr(est)) == 0
        p1, q1 = pf.snapshot()
        np.testing.assert_array_equal(p1.reshape(-1, 3), pos)
        np.testing.assert_array_equal(q1.reshape(-1, 4), quat)
    finally:
        pf.close()
    w = np.full(n, np.float32(1.0) / np.float32(n), np.float32)
    sums = oracle.est_sums(pos, quat, w)
    qh = np.zeros(4)
    pkg.core().pfcore_quat_mean(pkg.dptr(np.ascontiguousarray(sums[3:13])), pkg.dptr(qh))
    qd = est[pkg.PFC_EST_QUAT:pkg.PFC_EST_QUAT + 4]
    assert abs(np.linalg.norm(qd) - 1.0) < 1e-12
    assert qd[0] >= 0.0
    if kind == "clustered":
        assert np.max(np.abs(qd - qh)) < 1e-9, (qd, qh)
    else:
        # a near-degenerate top eigenvalue: any unit vector of the top
        # eigenspace is a solution, so compare the Rayleigh quotients
        m = np.zeros((4, 4))
        e = 3
        for r in range(4):
            for c in range(r, 4):
                m[r, c] = m[c, r] = sums[e]
                e += 1
        lam = np.linalg.eigvalsh(m)[-1]
        assert abs(qd @ m @ qd - lam) <= 1e-9 * lam
        assert abs(qh @ m @ qh - lam) <= 1e-9 * lam
    np.testing.assert_allclose(est[pkg.PFC_EST_POS:pkg.PFC_EST_POS + 3], sums[:3], rtol=1e-9)
