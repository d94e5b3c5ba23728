"""The fused cycle replayed from a CUDA graph gives the same bits as the same
cycle launched kernel by kernel: estimates, resampling decisions and every
particle, through parameter changes (re-capture), cycles without
observations (direct path) and the device-input entry point."""
import ctypes as C

import numpy as np
import pytest

import cuda_pf_localization_b200 as pkg
from cuda_pf_localization_b200 import sim

pytestmark = pytest.mark.gpu


def _run(lib, graph, sc, n, device_obs=False):
    h = lib.pfc_create(256)
    assert h
    try:
        assert lib.pfc_set_graph(h, 1 if graph else 0) == 0
        assert lib.pfc_init(h, n, 17) == 0
        lm = np.ascontiguousarray(sc.landmarks, np.float32).reshape(-1)
        assert lib.pfc_upload_landmarks(h, pkg.fptr(lm), len(sc.landmarks)) == 0
        pri = np.r_[sc.prior_p, sc.prior_q].astype(np.float32)
        ps, rs = np.full(3, 0.5, np.float32), np.full(3, 0.2, np.float32)
        assert lib.pfc_reinit(h, *map(float, pri), pkg.fptr(ps), pkg.fptr(rs)) == 0
        ests = []
        d_obs = None
        if device_obs:
            import torch
            recs = [pkg.cobs_records(st.obs) for st in sc.steps]
            d_obs = [torch.from_numpy(r.view(np.uint8).copy()).cuda() for r in recs]
        for k, st in enumerate(sc.steps):
            prm = pkg.PfcCycleParams(0.05, 0.02, 3.0 if k < 6 else 2.5, 0.5,
                                     0.01 if k % 4 else 0.02, 0)
            odom = pkg.PfcOdom()
            odom.t[:] = list(map(float, st.odom_t))
            odom.q[:] = list(map(float, st.odom_q))
            odom.tstd[:] = list(sc.trans_noise)
            odom.rstd[:] = list(sc.rot_noise)
            nobs = 0 if k == 3 else len(st.obs)
            est = np.zeros(pkg.PFC_EST_LEN)
            if device_obs:
                assert lib.pfc_cycle_device(h, C.byref(odom), C.c_void_p(d_obs[k].data_ptr()),
                                            nobs, C.byref(prm), pkg.dptr(est)) == 0
            else:
                obs = pkg.make_cobs(st.obs)
                assert lib.pfc_cycle(h, C.byref(odom), obs, nobs, C.byref(prm),
                                     pkg.dptr(est)) == 0
            ests.append(est)
        pos = np.zeros(3 * n, np.float32)
        quat = np.zeros(4 * n, np.float32)
        assert lib.pfc_snapshot(h, pkg.fptr(pos), pkg.fptr(quat)) == 0
        stats = pkg.PfcStats()
        lib.pfc_get_stats(h, C.byref(stats))
        return np.array(ests), pos, quat, int(stats.launches)
    finally:
        lib.pfc_destroy(h)


@pytest.mark.parametrize("device_obs", [False, True])
def test_graph_cycle_equals_direct(kernels, device_obs):
    sc = sim.scale_config(cycles=12, seed=11)
    n = 100_000
    e0, p0, q0, l0 = _run(kernels, False, sc, n, device_obs)
    e1, p1, q1, l1 = _run(kernels, True, sc, n, device_obs)
    assert np.array_equal(e0, e1)
    assert np.array_equal(p0, p1) and np.array_equal(q0, q1)
    assert e0[:, pkg.PFC_EST_RESAMPLED].sum() > 0
    assert l1 == l0  # a replayed graph counts the kernels it runs
