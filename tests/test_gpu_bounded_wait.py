"""Bounded device waits: a resampling look-back whose predecessor never
publishes gives up after its poll limit, the call reports the error instead of
hanging, and the CUDA context stays usable.

The failure is planted on the host (pfc_batch_set_wait_test): one filter's
first resampling tile publishes its prefix under a stale epoch, a flag that no
waiter accepts, and the poll limit is lowered so the waits of that filter's
later tiles run out within milliseconds.  No fault, trap or unbounded wait is
involved: a timed-out look-back returns a partial prefix (at most the true
one), so every count derived from it stays within the filter's particles."""
import ctypes as C

import numpy as np
import pytest

import cuda_pf_localization_b200 as pkg
from cuda_pf_localization_b200 import sim

pytestmark = pytest.mark.gpu

SIZES = [3000, 20000, 50000]   # filter 2 holds 13 resampling tiles of 4096
PRM = dict(sigma_r=0.05, sigma_b=0.02, gate=3.0, ess_ratio=0.5, inject=0.0)


def _setup(cycles):
    scen = [sim.helix_scenario(cycles, 16, (20.0, 20.0, 5.0), 32, 0.0, 40 + f)
            for f in range(len(SIZES))]
    b = pkg.BatchPF(SIZES, seeds=[7, 8, 9], obs_cap=4096)
    b.set_params(**PRM)
    b.set_landmarks([sc.landmarks for sc in scen])
    pose7 = np.array([np.r_[sc.prior_p, sc.prior_q] for sc in scen], np.float32)
    b.reinit(pose7, np.full((3, 3), 0.5), np.full((3, 3), 0.2))
    return b, scen


def _odom(sc, st):
    o = pkg.PfcOdom()
    o.t[:] = list(map(float, st.odom_t))
    o.q[:] = list(map(float, st.odom_q))
    o.tstd[:] = list(sc.trans_noise)
    o.rstd[:] = list(sc.rot_noise)
    return o


def _cycle(b, scen, k):
    return b.lib.pfc_batch_cycle(
        b.handle, (pkg.PfcOdom * len(SIZES))(*[_odom(sc, sc.steps[k]) for sc in scen]),
        pkg.make_cobs(np.concatenate([sc.steps[k].obs for sc in scen])),
        pkg.iptr(np.array([len(sc.steps[k].obs) for sc in scen], np.int32)),
        pkg.dptr(np.zeros((len(SIZES), pkg.PFC_EST_LEN))))


@pytest.mark.parametrize("graph", [True, False])
def test_lowered_limit_alone_does_not_fire(graph):
    b, scen = _setup(4)
    try:
        b.use_graph(graph)
        b.set_wait_test(spin_limit=1 << 16, stall_filter=-1)
        resampled = 0
        for k in range(4):
            est = b.cycle([_odom(sc, sc.steps[k]) for sc in scen],
                          [sc.steps[k].obs for sc in scen])
            resampled += int(est[2, pkg.PFC_EST_RESAMPLED])
        assert resampled > 0  # the look-backs did run
    finally:
        b.close()


@pytest.mark.parametrize("graph", [True, False])
def test_stalled_look_back_times_out_and_reports(graph):
    b, scen = _setup(6)
    try:
        b.use_graph(graph)
        b.set_wait_test(spin_limit=1 << 12, stall_filter=2)
        rcs = [_cycle(b, scen, k) for k in range(3)]
        # the first cycle in which filter 2 resamples fails, and the handle
        # keeps failing afterwards
        assert -1 in rcs
        first = rcs.index(-1)
        assert all(r == -1 for r in rcs[first:])
        assert "look-back wait timed out" in pkg.last_error()
    finally:
        b.close()
    # the context is still usable: a fresh handle and a single filter work
    b2, scen2 = _setup(2)
    try:
        est = b2.cycle([_odom(sc, sc.steps[0]) for sc in scen2],
                       [sc.steps[0].obs for sc in scen2])
        assert np.all(np.isfinite(est[:, :7]))
    finally:
        b2.close()
    lib = pkg.kernels()
    h = lib.pfc_create(64)
    try:
        assert lib.pfc_init(h, 5000, 3) == 0
        sc = scen2[0]
        lm = np.ascontiguousarray(sc.landmarks, np.float32).reshape(-1)
        assert lib.pfc_upload_landmarks(h, pkg.fptr(lm), len(sc.landmarks)) == 0
        prm = pkg.PfcCycleParams(0.05, 0.02, 3.0, 0.5, 0.0, 0)
        est = np.zeros(pkg.PFC_EST_LEN)
        st = sc.steps[0]
        assert lib.pfc_cycle(h, C.byref(_odom(sc, st)), pkg.make_cobs(st.obs), len(st.obs),
                             C.byref(prm), pkg.dptr(est)) == 0
        assert np.all(np.isfinite(est[:7]))
    finally:
        lib.pfc_destroy(h)


def test_wait_test_arguments_checked():
    b, _ = _setup(1)
    try:
        with pytest.raises(RuntimeError):
            b.set_wait_test(spin_limit=-1)
        with pytest.raises(RuntimeError):
            b.set_wait_test(stall_filter=len(SIZES))
        b.set_wait_test(0, -1)   # defaults restored
    finally:
        b.close()
