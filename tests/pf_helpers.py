"""Shared helpers for the GPU tests: thin drivers of the raw pfc_* ABI of this
project's library and of the reference library (oracle/_ref), and seeded
synthetic particle clouds."""
from __future__ import annotations

import ctypes as C

import numpy as np

import cuda_pf_localization_b200 as pkg
from cuda_pf_localization_b200 import sim


def f32p(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def f64p(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def i32p(a):
    return a.ctypes.data_as(C.POINTER(C.c_int))


class RawPF:
    """Direct pfc_* driver for one library (ours or the reference)."""

    def __init__(self, lib, n, seed=42, cap_obs=256):
        self.lib = lib
        self.n = n
        self.h = lib.pfc_create(cap_obs)
        assert self.h, "pfc_create failed"
        assert lib.pfc_init(self.h, n, seed) == 0

    def close(self):
        if self.h:
            self.lib.pfc_destroy(self.h)
            self.h = None

    def landmarks(self, lm):
        a = np.ascontiguousarray(lm, dtype=np.float32).reshape(-1)
        assert self.lib.pfc_upload_landmarks(self.h, f32p(a), a.size // 3) == 0

    def weight(self, obs_rows, sr=0.05, sb=0.02, gate=3.0):
        arr = pkg.make_cobs(obs_rows)
        return self.lib.pfc_weight(self.h, C.cast(arr, C.c_void_p) if self.lib is not pkg.kernels()
                                   else arr, len(obs_rows), sr, sb, gate)

    def reinit(self, pose7, ps, rs):
        ps = np.asarray(ps, np.float32)
        rs = np.asarray(rs, np.float32)
        assert self.lib.pfc_reinit(self.h, *map(float, pose7), f32p(ps), f32p(rs)) == 0

    def predict(self, t, q, tn, rn):
        tn = np.asarray(tn, np.float32)
        rn = np.asarray(rn, np.float32)
        assert self.lib.pfc_predict(self.h, *map(float, t), *map(float, q), f32p(tn),
                                    f32p(rn)) == 0

    def est_sums(self):
        out = np.zeros(14)
        assert self.lib.pfc_est_sums(self.h, f64p(out)) == 0
        return out

    def covs(self, mp, mq):
        out = np.zeros(12)
        assert self.lib.pfc_covs(self.h, *map(float, mp), *map(float, mq), f64p(out)) == 0
        return out

    def snapshot(self):
        pos = np.zeros(3 * self.n, np.float32)
        quat = np.zeros(4 * self.n, np.float32)
        assert self.lib.pfc_snapshot(self.h, f32p(pos), f32p(quat)) == 0
        return pos, quat

    def resample(self, inject=0.0):
        assert self.lib.pfc_resample(self.h, inject) == 0


def ours_set_state(pf: RawPF, pos, quat, w=None):
    lib = pf.lib
    pos = np.ascontiguousarray(pos, np.float32).reshape(-1)
    quat = np.ascontiguousarray(quat, np.float32).reshape(-1)
    wp = None
    if w is not None:
        w = np.ascontiguousarray(w, np.float32)
        wp = f32p(w)
    assert lib.pfc_set_state(pf.h, f32p(pos), f32p(quat), wp) == 0


def ours_weights(pf: RawPF):
    w = np.zeros(pf.n, np.float32)
    assert pf.lib.pfc_get_weights(pf.h, f32p(w)) == 0
    return w


def ours_ll(pf: RawPF):
    ll = np.zeros(pf.n, np.float32)
    assert pf.lib.pfc_get_ll(pf.h, f32p(ll)) == 0
    return ll


def ref_set_state(ref, pf: RawPF, pos, quat, w=None):
    pos = np.ascontiguousarray(pos, np.float32).reshape(-1)
    quat = np.ascontiguousarray(quat, np.float32).reshape(-1)
    wp = f32p(np.ascontiguousarray(w, np.float32)) if w is not None else None
    assert ref.ref_set_state(pf.h, f32p(pos), f32p(quat), wp) == 0


def ref_weights(ref, pf: RawPF):
    w = np.zeros(pf.n, np.float32)
    assert ref.ref_get_w(pf.h, f32p(w)) == 0
    return w


def ref_ll(ref, pf: RawPF):
    ll = np.zeros(pf.n, np.float32)
    assert ref.ref_get_ll(pf.h, f32p(ll)) == 0
    return ll


def cloud(n, seed, centre=(0.0, 0.0, 0.0), pos_std=0.5, rot_std=0.2, yaw=0.3):
    """Seeded f32 cloud: Gaussian positions, quaternions = yaw * small noise,
    each quaternion normalised in f64 then rounded to f32."""
    rng = np.random.default_rng(seed)
    pos = (np.asarray(centre) + rng.normal(scale=pos_std, size=(n, 3))).astype(np.float32)
    base = sim.q_yaw(yaw)
    ax = rng.normal(scale=rot_std, size=(n, 3))
    ang = np.linalg.norm(ax, axis=1)
    half = 0.5 * ang
    s = np.where(ang > 1e-12, np.sin(half) / np.maximum(ang, 1e-300), 0.5)
    dq = np.concatenate([np.cos(half)[:, None], ax * s[:, None]], axis=1)
    q = np.stack([sim.qmul(base, d) for d in dq]) if n <= 20000 else _qmul_batch(base, dq)
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    return pos, q.astype(np.float32)


def _qmul_batch(a, b):
    aw, ax, ay, az = a
    bw, bx, by, bz = b.T
    return np.stack([aw * bw - ax * bx - ay * by - az * bz,
                     aw * bx + ax * bw + ay * bz - az * by,
                     aw * by - ax * bz + ay * bw + az * bx,
                     aw * bz + ax * by - ay * bx + az * bw], axis=1)


def scale_obs(seed=11, step=0):
    """Landmarks and one cycle of the at-scale workload (64 landmarks in a
    50 x 50 x 10 m box, 256 observations, 10 % outliers)."""
    sc = sim.helix_scenario(step + 1, 64, (50.0, 50.0, 10.0), 256, 0.10, seed)
    st = sc.steps[step]
    return sc.landmarks, st.obs, st.truth_p, st.truth_q


def rel_close(a, b, rtol, atol=0.0):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.abs(a - b) <= rtol * np.abs(b) + atol
