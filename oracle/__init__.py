"""CPU oracle bindings — TEST INFRASTRUCTURE ONLY.

Imported only by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
leg, always as the checker (or the timed CPU baseline), never as the product.

* ``lib()``      liboracle.so: the C++ restatement of the reference CPU path
                 (pf_oracle.cpp; every function cites the reference file:line
                 it follows) plus mirrors of the GPU path's deterministic specs.
* ``ref_lib()``  oracle/_ref/libpf_kernels_ref.so: the reference's own CUDA
                 library compiled from its source (GPU tests only).
"""
from __future__ import annotations

import ctypes as C
from ctypes import POINTER, c_double, c_float, c_int, c_uint, c_uint64, c_ulonglong, c_void_p
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_SO = HERE / "liboracle.so"
REF_SO = HERE / "_ref" / "libpf_kernels_ref.so"

_fp, _dp, _ip, _u8p = POINTER(c_float), POINTER(c_double), POINTER(c_int), POINTER(C.c_ubyte)
_u32p = POINTER(C.c_uint32)


class OrcObs(C.Structure):
    _fields_ = [("id", c_int), ("mode", c_int), ("v", c_double * 3), ("range", c_double)]


_SIGS = {
    "orc_philox4x32_10": (None, [_u32p, c_uint64, _u32p]),
    "orc_normals6": (None, [c_uint64, c_uint64, C.c_uint32, _dp]),
    "orc_pf_new": (c_void_p, [c_int, c_uint64, c_double, c_double, c_double, c_double, c_double]),
    "orc_pf_free": (None, [c_void_p]),
    "orc_threads": (c_int, []),
    "orc_set_threads": (None, [c_int]),
    "orc_pf_set_state": (None, [c_void_p, _dp, _dp, _dp]),
    "orc_pf_get_state": (None, [c_void_p, _dp, _dp, _dp]),
    "orc_pf_set_gen": (None, [c_void_p, c_uint64]),
    "orc_pf_set_lcg": (None, [c_void_p, c_uint64]),
    "orc_pf_reinit": (None, [c_void_p, _dp, _dp, _dp]),
    "orc_pf_predict": (None, [c_void_p, _dp, _dp, _dp, _dp]),
    "orc_loglik": (None, [c_int, _dp, _dp, _dp, c_int, POINTER(OrcObs), c_int, c_double,
                          c_double, c_double, _dp]),
    "orc_pf_weight": (c_int, [c_void_p, _dp, c_int, POINTER(OrcObs), c_int]),
    "orc_inject_draw": (None, [c_uint64, c_uint64, c_int, c_int, _ip, _fp]),
    "orc_lcg_next": (c_uint64, [c_uint64]),
    "orc_lcg_u01": (c_double, [c_uint64]),
    "orc_resample_fixed": (c_int, [_fp, c_int, c_double, _ip, _dp]),
    "orc_resample_f64": (c_int, [_dp, c_int, c_double, _ip]),
    "orc_pick_from_cum": (None, [_dp, c_int, c_double, c_double, _ip]),
    "orc_inject_apply": (None, [_fp, c_int, c_int, c_uint64, c_uint64]),
    "orc_pf_resample": (None, [c_void_p]),
    "orc_quat_mean": (None, [_dp, _dp]),
    "orc_est_sums": (None, [c_int, _fp, _fp, _fp, _dp]),
    "orc_covs": (None, [c_int, _fp, _fp, _fp, _fp, _fp, _dp]),
    "orc_pf_estimate": (None, [c_void_p, _dp]),
    "orc_pf_update": (c_int, [c_void_p, _dp, _dp, _dp, _dp, _dp, c_int, POINTER(OrcObs), c_int,
                              _dp]),
    "orc_cast_ray": (c_double, [c_int, c_int, c_double, c_double, c_double, _u8p, c_double,
                                c_double, c_double, c_double, c_double]),
    "orc_map_scan": (None, [c_int, c_int, c_double, c_double, c_double, _u8p, c_double,
                            c_double, c_double, c_int, c_double, c_double, _dp]),
    "orc_caer": (None, [c_int, c_int, c_double, c_double, c_double, _u8p, _dp, c_int, c_double,
                        c_double, _dp, c_int, _dp]),
    "orc_disperse": (None, [c_int, c_int, c_double, c_double, c_double, _u8p, c_int, c_uint64,
                            _dp]),
    "orc_gl_localize": (c_int, [c_int, c_int, c_double, c_double, c_double, _u8p, _dp, c_int,
                                c_double, c_double, c_int, c_int, c_uint64, _dp]),
    "orc_topk_from_scores": (None, [_fp, c_int, c_int, _ip]),
    "orc_cast_ray_f32": (c_float, [c_int, c_int, c_float, c_float, c_float, _u8p, c_float,
                                   c_float, c_float, c_float, c_float]),
    "orc_caer_f32": (None, [c_int, c_int, c_float, c_float, c_float, _u8p, _fp, c_int, c_float,
                            c_float, _fp, c_int, _fp]),
    "orc_gl_generate": (None, [c_int, _ip, c_float, c_float, c_float, c_int, c_int, c_uint64,
                               _fp]),
}

_lib = None
_ref = None


def lib():
    global _lib
    if _lib is None:
        if not ORACLE_SO.exists():
            raise RuntimeError(f"{ORACLE_SO} missing: run `python oracle/build.py`")
        _lib = C.CDLL(str(ORACLE_SO))
        for name, (res, args) in _SIGS.items():
            fn = getattr(_lib, name)
            fn.restype = res
            fn.argtypes = args
    return _lib


def f32(a):
    a = np.ascontiguousarray(a, dtype=np.float32)
    return a, a.ctypes.data_as(_fp)


def f64(a):
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a, a.ctypes.data_as(_dp)


def i32(a):
    a = np.ascontiguousarray(a, dtype=np.int32)
    return a, a.ctypes.data_as(_ip)


def u8(a):
    a = np.ascontiguousarray(a, dtype=np.uint8)
    return a, a.ctypes.data_as(_u8p)


def make_obs(rows) -> "C.Array":
    arr = (OrcObs * max(1, len(rows)))()
    for k, r in enumerate(rows):
        arr[k].id = int(r[0])
        arr[k].mode = int(r[1])
        arr[k].v[:] = [float(r[2]), float(r[3]), float(r[4])]
        arr[k].range = float(r[5])
    return arr


# ------------------------------------------------------------- PF helpers

def normals6(seed: int, gen: int, i: int) -> np.ndarray:
    out = np.zeros(6)
    lib().orc_normals6(seed, gen, i, out.ctypes.data_as(_dp))
    return out


def loglik(pos3, quat4, lm3, obs_rows, sr, sb, gate) -> np.ndarray:
    pos, pp = f64(pos3)
    quat, qp = f64(quat4)
    lm, lp = f64(lm3)
    n = pos.size // 3
    out = np.zeros(n)
    obs = make_obs(obs_rows)
    lib().orc_loglik(n, pp, qp, lp, lm.size // 3, obs, len(obs_rows), sr, sb, gate,
                     out.ctypes.data_as(_dp))
    return out


def resample_fixed(w_f32, u01):
    w, wp = f32(w_f32)
    anc = np.zeros(w.size, dtype=np.int32)
    tot = np.zeros(1)
    ok = lib().orc_resample_fixed(wp, w.size, u01, anc.ctypes.data_as(_ip),
                                  tot.ctypes.data_as(_dp))
    return (anc if ok else None), float(tot[0])


def resample_f64(w, u01):
    w, wp = f64(w)
    anc = np.zeros(w.size, dtype=np.int32)
    ok = lib().orc_resample_f64(wp, w.size, u01, anc.ctypes.data_as(_ip))
    return anc if ok else None


def pick_from_cum(cum, u0, total):
    cum, cp = f64(cum)
    anc = np.zeros(cum.size, dtype=np.int32)
    lib().orc_pick_from_cum(cp, cum.size, u0, total, anc.ctypes.data_as(_ip))
    return anc


def inject_apply(pos3_f32, k, lcg, gen):
    pos, pp = f32(np.array(pos3_f32, dtype=np.float32, copy=True))
    lib().orc_inject_apply(pp, pos.size // 3, k, lcg, gen)
    return pos


def lcg_next(lcg: int) -> int:
    return lib().orc_lcg_next(lcg)


def lcg_u01(lcg: int) -> float:
    return lib().orc_lcg_u01(lcg)


def est_sums(pos3_f32, quat4_f32, w_f32) -> np.ndarray:
    pos, pp = f32(pos3_f32)
    quat, qp = f32(quat4_f32)
    w, wp = f32(w_f32)
    out = np.zeros(14)
    lib().orc_est_sums(w.size, pp, qp, wp, out.ctypes.data_as(_dp))
    return out


def covs(pos3_f32, quat4_f32, w_f32, mp_f32, mq_f32) -> np.ndarray:
    pos, pp = f32(pos3_f32)
    quat, qp = f32(quat4_f32)
    w, wp = f32(w_f32)
    mp, mpp = f32(mp_f32)
    mq, mqp = f32(mq_f32)
    out = np.zeros(12)
    lib().orc_covs(w.size, pp, qp, wp, mpp, mqp, out.ctypes.data_as(_dp))
    return out


def quat_mean(m4x4) -> np.ndarray:
    m, mp = f64(np.asarray(m4x4, dtype=np.float64).reshape(16))
    q = np.zeros(4)
    lib().orc_quat_mean(mp, q.ctypes.data_as(_dp))
    return q


class OraclePF:
    """The reference CpuBackend (cpu.rs) in FP64 with the GPU noise spec."""

    def __init__(self, n, seed=42, range_noise=0.05, bearing_noise=0.02, gate=0.0,
                 ess_ratio=0.5, inject=0.0):
        self.n = n
        self._h = lib().orc_pf_new(n, seed, range_noise, bearing_noise, gate, ess_ratio, inject)

    def __del__(self):
        if getattr(self, "_h", None):
            lib().orc_pf_free(self._h)
            self._h = None

    def set_state(self, pos3, quat4, w=None):
        p, pp = f64(pos3)
        q, qp = f64(quat4)
        if w is None:
            lib().orc_pf_set_state(self._h, pp, qp, None)
        else:
            ww, wp = f64(w)
            lib().orc_pf_set_state(self._h, pp, qp, wp)

    def state(self):
        p = np.zeros(3 * self.n)
        q = np.zeros(4 * self.n)
        w = np.zeros(self.n)
        lib().orc_pf_get_state(self._h, p.ctypes.data_as(_dp), q.ctypes.data_as(_dp),
                               w.ctypes.data_as(_dp))
        return p.reshape(-1, 3), q.reshape(-1, 4), w

    def set_gen(self, g):
        lib().orc_pf_set_gen(self._h, g)

    def set_lcg(self, v):
        lib().orc_pf_set_lcg(self._h, v)

    def reinit(self, pose7, ps, rs):
        a, ap = f64(pose7)
        b, bp = f64(ps)
        c, cp = f64(rs)
        lib().orc_pf_reinit(self._h, ap, bp, cp)

    def predict(self, t, q, tn, rn):
        a, ap = f64(t)
        b, bp = f64(q)
        c, cp = f64(tn)
        d, dp = f64(rn)
        lib().orc_pf_predict(self._h, ap, bp, cp, dp)

    def weight(self, lm3, obs_rows):
        lm, lp = f64(lm3)
        valid = [r for r in obs_rows if 0 <= int(r[0]) < lm.size // 3]
        obs = make_obs(valid)
        return lib().orc_pf_weight(self._h, lp, lm.size // 3, obs, len(valid))

    def resample(self):
        lib().orc_pf_resample(self._h)

    def estimate(self) -> dict:
        out = np.zeros(26)
        lib().orc_pf_estimate(self._h, out.ctypes.data_as(_dp))
        return dict(position=out[0:3], attitude=out[3:7], pos_cov=out[7:16].reshape(3, 3),
                    att_cov=out[16:25].reshape(3, 3), ess=float(out[25]))

    def update(self, t, q, tn, rn, lm3, obs_rows) -> tuple[dict, bool]:
        a, ap = f64(t)
        b, bp = f64(q)
        c, cp = f64(tn)
        d, dp = f64(rn)
        lm, lp = f64(lm3)
        obs = make_obs(obs_rows)
        out = np.zeros(26)
        rs = lib().orc_pf_update(self._h, ap, bp, cp, dp, lp, lm.size // 3, obs, len(obs_rows),
                                 out.ctypes.data_as(_dp))
        return dict(position=out[0:3], attitude=out[3:7], pos_cov=out[7:16].reshape(3, 3),
                    att_cov=out[16:25].reshape(3, 3), ess=float(out[25])), bool(rs)


# ------------------------------------------------------------- GL helpers

def cast_ray(cells, res, origin, px, py, dx, dy, rmax) -> float:
    c, cp = u8(cells)
    h, w = c.shape
    return lib().orc_cast_ray(w, h, res, origin[0], origin[1], cp, px, py, dx, dy, rmax)


def map_scan(cells, res, origin, x, y, th, nrays, span, rmax) -> np.ndarray:
    c, cp = u8(cells)
    h, w = c.shape
    out = np.zeros(nrays)
    lib().orc_map_scan(w, h, res, origin[0], origin[1], cp, x, y, th, nrays, span, rmax,
                       out.ctypes.data_as(_dp))
    return out


def caer(cells, res, origin, scan, span, rmax, hyp3) -> np.ndarray:
    c, cp = u8(cells)
    h, w = c.shape
    s, sp = f64(scan)
    hy, hp = f64(np.asarray(hyp3, dtype=np.float64).reshape(-1))
    n = hy.size // 3
    out = np.zeros(n)
    lib().orc_caer(w, h, res, origin[0], origin[1], cp, sp, s.size, span, rmax, hp, n,
                   out.ctypes.data_as(_dp))
    return out


def dda_visits(cells, res, origin, hyp3, nrays, span) -> int:
    """DDA cell steps of every ray of the hypotheses (see orc_dda_visits)."""
    c, cp = u8(cells)
    h, w = c.shape
    hy, hp = f32(np.asarray(hyp3, dtype=np.float32).reshape(-1))
    fn = lib().orc_dda_visits
    fn.restype = C.c_longlong
    return int(fn(w, h, C.c_float(res), C.c_float(origin[0]), C.c_float(origin[1]), cp, hp,
                  hy.size // 3, nrays, C.c_float(span)))


def caer_f32(cells, res, origin, scan, span, rmax, hyp3) -> np.ndarray:
    c, cp = u8(cells)
    h, w = c.shape
    s, sp = f32(scan)
    hy, hp = f32(np.asarray(hyp3, dtype=np.float32).reshape(-1))
    n = hy.size // 3
    out = np.zeros(n, dtype=np.float32)
    lib().orc_caer_f32(w, h, res, origin[0], origin[1], cp, sp, s.size, span, rmax, hp, n,
                       out.ctypes.data_as(_fp))
    return out


def disperse(cells, res, origin, n, seed) -> np.ndarray:
    c, cp = u8(cells)
    h, w = c.shape
    out = np.zeros(3 * n)
    lib().orc_disperse(w, h, res, origin[0], origin[1], cp, n, seed, out.ctypes.data_as(_dp))
    return out.reshape(-1, 3)


def gl_localize(cells, res, origin, scan, span, rmax, nh, topk, seed) -> np.ndarray:
    c, cp = u8(cells)
    h, w = c.shape
    s, sp = f64(scan)
    out = np.zeros(4 * topk)
    k = lib().orc_gl_localize(w, h, res, origin[0], origin[1], cp, sp, s.size, span, rmax, nh,
                              topk, seed, out.ctypes.data_as(_dp))
    return out.reshape(-1, 4)[:k]


def topk_from_scores(caer_f32_arr, k) -> np.ndarray:
    s, sp = f32(caer_f32_arr)
    out = np.zeros(min(k, s.size), dtype=np.int32)
    lib().orc_topk_from_scores(sp, s.size, k, out.ctypes.data_as(_ip))
    return out


def free_list(cells) -> np.ndarray:
    ys, xs = np.nonzero(np.asarray(cells) == 0)
    order = np.argsort(ys * cells.shape[1] + xs, kind="stable")
    return np.stack([xs[order], ys[order]], axis=1).astype(np.int32)


def gl_generate(cells, res, origin, n_pos, n_yaw, seed) -> np.ndarray:
    fr = free_list(cells)
    f, fp = i32(fr.reshape(-1))
    out = np.zeros(3 * n_pos * n_yaw, dtype=np.float32)
    lib().orc_gl_generate(len(fr), fp, origin[0], origin[1], res, n_pos, n_yaw, seed,
                          out.ctypes.data_as(_fp))
    return out.reshape(-1, 3)


# --------------------------------------------- reference CUDA library (GPU)

_REF_SIGS = {
    "pfc_create": (c_void_p, [c_int]),
    "pfc_destroy": (c_int, [c_void_p]),
    "pfc_init": (c_int, [c_void_p, c_int, c_uint]),
    "pfc_upload_landmarks": (c_int, [c_void_p, _fp, c_int]),
    "pfc_reinit": (c_int, [c_void_p] + [c_float] * 7 + [_fp, _fp]),
    "pfc_predict": (c_int, [c_void_p] + [c_float] * 7 + [_fp, _fp]),
    "pfc_weight": (c_int, [c_void_p, c_void_p, c_int, c_float, c_float, c_float]),
    "pfc_resample": (c_int, [c_void_p, c_float]),
    "pfc_est_sums": (c_int, [c_void_p, _dp]),
    "pfc_covs": (c_int, [c_void_p] + [c_float] * 7 + [_dp]),
    "pfc_snapshot": (c_int, [c_void_p, _fp, _fp]),
    "pfc_device_available": (c_int, []),
    "pfgl_create": (c_void_p, [c_int, c_int, c_float, c_float, c_float, _u8p, c_int]),
    "pfgl_destroy": (c_int, [c_void_p]),
    "pfgl_free_cells": (c_int, [c_void_p]),
    "pfgl_generate": (c_int, [c_void_p, c_int, c_ulonglong]),
    "pfgl_score": (c_int, [c_void_p, _fp, c_int, c_float, c_float]),
    "pfgl_topk": (c_int, [c_void_p, c_int, _fp]),
    "ref_set_state": (c_int, [c_void_p, _fp, _fp, _fp]),
    "ref_get_w": (c_int, [c_void_p, _fp]),
    "ref_get_ll": (c_int, [c_void_p, _fp]),
    "ref_get_cum": (c_int, [c_void_p, _dp]),
    "ref_get_lcg": (c_ulonglong, [c_void_p]),
    "ref_set_lcg": (c_int, [c_void_p, c_ulonglong]),
    "ref_get_gen": (c_ulonglong, [c_void_p]),
    "ref_gl_set_hyps": (c_int, [c_void_p, _fp, c_int]),
    "ref_gl_get_hyps": (c_int, [c_void_p, _fp]),
    "ref_gl_get_caer": (c_int, [c_void_p, _fp]),
    "ref_gl_set_caer": (c_int, [c_void_p, _fp, c_int]),
    "ref_gl_get_sorted": (c_int, [c_void_p, _ip, c_int]),
}


def ref_lib():
    """The reference library built from its own source (GPU tests only)."""
    global _ref
    if _ref is None:
        if not REF_SO.exists():
            return None
        _ref = C.CDLL(str(REF_SO), mode=C.RTLD_LOCAL)
        for name, (res, args) in _REF_SIGS.items():
            fn = getattr(_ref, name)
            fn.restype = res
            fn.argtypes = args
    return _ref
