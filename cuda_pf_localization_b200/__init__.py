"""B200-native particle-filter localization and CBGL global localization.

The product is the shared library ``libpf_kernels.so`` (hand-written sm_100a
CUDA behind the reference's ``pfc_*`` / ``pfgl_*`` C-ABI, declared in
``include/pfc_abi.h``) and ``libpf_core.so`` (the C++ host layer that drives
it the way the reference's Rust ``pf_core`` does, ``include/pf_core.h``).
This package loads both with ctypes and exposes thin Python views of them.

Nothing here computes on the CPU: every call goes through the CUDA library,
and importing the bindings fails loudly when the library is missing.
"""
from __future__ import annotations

import ctypes as C
from ctypes import POINTER, byref, c_double, c_float, c_int, c_uint, c_ulonglong, c_void_p
from pathlib import Path

import numpy as np

PKG_DIR = Path(__file__).resolve().parent
KERNELS_SO = PKG_DIR / "libpf_kernels.so"
CORE_SO = PKG_DIR / "libpf_core.so"

__all__ = [
    "CObservation", "PfcOdom", "PfcCycleParams", "PfcoreConfig", "PfcoreObservation",
    "PfcoreOdom", "PfcoreEstimate", "PfcoreGlParams", "PfcorePoseHypothesis",
    "kernels", "core", "ParticleFilter", "GlobalLoc", "PFC_EST_LEN", "PF_ABI_SYMBOLS",
]

PFC_EST_LEN = 24
PFC_EST = dict(POS=0, QUAT=3, POSCOV=7, ATTCOV=13, ESS=19, RESAMPLED=20, ESS_PRE=21)
PFC_EST_POS, PFC_EST_QUAT, PFC_EST_POSCOV, PFC_EST_ATTCOV = 0, 3, 7, 13
PFC_EST_ESS, PFC_EST_RESAMPLED, PFC_EST_ESS_PRE = 19, 20, 21

# The 18 drop-in symbols the reference's Rust crate binds
# (crates/pf_core/src/cuda.rs:33-88, crates/pf_core/src/global_loc.rs:261-271).
PF_ABI_SYMBOLS = (
    "pfc_create", "pfc_destroy", "pfc_init", "pfc_upload_landmarks", "pfc_reinit",
    "pfc_predict", "pfc_weight", "pfc_resample", "pfc_est_sums", "pfc_covs",
    "pfc_snapshot", "pfc_device_available", "pfgl_create", "pfgl_destroy",
    "pfgl_free_cells", "pfgl_generate", "pfgl_score", "pfgl_topk",
)


class CObservation(C.Structure):
    _fields_ = [("id", c_int), ("mode", c_int), ("dx", c_float), ("dy", c_float),
                ("dz", c_float), ("range", c_float)]


class PfcOdom(C.Structure):
    _fields_ = [("t", c_float * 3), ("q", c_float * 4), ("tstd", c_float * 3),
                ("rstd", c_float * 3)]


class PfcCycleParams(C.Structure):
    _fields_ = [("sigma_r", c_float), ("sigma_b", c_float), ("gate", c_float),
                ("resample_ess_ratio", c_double), ("random_inject_ratio", c_float),
                ("reserved", c_int)]


class PfcStats(C.Structure):
    _fields_ = [("launches", c_ulonglong), ("h2d_bytes", c_ulonglong),
                ("d2h_bytes", c_ulonglong), ("host_syncs", c_ulonglong)]


PFC_KERNEL_KINDS = ("reinit", "predict", "weight", "est", "covs", "scan", "gather",
                    "inject", "commit", "misc")


class PfcoreConfig(C.Structure):
    _fields_ = [("particle_count", c_int), ("trans_noise", c_double * 3),
                ("rot_noise", c_double * 3), ("range_noise", c_double),
                ("bearing_noise", c_double), ("resample_ess_ratio", c_double),
                ("random_inject_ratio", c_double), ("gate_sigma", c_double),
                ("seed", c_ulonglong)]


class PfcoreObservation(C.Structure):
    _fields_ = [("landmark_id", c_int), ("mode", c_int), ("vector", c_double * 3),
                ("range", c_double)]


class PfcoreOdom(C.Structure):
    _fields_ = [("translation", c_double * 3), ("rotation", c_double * 4),
                ("trans_noise", c_double * 3), ("rot_noise", c_double * 3)]


class PfcoreEstimate(C.Structure):
    _fields_ = [("position", c_double * 3), ("attitude", c_double * 4),
                ("pos_cov", c_double * 9), ("att_cov", c_double * 9), ("ess", c_double),
                ("valid", c_int), ("resampled", c_int)]


class PfcoreGlParams(C.Structure):
    _fields_ = [("hypotheses", c_int), ("rays", c_int), ("rmax", c_double),
                ("ang_span", c_double), ("topk", c_int), ("seed", c_ulonglong)]


class PfcorePoseHypothesis(C.Structure):
    _fields_ = [("x", c_double), ("y", c_double), ("theta", c_double), ("caer", c_double)]


assert C.sizeof(CObservation) == 24  # repr(C) layout of cuda.rs:18-27

_fp = POINTER(c_float)
_dp = POINTER(c_double)
_ip = POINTER(c_int)
_u8p = POINTER(C.c_ubyte)

_KERNEL_SIGS = {
    "pfc_create": (c_void_p, [c_int]),
    "pfc_destroy": (c_int, [c_void_p]),
    "pfc_init": (c_int, [c_void_p, c_int, c_uint]),
    "pfc_upload_landmarks": (c_int, [c_void_p, _fp, c_int]),
    "pfc_reinit": (c_int, [c_void_p] + [c_float] * 7 + [_fp, _fp]),
    "pfc_predict": (c_int, [c_void_p] + [c_float] * 7 + [_fp, _fp]),
    "pfc_weight": (c_int, [c_void_p, POINTER(CObservation), c_int, c_float, c_float, c_float]),
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
    "pfc_last_error_message": (C.c_char_p, []),
    "pfc_version": (c_int, []),
    "pfc_cycle": (c_int, [c_void_p, POINTER(PfcOdom), POINTER(CObservation), c_int,
                          POINTER(PfcCycleParams), _dp]),
    "pfc_cycle_device": (c_int, [c_void_p, POINTER(PfcOdom), c_void_p, c_int,
                                 POINTER(PfcCycleParams), _dp]),
    "pfc_cycle_result": (c_int, [c_void_p, _dp]),
    "pfc_set_graph": (c_int, [c_void_p, c_int]),
    "pfc_shard_init": (c_int, [c_void_p, c_int, c_int, c_int, c_uint]),
    "pfc_shard_layout": (c_int, [c_void_p, _ip, _ip]),
    "pfc_shard_weight": (c_int, [c_void_p, POINTER(PfcOdom), c_void_p, c_int,
                                 POINTER(PfcCycleParams)]),
    "pfc_shard_views": (c_int, [c_void_p, POINTER(c_void_p), POINTER(c_void_p),
                                POINTER(c_void_p)]),
    "pfc_shard_finish": (c_int, [c_void_p, POINTER(PfcCycleParams), _dp]),
    "pfc_stream": (c_void_p, [c_void_p]),
    "pfc_size": (c_int, [c_void_p]),
    "pfc_get_weights": (c_int, [c_void_p, _fp]),
    "pfc_get_ll": (c_int, [c_void_p, _fp]),
    "pfc_set_state": (c_int, [c_void_p, _fp, _fp, _fp]),
    "pfc_resample_u01": (c_int, [c_void_p, c_double, c_float]),
    "pfc_record_ancestors": (c_int, [c_void_p, c_int]),
    "pfc_get_ancestors": (c_int, [c_void_p, _ip]),
    "pfc_pick_from_cum": (c_int, [c_void_p, _dp, c_int, c_double, c_double, _ip]),
    "pfc_weight_div_check": (c_int, [c_void_p, _fp, _fp, c_int, _fp, _fp]),
    "pfc_set_ess_hint": (c_int, [c_void_p, c_double]),
    "pfc_est_ess": (c_int, [c_void_p, _dp]),
    "pfc_get_lcg": (c_int, [c_void_p, POINTER(c_ulonglong)]),
    "pfc_set_lcg": (c_int, [c_void_p, c_ulonglong]),
    "pfc_set_weight_kernel": (c_int, [c_void_p, c_int]),
    "pfc_get_stats": (c_int, [c_void_p, POINTER(PfcStats)]),
    "pfc_reset_stats": (c_int, [c_void_p]),
    "pfc_profile": (c_int, [c_void_p, c_int]),
    "pfc_profile_read": (c_int, [c_void_p, _dp, POINTER(C.c_longlong)]),
    "pfgl_generate_yaws": (c_int, [c_void_p, c_int, c_int, c_ulonglong]),
    "pfgl_generate_yaws_range": (c_int, [c_void_p, c_int, c_int, c_int, c_ulonglong]),
    "pfgl_set_hyps": (c_int, [c_void_p, _fp, c_int]),
    "pfgl_get_hyps": (c_int, [c_void_p, _fp]),
    "pfgl_get_caer": (c_int, [c_void_p, _fp]),
    "pfgl_count_visits": (C.c_longlong, [c_void_p, c_int, c_float]),
    "pfgl_topk_ex": (c_int, [c_void_p, c_int, _fp, _fp, _ip]),
    "pfgl_topk_from_scores": (c_int, [c_void_p, _fp, c_int, c_int, _ip]),
    "pfgl_select_from_scores": (c_int, [c_void_p, _fp, c_int, c_int, c_int, _ip]),
    "pfgl_localize": (c_int, [c_void_p, _fp, c_int, c_float, c_float, c_int, _fp, _fp, _ip]),
    "pfgl_cell": (c_int, [c_void_p, c_int, c_int]),
    "pfc_reinit_poses": (c_int, [c_void_p, c_void_p, c_int, c_float, _fp, _fp]),
    "pfgl_topk_device": (c_void_p, [c_void_p, _ip]),
    "pfc_batch_create": (c_void_p, [c_int, _ip, POINTER(c_uint), c_int]),
    "pfc_batch_destroy": (c_int, [c_void_p]),
    "pfc_batch_set_params": (c_int, [c_void_p, POINTER(PfcCycleParams)]),
    "pfc_batch_upload_landmarks": (c_int, [c_void_p, _fp, _ip]),
    "pfc_batch_reinit": (c_int, [c_void_p, _fp, _fp, _fp]),
    "pfc_batch_cycle": (c_int, [c_void_p, POINTER(PfcOdom), POINTER(CObservation), _ip, _dp]),
    "pfc_batch_cycle_device": (c_int, [c_void_p, c_void_p, c_void_p, c_int, _dp]),
    "pfc_batch_result": (c_int, [c_void_p, _dp]),
    "pfc_batch_use_graph": (c_int, [c_void_p, c_int]),
    "pfc_batch_set_tiles": (c_int, [c_void_p, _ip, c_int]),
    "pfc_batch_get_tiles": (c_int, [c_void_p, _ip, _ip]),
    "pfc_batch_autotune": (c_int, [c_void_p, c_int, _ip, _ip]),
    "pfc_batch_snapshot": (c_int, [c_void_p, c_int, _fp, _fp]),
    "pfc_batch_get_weights": (c_int, [c_void_p, c_int, _fp]),
    "pfc_batch_size": (c_int, [c_void_p, c_int]),
    "pfc_batch_stream": (c_void_p, [c_void_p]),
    "pfc_batch_launches": (C.c_longlong, [c_void_p]),
    "pfc_batch_set_wait_test": (c_int, [c_void_p, c_int, c_int]),
    "pfgl_learned_create": (c_void_p, [c_void_p, c_int, c_ulonglong]),
    "pfgl_learned_destroy": (c_int, [c_void_p]),
    "pfgl_learned_num_params": (C.c_longlong, []),
    "pfgl_learned_get_params": (c_int, [c_void_p, _fp]),
    "pfgl_learned_set_params": (c_int, [c_void_p, _fp]),
    "pfgl_render_scans": (c_int, [c_void_p, _fp, c_int, c_int, c_float, c_float, c_float,
                                  c_ulonglong, _fp]),
    "pfgl_learned_make_data": (c_int, [c_void_p, C.c_longlong, c_int, c_float, c_float,
                                       c_float, c_ulonglong]),
    "pfgl_learned_train": (c_int, [c_void_p, c_int, c_int, c_float, _fp]),
    "pfgl_learned_grad": (c_int, [c_void_p, _fp, _fp, _fp, _fp]),
    "pfgl_learned_forward": (c_int, [c_void_p, _fp, c_int, _fp]),
    "pfgl_learned_norm": (c_int, [c_void_p, _fp]),
    "pfgl_learned_localize": (c_int, [c_void_p, _fp, c_int, c_float, c_float, c_int, c_int,
                                      c_int, _fp, _fp, _ip, _ip]),
    "pfgl_learned_localize_batch": (c_int, [c_void_p, _fp, c_int, c_int, c_float, c_float,
                                            c_int, c_int, c_int, _fp, _fp, _ip, _ip]),
    "pfgl_localize_batch": (c_int, [c_void_p, _fp, c_int, c_int, c_float, c_float, c_int,
                                    c_int, POINTER(c_ulonglong), c_int, _fp, _fp, _ip]),
    "pfgl_learned_calibrate": (c_int, [c_void_p, c_int, c_int, c_float, c_float, c_float,
                                       c_int, c_float, c_ulonglong, _fp, _fp]),
    "pfgl_learned_set_threshold": (c_int, [c_void_p, c_float]),
    "pfgl_learned_set_graph": (c_int, [c_void_p, c_int]),
    "pfgl_learned_gemm": (c_int, [c_int, c_int, c_int, POINTER(C.c_ushort),
                                  POINTER(C.c_ushort), _fp]),
}

_CORE_SIGS = {
    "pfcore_config_default": (None, [POINTER(PfcoreConfig)]),
    "pfcore_filter_new": (c_void_p, [POINTER(PfcoreConfig)]),
    "pfcore_filter_free": (None, [c_void_p]),
    "pfcore_map_add": (c_int, [c_void_p, c_int, c_double, c_double, c_double]),
    "pfcore_map_clear": (c_int, [c_void_p]),
    "pfcore_map_load_text": (c_int, [c_void_p, C.c_char_p]),
    "pfcore_map_capacity": (c_int, [c_void_p]),
    "pfcore_landmarks_new": (c_void_p, []),
    "pfcore_landmarks_free": (None, [c_void_p]),
    "pfcore_landmarks_add": (c_int, [c_void_p, c_int, c_double, c_double, c_double]),
    "pfcore_landmarks_has": (c_int, [c_void_p, c_int]),
    "pfcore_landmarks_at": (c_int, [c_void_p, c_int, _dp]),
    "pfcore_landmarks_capacity": (c_int, [c_void_p]),
    "pfcore_landmarks_len_defined": (c_int, [c_void_p]),
    "pfcore_landmarks_load_text": (c_int, [c_void_p, C.c_char_p]),
    "pfcore_filter_set_map": (c_int, [c_void_p, c_void_p]),
    "pfcore_filter_reinitialize": (c_int, [c_void_p, _dp, _dp, _dp]),
    "pfcore_filter_update": (c_int, [c_void_p, POINTER(PfcoreOdom),
                                     POINTER(PfcoreObservation), c_int,
                                     POINTER(PfcoreEstimate)]),
    "pfcore_filter_update_fused": (c_int, [c_void_p, POINTER(PfcoreOdom),
                                           POINTER(PfcoreObservation), c_int,
                                           POINTER(PfcoreEstimate)]),
    "pfcore_filter_snapshot": (c_int, [c_void_p, _dp, _dp, _dp]),
    "pfcore_filter_handle": (c_void_p, [c_void_p]),
    "pfcore_quat_mean": (None, [_dp, _dp]),
    "pfcore_gl_params_default": (None, [POINTER(PfcoreGlParams)]),
    "pfcore_gl_new": (c_void_p, [c_int, c_int, c_double, c_double, c_double, _u8p,
                                 POINTER(PfcoreGlParams)]),
    "pfcore_gl_free": (None, [c_void_p]),
    "pfcore_gl_free_cells": (c_int, [c_void_p]),
    "pfcore_gl_set_seed": (c_int, [c_void_p, c_ulonglong]),
    "pfcore_gl_localize": (c_int, [c_void_p, _fp, c_int, POINTER(PfcorePoseHypothesis)]),
    "pfcore_gl_handle": (c_void_p, [c_void_p]),
    "pfcore_grid_from_pgm_yaml": (c_int, [C.c_char_p, C.c_size_t, C.c_char_p, _ip, _ip,
                                          _dp, _dp, _dp, _u8p]),
    "pfcore_last_error": (C.c_char_p, []),
}

_kernels = None
_core = None


def _bind(lib, sigs):
    for name, (res, args) in sigs.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


def kernels():
    """The drop-in CUDA library (raises when it has not been built)."""
    global _kernels
    if _kernels is None:
        if not KERNELS_SO.exists():
            raise RuntimeError(f"{KERNELS_SO} is missing: run "
                               "`python -m cuda_pf_localization_b200.build`")
        _kernels = _bind(C.CDLL(str(KERNELS_SO)), _KERNEL_SIGS)
    return _kernels


def core():
    """The C++ host layer (pf_core mirror) over the CUDA library."""
    global _core
    if _core is None:
        kernels()
        if not CORE_SO.exists():
            raise RuntimeError(f"{CORE_SO} is missing: run "
                               "`python -m cuda_pf_localization_b200.build`")
        _core = _bind(C.CDLL(str(CORE_SO)), _CORE_SIGS)
    return _core


def last_error() -> str:
    return kernels().pfc_last_error_message().decode(errors="replace")


def fptr(a: np.ndarray):
    assert a.dtype == np.float32 and a.flags.c_contiguous
    return a.ctypes.data_as(_fp)


def dptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_dp)


def iptr(a: np.ndarray):
    assert a.dtype == np.int32 and a.flags.c_contiguous
    return a.ctypes.data_as(_ip)


def u8ptr(a: np.ndarray):
    assert a.dtype == np.uint8 and a.flags.c_contiguous
    return a.ctypes.data_as(_u8p)


COBS_DTYPE = np.dtype([("id", "<i4"), ("mode", "<i4"), ("dx", "<f4"), ("dy", "<f4"),
                       ("dz", "<f4"), ("range", "<f4")])


def cobs_records(rows) -> np.ndarray:
    """CObservation records (numpy, 24 bytes each) from (id, mode, dx, dy, dz,
    range) rows."""
    rows = np.asarray(rows, dtype=np.float64).reshape(-1, 6)
    a = np.zeros(len(rows), COBS_DTYPE)
    a["id"] = rows[:, 0].astype(np.int32)
    a["mode"] = rows[:, 1].astype(np.int32)
    a["dx"], a["dy"], a["dz"], a["range"] = rows[:, 2], rows[:, 3], rows[:, 4], rows[:, 5]
    return a


def make_cobs(rows) -> "C.Array":
    """Array of CObservation from (id, mode, dx, dy, dz, range) rows."""
    a = cobs_records(rows)
    arr = (CObservation * max(1, len(a)))()
    if len(a):
        C.memmove(arr, a.ctypes.data, a.nbytes)
    return arr


def make_core_obs(rows):
    arr = (PfcoreObservation * max(1, len(rows)))()
    for k, r in enumerate(rows):
        arr[k].landmark_id = int(r[0])
        arr[k].mode = int(r[1])
        arr[k].vector[:] = [float(r[2]), float(r[3]), float(r[4])]
        arr[k].range = float(r[5])
    return arr


def make_core_odom(t, q, tn, rn) -> PfcoreOdom:
    o = PfcoreOdom()
    o.translation[:] = list(map(float, t))
    o.rotation[:] = list(map(float, q))
    o.trans_noise[:] = list(map(float, tn))
    o.rot_noise[:] = list(map(float, rn))
    return o


def estimate_dict(e: PfcoreEstimate) -> dict:
    return dict(position=np.array(e.position[:]), attitude=np.array(e.attitude[:]),
                pos_cov=np.array(e.pos_cov[:]).reshape(3, 3),
                att_cov=np.array(e.att_cov[:]).reshape(3, 3), ess=float(e.ess),
                valid=bool(e.valid), resampled=bool(e.resampled))


class LandmarkMap:
    """``pf_core::LandmarkMap`` (crates/pf_core/src/landmark_map.rs:7-80):
    dense id -> 3-D position, host only.  Where the reference panics (a
    negative id in ``add``, an absent id in ``at``) this raises ValueError;
    ``load_from_str`` raises ValueError at the first bad line, the lines before
    it staying in the map as in the reference."""

    def __init__(self):
        self._m = core().pfcore_landmarks_new()
        if not self._m:
            raise MemoryError("pfcore_landmarks_new failed")

    def close(self):
        if getattr(self, "_m", None):
            core().pfcore_landmarks_free(self._m)
            self._m = None

    __del__ = close

    @property
    def handle(self):
        return self._m

    def add(self, id: int, position) -> None:
        p = [float(v) for v in position]
        if core().pfcore_landmarks_add(self._m, int(id), p[0], p[1], p[2]) != 0:
            raise ValueError(core().pfcore_last_error().decode())

    def has(self, id: int) -> bool:
        return core().pfcore_landmarks_has(self._m, int(id)) == 1

    def at(self, id: int) -> np.ndarray:
        out = np.zeros(3)
        if core().pfcore_landmarks_at(self._m, int(id), dptr(out)) != 0:
            raise ValueError(core().pfcore_last_error().decode())
        return out

    def capacity(self) -> int:
        return int(core().pfcore_landmarks_capacity(self._m))

    def len_defined(self) -> int:
        return int(core().pfcore_landmarks_len_defined(self._m))

    def is_empty(self) -> bool:
        return self.len_defined() == 0

    def load_from_str(self, text: str) -> int:
        n = core().pfcore_landmarks_load_text(self._m, text.encode())
        if n < 0:
            raise ValueError(core().pfcore_last_error().decode())
        return n


class ParticleFilter:
    """``pf_core::ParticleFilter`` with the CUDA backend (through libpf_core)."""

    def __init__(self, particle_count=4096, seed=42, range_noise=0.05,
                 bearing_noise=0.02, resample_ess_ratio=0.5, random_inject_ratio=0.0,
                 gate_sigma=0.0, trans_noise=(0.05, 0.05, 0.02), rot_noise=(0.02, 0.02, 0.03)):
        lib = core()
        cfg = PfcoreConfig()
        lib.pfcore_config_default(byref(cfg))
        cfg.particle_count = int(particle_count)
        cfg.seed = int(seed)
        cfg.range_noise = range_noise
        cfg.bearing_noise = bearing_noise
        cfg.resample_ess_ratio = resample_ess_ratio
        cfg.random_inject_ratio = random_inject_ratio
        cfg.gate_sigma = gate_sigma
        cfg.trans_noise[:] = list(trans_noise)
        cfg.rot_noise[:] = list(rot_noise)
        self.cfg = cfg
        self.n = int(particle_count)
        self._h = lib.pfcore_filter_new(byref(cfg))
        if not self._h:
            raise RuntimeError("pfcore_filter_new failed: "
                               + lib.pfcore_last_error().decode())

    def close(self):
        if getattr(self, "_h", None):
            core().pfcore_filter_free(self._h)
            self._h = None

    __del__ = close

    @property
    def handle(self):
        return core().pfcore_filter_handle(self._h)

    def set_map(self, landmarks):
        """A ``LandmarkMap`` (copied, as ``ParticleFilter::set_map``) or a
        dict id -> (x, y, z)."""
        lib = core()
        if isinstance(landmarks, LandmarkMap):
            if lib.pfcore_filter_set_map(self._h, landmarks.handle) != 0:
                raise RuntimeError("set_map failed")
            return
        lib.pfcore_map_clear(self._h)
        for i, p in landmarks.items():
            if lib.pfcore_map_add(self._h, int(i), float(p[0]), float(p[1]),
                                  float(p[2])) != 0:
                raise ValueError(lib.pfcore_last_error().decode())

    def load_map_text(self, text: str) -> int:
        lib = core()
        lib.pfcore_map_clear(self._h)
        n = lib.pfcore_map_load_text(self._h, text.encode())
        if n < 0:
            raise ValueError(lib.pfcore_last_error().decode())
        return n

    def reinitialize(self, pose, pos_std, rot_std):
        pose = np.ascontiguousarray(pose, dtype=np.float64)
        ps = np.ascontiguousarray(pos_std, dtype=np.float64)
        rs = np.ascontiguousarray(rot_std, dtype=np.float64)
        rc = core().pfcore_filter_reinitialize(self._h, dptr(pose), dptr(ps), dptr(rs))
        if rc != 0:
            raise RuntimeError("reinitialize failed")

    def update(self, odom: PfcoreOdom, obs_rows, fused=False) -> dict:
        arr = make_core_obs(obs_rows)
        est = PfcoreEstimate()
        fn = core().pfcore_filter_update_fused if fused else core().pfcore_filter_update
        rc = fn(self._h, byref(odom), arr, len(obs_rows), byref(est))
        if rc != 0:
            raise RuntimeError("update failed: " + core().pfcore_last_error().decode())
        return estimate_dict(est)

    def snapshot(self):
        pos = np.zeros(3 * self.n)
        quat = np.zeros(4 * self.n)
        w = np.zeros(self.n)
        if core().pfcore_filter_snapshot(self._h, dptr(pos), dptr(quat), dptr(w)) != 0:
            raise RuntimeError("snapshot failed")
        return pos.reshape(-1, 3), quat.reshape(-1, 4), w


class GlobalLoc:
    """``pf_core::global_loc::CudaGlobalLoc`` (through libpf_core)."""

    def __init__(self, cells: np.ndarray, res=0.05, origin=(0.0, 0.0), hypotheses=50000,
                 rays=360, rmax=10.0, ang_span=2 * np.pi, topk=10, seed=42):
        lib = core()
        cells = np.ascontiguousarray(cells, dtype=np.uint8)
        self.h_cells, self.w_cells = cells.shape
        p = PfcoreGlParams(int(hypotheses), int(rays), float(rmax), float(ang_span),
                           int(topk), int(seed))
        self.params = p
        self._h = lib.pfcore_gl_new(self.w_cells, self.h_cells, res, origin[0], origin[1],
                                    u8ptr(cells), byref(p))
        if not self._h:
            raise RuntimeError("pfcore_gl_new failed")

    def close(self):
        if getattr(self, "_h", None):
            core().pfcore_gl_free(self._h)
            self._h = None

    __del__ = close

    @property
    def handle(self):
        return core().pfcore_gl_handle(self._h)

    def free_cells(self) -> int:
        return core().pfcore_gl_free_cells(self._h)

    def set_seed(self, seed: int):
        core().pfcore_gl_set_seed(self._h, int(seed))

    def localize(self, scan_f32: np.ndarray):
        scan = np.ascontiguousarray(scan_f32, dtype=np.float32)
        out = (PfcorePoseHypothesis * self.params.topk)()
        k = core().pfcore_gl_localize(self._h, fptr(scan), len(scan), out)
        if k <= 0:
            raise RuntimeError("localize failed: " + core().pfcore_last_error().decode())
        return [(out[j].x, out[j].y, out[j].theta, out[j].caer) for j in range(k)]


# ----------------------------------------------------------- learned proposal

LP_IN, LP_HIDDEN, LP_OUT, LP_COMP, LP_LAYERS = 384, 1024, 384, 32, 5


class LearnedProposal:
    """Per-map learned proposal for global localization (``pfgl_learned_*``).

    Borrows a raw ``pfgl_*`` handle (map, scorer, stream); close this object
    before destroying that handle.
    """

    def __init__(self, gl_handle, batch: int = 1024, seed: int = 1):
        self.lib = kernels()
        self.gl = gl_handle
        self.batch = int(batch)
        self._h = self.lib.pfgl_learned_create(gl_handle, self.batch, int(seed))
        if not self._h:
            raise RuntimeError("pfgl_learned_create failed: " + last_error())

    def close(self):
        if getattr(self, "_h", None):
            self.lib.pfgl_learned_destroy(self._h)
            self._h = None

    __del__ = close

    def _ok(self, rc, what):
        if rc < 0:
            raise RuntimeError(f"{what} failed: {last_error()}")
        return rc

    @staticmethod
    def num_params() -> int:
        return int(kernels().pfgl_learned_num_params())

    def params(self) -> np.ndarray:
        out = np.zeros(self.num_params(), np.float32)
        self._ok(self.lib.pfgl_learned_get_params(self._h, fptr(out)), "get_params")
        return out

    def set_params(self, flat: np.ndarray):
        flat = np.ascontiguousarray(flat, np.float32)
        self._ok(self.lib.pfgl_learned_set_params(self._h, fptr(flat)), "set_params")

    def norm(self):
        c = np.zeros(4, np.float32)
        self._ok(self.lib.pfgl_learned_norm(self._h, fptr(c)), "norm")
        return c

    def make_data(self, n_pairs: int, nrays=360, rmax=10.0, span=2 * np.pi, noise=0.01,
                  seed=7):
        self._ok(self.lib.pfgl_learned_make_data(self._h, int(n_pairs), nrays, rmax, span,
                                                 noise, int(seed)), "make_data")

    def train(self, steps: int, total_steps: int | None = None, lr: float = 1e-3):
        loss = np.zeros(steps, np.float32)
        self._ok(self.lib.pfgl_learned_train(self._h, int(steps), int(total_steps or steps),
                                             float(lr), fptr(loss)), "train")
        return loss

    def grad(self, x: np.ndarray, y: np.ndarray):
        x = np.ascontiguousarray(x, np.float32)
        y = np.ascontiguousarray(y, np.float32)
        assert x.shape == (self.batch, LP_IN) and y.shape == (self.batch, 4)
        g = np.zeros(self.num_params(), np.float32)
        loss = np.zeros(1, np.float32)
        self._ok(self.lib.pfgl_learned_grad(self._h, fptr(x), fptr(y), fptr(loss), fptr(g)),
                 "grad")
        return float(loss[0]), g

    def forward(self, x: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(x, np.float32)
        out = np.zeros((x.shape[0], LP_COMP * 9), np.float32)
        self._ok(self.lib.pfgl_learned_forward(self._h, fptr(x), x.shape[0], fptr(out)),
                 "forward")
        return out

    def calibrate(self, n_queries=200, nrays=360, rmax=10.0, span=2 * np.pi, noise=0.01,
                  n_samples=20000, quantile=0.98, seed=99):
        tau = np.zeros(1, np.float32)
        ok = np.zeros(1, np.float32)
        self._ok(self.lib.pfgl_learned_calibrate(self._h, n_queries, nrays, rmax, span, noise,
                                                 n_samples, quantile, int(seed), fptr(tau),
                                                 fptr(ok)), "calibrate")
        return float(tau[0]), float(ok[0])

    def use_graph(self, on: bool = True):
        self._ok(self.lib.pfgl_learned_set_graph(self._h, 1 if on else 0), "set_graph")

    def set_threshold(self, tau: float):
        self._ok(self.lib.pfgl_learned_set_threshold(self._h, float(tau)), "set_threshold")

    def localize_batch(self, scans: np.ndarray, n_samples=1000, n_fallback=200000, k=64,
                       rmax=10.0, span=2 * np.pi):
        """``pfgl_learned_localize_batch``: returns (poses nq x k x 3, CAERs
        nq x k, sample indices nq x k, info nq)."""
        scans = np.ascontiguousarray(scans, np.float32)
        nq, nrays = scans.shape
        kk = min(k, n_samples)
        out = np.zeros((nq, kk, 3), np.float32)
        cs = np.zeros((nq, kk), np.float32)
        ids = np.zeros((nq, kk), np.int32)
        info = np.zeros(nq, np.int32)
        self._ok(self.lib.pfgl_learned_localize_batch(self._h, fptr(scans), nq, nrays, rmax,
                                                      span, n_samples, n_fallback, kk,
                                                      fptr(out), fptr(cs), iptr(ids),
                                                      iptr(info)), "localize_batch")
        return out, cs, ids, info

    def localize(self, scan: np.ndarray, n_samples=20000, n_fallback=200000, k=64,
                 rmax=10.0, span=2 * np.pi):
        scan = np.ascontiguousarray(scan, np.float32)
        out = np.zeros(3 * k, np.float32)
        cs = np.zeros(k, np.float32)
        ids = np.zeros(k, np.int32)
        info = np.zeros(1, np.int32)
        r = self._ok(self.lib.pfgl_learned_localize(self._h, fptr(scan), len(scan), rmax, span,
                                                    n_samples, n_fallback, k, fptr(out),
                                                    fptr(cs), iptr(ids), iptr(info)),
                     "localize")
        return out[:3 * r].reshape(r, 3), cs[:r], ids[:r], int(info[0])


def localize_batch(gl_handle, scans: np.ndarray, n_pos: int, n_yaw: int, seeds, k=64,
                   rmax=10.0, span=2 * np.pi):
    """Batched uniform CBGL (``pfgl_localize_batch``): query q scored against
    its own dispersion (n_pos x n_yaw, seeds[q]).  Returns (poses nq x k x 3,
    CAERs nq x k, indices nq x k)."""
    scans = np.ascontiguousarray(scans, np.float32)
    nq, nrays = scans.shape
    sd = np.ascontiguousarray(seeds, np.uint64)
    out = np.zeros((nq, k, 3), np.float32)
    cs = np.zeros((nq, k), np.float32)
    ids = np.zeros((nq, k), np.int32)
    r = kernels().pfgl_localize_batch(gl_handle, fptr(scans), nq, nrays, rmax, span, n_pos,
                                      n_yaw, sd.ctypes.data_as(POINTER(c_ulonglong)), k,
                                      fptr(out), fptr(cs), iptr(ids))
    if r < 0:
        raise RuntimeError("pfgl_localize_batch failed: " + last_error())
    return out[:, :r], cs[:, :r], ids[:, :r]


def render_scans(gl_handle, poses: np.ndarray, nrays=360, rmax=10.0, span=2 * np.pi,
                 noise=0.0, seed=0) -> np.ndarray:
    """Scans at poses (n x 3) from the library's raycaster (CAER ray geometry)."""
    poses = np.ascontiguousarray(poses, np.float32).reshape(-1, 3)
    out = np.zeros((len(poses), nrays), np.float32)
    rc = kernels().pfgl_render_scans(gl_handle, fptr(poses), len(poses), nrays, rmax, span,
                                     noise, int(seed), fptr(out))
    if rc != 0:
        raise RuntimeError("pfgl_render_scans failed: " + last_error())
    return out


def learned_gemm(a_bf16: np.ndarray, b_bf16: np.ndarray) -> np.ndarray:
    """D = A B^T on the tcgen05 GEMM (A: M x K, B: N x K as uint16 bf16 bits)."""
    a = np.ascontiguousarray(a_bf16, np.uint16)
    b = np.ascontiguousarray(b_bf16, np.uint16)
    M, K = a.shape
    N = b.shape[0]
    d = np.zeros((M, N), np.float32)
    rc = kernels().pfgl_learned_gemm(M, N, K, a.ctypes.data_as(POINTER(C.c_ushort)),
                                     b.ctypes.data_as(POINTER(C.c_ushort)), fptr(d))
    if rc != 0:
        raise RuntimeError("pfgl_learned_gemm failed: " + last_error())
    return d


# ------------------------------------------------------------ batched filters

class PfcBatchCycle(C.Structure):
    _fields_ = [("odom", PfcOdom), ("obs_off", c_int), ("nobs", c_int)]


class BatchPF:
    """Many independent filters advanced by one graph launch per cycle
    (``pfc_batch_*``)."""

    def __init__(self, sizes, seeds=None, obs_cap=1 << 16):
        self.lib = kernels()
        self.sizes = np.ascontiguousarray(sizes, np.int32)
        self.nf = len(self.sizes)
        sd = None
        if seeds is not None:
            self._seeds = (c_uint * self.nf)(*[int(x) for x in seeds])
            sd = self._seeds
        self._h = self.lib.pfc_batch_create(self.nf, iptr(self.sizes), sd, int(obs_cap))
        if not self._h:
            raise RuntimeError("pfc_batch_create failed: " + last_error())

    def close(self):
        if getattr(self, "_h", None):
            self.lib.pfc_batch_destroy(self._h)
            self._h = None

    __del__ = close

    @property
    def handle(self):
        return self._h

    def _ok(self, rc, what):
        if rc != 0:
            raise RuntimeError(f"{what} failed: {last_error()}")

    def set_params(self, sigma_r=0.05, sigma_b=0.02, gate=3.0, ess_ratio=0.5, inject=0.0):
        arr = (PfcCycleParams * self.nf)()
        for f in range(self.nf):
            arr[f] = PfcCycleParams(sigma_r, sigma_b, gate, ess_ratio, inject, 0)
        self._ok(self.lib.pfc_batch_set_params(self._h, arr), "set_params")

    def set_landmarks(self, tables):
        counts = np.array([len(t) for t in tables], np.int32)
        xyz = np.ascontiguousarray(np.concatenate([np.asarray(t, np.float32).reshape(-1, 3)
                                                   for t in tables]).reshape(-1), np.float32)
        self._ok(self.lib.pfc_batch_upload_landmarks(self._h, fptr(xyz), iptr(counts)),
                 "upload_landmarks")

    def reinit(self, pose7, pos_std3, rot_std3):
        p = np.ascontiguousarray(pose7, np.float32).reshape(-1)
        a = np.ascontiguousarray(pos_std3, np.float32).reshape(-1)
        b = np.ascontiguousarray(rot_std3, np.float32).reshape(-1)
        self._ok(self.lib.pfc_batch_reinit(self._h, fptr(p), fptr(a), fptr(b)), "reinit")

    def cycle(self, odoms, obs_rows, want_est=True):
        """odoms: list of PfcOdom; obs_rows: list of (k, 6) arrays per filter."""
        od = (PfcOdom * self.nf)(*odoms)
        nobs = np.array([len(r) for r in obs_rows], np.int32)
        allrows = [r for r in obs_rows if len(r)]
        obs = make_cobs(np.concatenate(allrows)) if allrows else None
        est = np.zeros((self.nf, PFC_EST_LEN)) if want_est else None
        self._ok(self.lib.pfc_batch_cycle(self._h, od, obs, iptr(nobs),
                                          dptr(est) if want_est else None), "cycle")
        return est

    def snapshot(self, f):
        n = int(self.sizes[f])
        pos = np.zeros(3 * n, np.float32)
        quat = np.zeros(4 * n, np.float32)
        self._ok(self.lib.pfc_batch_snapshot(self._h, f, fptr(pos), fptr(quat)), "snapshot")
        return pos, quat

    def weights(self, f):
        w = np.zeros(int(self.sizes[f]), np.float32)
        self._ok(self.lib.pfc_batch_get_weights(self._h, f, fptr(w)), "get_weights")
        return w

    def use_graph(self, on: bool):
        self._ok(self.lib.pfc_batch_use_graph(self._h, 1 if on else 0), "use_graph")

    def set_wait_test(self, spin_limit: int = 0, stall_filter: int = -1):
        """Bounded-wait test hook (pfc_batch_set_wait_test)."""
        self._ok(self.lib.pfc_batch_set_wait_test(self._h, int(spin_limit),
                                                  int(stall_filter)), "set_wait_test")

    def tiles(self):
        t = np.zeros(4, np.int32)
        pk = np.zeros(1, np.int32)
        self._ok(self.lib.pfc_batch_get_tiles(self._h, iptr(t), iptr(pk)), "get_tiles")
        return t, int(pk[0])

    def set_tiles(self, est_tile4, packed=1):
        t = np.ascontiguousarray(est_tile4, np.int32)
        self._ok(self.lib.pfc_batch_set_tiles(self._h, iptr(t), int(packed)), "set_tiles")

    def autotune(self, reps=3):
        t = np.zeros(4, np.int32)
        pk = np.zeros(1, np.int32)
        self._ok(self.lib.pfc_batch_autotune(self._h, int(reps), iptr(t), iptr(pk)),
                 "autotune")
        return t, int(pk[0])
