"""Generate tests/golden/reference_outputs.npz from the reference library.

Runs the reference's own CUDA library (compiled from its source by
oracle/build.py into oracle/_ref/) on a GPU, on small seeded inputs, and
stores inputs and outputs.  tests/test_golden_reference.py then checks the
CPU oracle against these outputs without a GPU.

    python tests/golden/make_golden.py        # needs a CUDA device and oracle/_ref

Cases
  cart_gated   2048 particles, 64 landmarks, 256 Cartesian observations (10 %
               outliers), sigma_r 1.0, gate 3: log-likelihoods, weights, the
               14 estimate sums and the 12 covariance sums around the f32
               means (host Markley mean)
  cart_ungated same inputs, gate 0: log-likelihoods
  range_bearing same cloud, the observations as range + unit bearing: ll
  caer         4096 hypotheses (64 positions x 64 yaws) on the 10 x 10 m test
               room against a rendered scan: CAER per hypothesis
  topk         bottom-64 indices of the reference's radix sort fed scores with
               many ties
"""
from __future__ import annotations

import ctypes as C
import math
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path[:0] = [str(ROOT), str(ROOT / "tests")]

import oracle  # noqa: E402
import cuda_pf_localization_b200 as pkg  # noqa: E402
from cuda_pf_localization_b200 import sim  # noqa: E402
from pf_helpers import RawPF, cloud, ref_ll, ref_set_state, ref_weights, scale_obs  # noqa: E402


def markley(est):
    m = np.zeros((4, 4))
    e = 3
    for r in range(4):
        for c in range(r, 4):
            m[r, c] = m[c, r] = est[e]
            e += 1
    vals, vecs = np.linalg.eigh(m)
    q = vecs[:, int(np.argmax(vals))]
    return q if q[0] >= 0 else -q


def main():
    ref = oracle.ref_lib()
    assert ref is not None, "oracle/_ref/libpf_kernels_ref.so is required"
    out = {}
    n = 2048
    pos, quat = cloud(n, 3, centre=(1.0, -2.0, 0.5))
    lm, obs, _, _ = scale_obs(seed=11, step=0)
    lm32 = np.ascontiguousarray(lm, np.float32)
    obs_rec = pkg.cobs_records(obs)
    out.update(pos=pos, quat=quat, landmarks=lm32, obs=obs_rec.view(np.uint8).reshape(-1, 24))

    pf = RawPF(ref, n, seed=5)
    try:
        pf.landmarks(lm32)
        ref_set_state(ref, pf, pos, quat)
        assert pf.weight(obs, sr=1.0, sb=0.02, gate=3.0) == 0
        out["ll_gated"] = ref_ll(ref, pf)
        w = ref_weights(ref, pf)
        out["w_gated"] = w
        est = pf.est_sums()
        out["est"] = est
        mp = np.float32(est[:3])
        mq = np.float32(markley(est))
        out["cov_mean_p"], out["cov_mean_q"] = mp, mq
        out["covs"] = pf.covs(mp, mq)

        ref_set_state(ref, pf, pos, quat)
        assert pf.weight(obs, sr=1.0, sb=0.02, gate=0.0) == 0
        out["ll_ungated"] = ref_ll(ref, pf)

        rb = obs.copy()
        v = rb[:, 2:5]
        r = np.linalg.norm(v, axis=1)
        rb[:, 1] = 1
        rb[:, 5] = r
        rb[:, 2:5] = v / np.maximum(r, 1e-9)[:, None]
        out["obs_rb"] = pkg.cobs_records(rb).view(np.uint8).reshape(-1, 24)
        ref_set_state(ref, pf, pos, quat)
        assert pf.weight(rb, sr=0.3, sb=0.05, gate=3.0) == 0
        out["ll_rb"] = ref_ll(ref, pf)
    finally:
        pf.close()

    # GL: CAER on fed hypotheses and bottom-k of fed scores
    g = np.ascontiguousarray(sim.room_grid())
    gh = ref.pfgl_create(200, 200, 0.05, 0.0, 0.0, pkg.u8ptr(g), 4096)
    try:
        truth = (6.0, 7.0, 0.8)
        scan = oracle.map_scan(g, 0.05, (0, 0), *truth, 360, 2 * math.pi, 10.0)
        scan = (scan + np.random.default_rng(1).normal(0, 0.01, 360)).astype(np.float32)
        hyp = oracle.gl_generate(g, 0.05, (0, 0), 64, 64, 9).astype(np.float32)
        flat = np.ascontiguousarray(hyp.reshape(-1))
        assert ref.ref_gl_set_hyps(gh, pkg.fptr(flat), 4096) == 0
        assert ref.pfgl_score(gh, pkg.fptr(scan), 360, 10.0, 2 * math.pi) == 0
        caer = np.zeros(4096, np.float32)
        assert ref.ref_gl_get_caer(gh, pkg.fptr(caer)) == 0
        out.update(grid=g, scan=scan, hyp=hyp, caer=caer)

        scores = np.round(np.random.default_rng(2).uniform(0, 50, 4096), 1).astype(np.float32)
        assert ref.ref_gl_set_caer(gh, pkg.fptr(scores), 4096) == 0
        top3 = np.zeros(3 * 64, np.float32)
        assert ref.pfgl_topk(gh, 64, pkg.fptr(top3)) == 64
        idx = np.zeros(64, np.int32)
        assert ref.ref_gl_get_sorted(gh, pkg.iptr(idx), 64) == 0
        out.update(topk_scores=scores, topk_idx=idx)
    finally:
        ref.pfgl_destroy(gh)

    np.savez_compressed(HERE / "reference_outputs.npz", **out)
    print("wrote", HERE / "reference_outputs.npz")


if __name__ == "__main__":
    main()
