"""The CPU oracle against outputs of the reference's own CUDA library.

tests/golden/reference_outputs.npz holds inputs and the reference library's
outputs for small seeded cases (made by tests/golden/make_golden.py on a GPU
from the reference source compiled by oracle/build.py).  These checks pin the
oracle's restatement of the weighting model, the softmax, the estimate and
covariance sums, the CAER raycast and the bottom-k order to the reference
itself, with no GPU needed.
"""
from pathlib import Path

import numpy as np
import pytest

import cuda_pf_localization_b200 as pkg
import oracle

GOLD = Path(__file__).resolve().parent / "golden" / "reference_outputs.npz"

pytestmark = pytest.mark.skipif(not GOLD.exists(), reason="golden fixtures not generated")


@pytest.fixture(scope="module")
def g():
    return dict(np.load(GOLD))


def _rows(raw):
    rec = np.ascontiguousarray(raw).view(pkg.COBS_DTYPE).reshape(-1)
    return [(int(r["id"]), int(r["mode"]), float(r["dx"]), float(r["dy"]), float(r["dz"]),
             float(r["range"])) for r in rec]


def _ll(g, key_obs, sr, sb, gate):
    return oracle.loglik(g["pos"].astype(np.float64).reshape(-1, 3),
                         g["quat"].astype(np.float64).reshape(-1, 4),
                         g["landmarks"].astype(np.float64).reshape(-1, 3),
                         _rows(g[key_obs]), sr, sb, gate)


def test_loglik_gated(g):
    ll = _ll(g, "obs", 1.0, 0.02, 3.0)
    # FP64 oracle vs the reference's f32 accumulation over 256 terms
    assert np.allclose(ll, g["ll_gated"], rtol=1e-5, atol=1e-4)


def test_loglik_ungated(g):
    ll = _ll(g, "obs", 1.0, 0.02, 0.0)
    assert np.allclose(ll, g["ll_ungated"], rtol=1e-5, atol=1e-4)


def test_loglik_range_bearing(g):
    ll = _ll(g, "obs_rb", 0.3, 0.05, 3.0)
    assert np.allclose(ll, g["ll_rb"], rtol=1e-5, atol=1e-3)


def test_softmax_weights(g):
    ll = g["ll_gated"].astype(np.float64)
    w = np.exp(ll - ll.max())
    w /= w.sum()
    ref = g["w_gated"].astype(np.float64)
    big = ref > 1e-6 * ref.max()
    assert big.sum() >= 10
    assert np.allclose(w[big], ref[big], rtol=1e-5)
    assert np.allclose(w, ref, rtol=0, atol=1e-6 * ref.max())


def test_estimate_and_covariance_sums(g):
    est = oracle.est_sums(g["pos"], g["quat"], g["w_gated"])
    assert np.allclose(est, g["est"], rtol=1e-5, atol=1e-9)
    cv = oracle.covs(g["pos"], g["quat"], g["w_gated"], g["cov_mean_p"], g["cov_mean_q"])
    assert np.allclose(cv, g["covs"], rtol=1e-4, atol=1e-9)


def test_caer_on_fed_hypotheses(g):
    c = oracle.caer_f32(g["grid"], 0.05, (0, 0), g["scan"], 2 * np.pi, 10.0, g["hyp"])
    rel = np.abs(c - g["caer"]) / np.maximum(g["caer"], 1e-3)
    assert np.max(rel) < 1e-5


def test_bottom_k_order(g):
    assert np.array_equal(oracle.topk_from_scores(g["topk_scores"], 64), g["topk_idx"])
