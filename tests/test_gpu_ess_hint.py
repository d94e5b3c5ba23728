"""pfc_set_ess_hint: told ParticleFilter::update's rule (resample when the ESS
of the estimate after a weighting is below ratio * N), the library reports
only the ESS of an estimate that a resample will discard (pfc_est_ess) and
skips its other sums and its covariance pass.  Bar: a handle with the hint
and one without, stepped through the same calls, return the same ESS,
estimate sums and covariances bit for bit, on cycles that resample and
cycles that do not, including when the caller asks for the skipped sums and
covariances (computed on demand)."""
import numpy as np
import pytest

import cuda_pf_localization_b200 as pkg
from cuda_pf_localization_b200 import sim
from tests.pf_helpers import RawPF

pytestmark = pytest.mark.gpu

RATIO = 0.5


def _mean(sums):
    m = np.zeros((4, 4))
    e = 3
    for r in range(4):
        for c in range(r, 4):
            m[r, c] = m[c, r] = sums[e]
            e += 1
    q = np.linalg.eigh(m)[1][:, -1]
    q = -q if q[0] < 0 else q
    return sums[:3].astype(np.float32), q.astype(np.float32)


def _ess(kernels, f):
    out = np.zeros(1)
    assert kernels.pfc_est_ess(f.h, pkg.dptr(out)) == 0
    return float(out[0])


def test_hint_keeps_every_result(kernels):
    n = 100_003
    sc = sim.scale_config(cycles=8, seed=5)
    a, b = RawPF(kernels, n, seed=9), RawPF(kernels, n, seed=9)
    try:
        assert kernels.pfc_set_ess_hint(a.h, RATIO) == 0
        assert kernels.pfc_set_ess_hint(a.h, float("nan")) == -1
        for f in (a, b):
            f.landmarks(sc.landmarks)
            f.reinit(np.r_[sc.prior_p, sc.prior_q], [0.5] * 3, [0.2] * 3)
        seen = {True: 0, False: 0}
        for k, st in enumerate(sc.steps):
            rows = st.obs if k % 2 == 0 else []  # no observations: uniform, no resample
            for f in (a, b):
                f.predict(st.odom_t, st.odom_q, sc.trans_noise, sc.rot_noise)
                assert f.weight(rows) == 0
            ess = _ess(kernels, a)
            assert ess == _ess(kernels, b)
            resample = ess < RATIO * n
            seen[resample] += 1
            if not resample or k % 4 == 0:
                # the kept estimate, or the caller asks for the discarded one
                # (the hinted handle computes it on demand)
                sa, sb = a.est_sums(), b.est_sums()
                np.testing.assert_array_equal(sa, sb)
                assert ess == (1.0 / sa[13] if sa[13] > 0 else 0.0)
                mp, mq = _mean(sa)
                np.testing.assert_array_equal(a.covs(mp, mq), b.covs(mp, mq))
            if resample:
                for f in (a, b):
                    f.resample(0.01)
                sa, sb = a.est_sums(), b.est_sums()
                np.testing.assert_array_equal(sa, sb)
                mp, mq = _mean(sa)
                np.testing.assert_array_equal(a.covs(mp, mq), b.covs(mp, mq))
        assert seen[True] >= 2 and seen[False] >= 2
        pa, qa = a.snapshot()
        pb, qb = b.snapshot()
        np.testing.assert_array_equal(pa, pb)
        np.testing.assert_array_equal(qa, qb)
    finally:
        a.close()
        b.close()


def test_update_mirror_reports_covariances_either_way(kernels):
    """The host mirror of ParticleFilter::update (which sets the hint and
    takes the first estimate's covariances only when it returns it) still
    reports covariances on cycles that resample and on cycles that do not."""
    sc = sim.scale_config(cycles=6, seed=3)
    filt = dict(range_noise=0.05, bearing_noise=0.02, gate_sigma=3.0,
                resample_ess_ratio=RATIO, random_inject_ratio=0.01)
    pf = pkg.ParticleFilter(50_000, seed=42, trans_noise=sc.trans_noise,
                            rot_noise=sc.rot_noise, **filt)
    try:
        pf.set_map(sc.landmark_dict())
        pf.reinitialize(np.r_[sc.prior_p, sc.prior_q], [0.5] * 3, [0.2] * 3)
        kinds = set()
        for k, st in enumerate(sc.steps):
            rows = st.obs if k % 2 == 0 else []
            e = pf.update(pkg.make_core_odom(st.odom_t, st.odom_q, sc.trans_noise,
                                             sc.rot_noise), rows)
            kinds.add(bool(e["resampled"]))
            assert e["valid"]
            cov = np.asarray(e["pos_cov"]).reshape(3, 3)
            assert np.all(np.isfinite(cov)) and np.all(np.diag(cov) > 0)
        assert kinds == {True, False}
    finally:
        pf.close()
