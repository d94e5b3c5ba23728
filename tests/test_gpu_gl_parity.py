"""GPU parity of the global-localization path against the oracle and the
reference library built from its own source, through the C-ABI.

Tolerances: CAER 1e-5 relative to the reference on fed hypotheses (same f32
DDA arithmetic, different summation order); bottom-k indices bit-exact when
fed identical scores; dispersion bit-exact against the oracle's mirror of the
Philox spec; the fused pruned localizer bit-exact against exhaustive scoring.
"""
import ctypes as C
import math

import numpy as np
import pytest

import cuda_pf_localization_b200 as pkg
import oracle
from cuda_pf_localization_b200 import sim
from tests.pf_helpers import f32p, i32p

pytestmark = pytest.mark.gpu
TAU = 2 * math.pi
U8P = C.POINTER(C.c_ubyte)


class Gl:
    def __init__(self, lib, cells, cap, res=0.05, origin=(0.0, 0.0)):
        self.lib = lib
        self.cells = np.ascontiguousarray(cells, np.uint8)
        h, w = self.cells.shape
        self.h = lib.pfgl_create(w, h, res, origin[0], origin[1],
                                 self.cells.ctypes.data_as(U8P), cap)
        assert self.h

    def close(self):
        if self.h:
            self.lib.pfgl_destroy(self.h)
            self.h = None


def _scene(seed=3, n_hyp=20_000):
    g = sim.rooms_grid(seed)
    rng = np.random.default_rng(seed)
    x, y, th = sim.free_pose(g, rng)
    scan = oracle.map_scan(g, 0.05, (0, 0), x, y, th, 360, TAU, 10.0)
    scan = (scan + rng.normal(0, 0.01, scan.size)).astype(np.float32)
    hyp = oracle.gl_generate(g, 0.05, (0, 0), n_hyp // 16, 16, seed + 100)
    return g, (x, y, th), scan, hyp


def test_dispersion_bit_exact_vs_spec(kernels):
    g = sim.rooms_grid(5)
    gl = Gl(kernels, g, 64_000)
    try:
        assert kernels.pfgl_free_cells(gl.h) == int((g == 0).sum())
        assert kernels.pfgl_generate_yaws(gl.h, 4000, 16, 77) == 0
        got = np.zeros(3 * 64_000, np.float32)
        assert kernels.pfgl_get_hyps(gl.h, f32p(got)) == 0
        ref = oracle.gl_generate(g, 0.05, (0, 0), 4000, 16, 77)
        assert np.array_equal(got.reshape(-1, 3), ref)
        # plain pfgl_generate = one yaw per position
        assert kernels.pfgl_generate(gl.h, 1000, 9) == 0
        got1 = np.zeros(3000, np.float32)
        assert kernels.pfgl_get_hyps(gl.h, f32p(got1)) == 0
        assert np.array_equal(got1.reshape(-1, 3), oracle.gl_generate(g, 0.05, (0, 0), 1000, 1, 9))
    finally:
        gl.close()


def test_caer_matches_reference_on_fed_hypotheses(kernels, ref):
    g, truth, scan, hyp = _scene()
    n = len(hyp)
    ours, theirs = Gl(kernels, g, n), Gl(ref, g, n)
    try:
        flat = np.ascontiguousarray(hyp.reshape(-1))
        assert kernels.pfgl_set_hyps(ours.h, f32p(flat), n) == 0
        assert ref.ref_gl_set_hyps(theirs.h, f32p(flat), n) == 0
        assert kernels.pfgl_score(ours.h, f32p(scan), scan.size, 10.0, TAU) == 0
        assert ref.pfgl_score(theirs.h, f32p(scan), scan.size, 10.0, TAU) == 0
        a = np.zeros(n, np.float32)
        b = np.zeros(n, np.float32)
        assert kernels.pfgl_get_caer(ours.h, f32p(a)) == 0
        assert ref.ref_gl_get_caer(theirs.h, f32p(b)) == 0
        rel = np.abs(a.astype(np.float64) - b) / np.maximum(np.abs(b), 1e-3)
        print(f"CAER max rel diff {rel.max():.3e}, identical {np.mean(a == b):.4f}")
        assert rel.max() <= 1e-5
        # against the f32 CPU mirror (libm sin/cos may differ by an ulp,
        # which can move a grazing ray to a neighbouring cell)
        o = oracle.caer_f32(g, 0.05, (0, 0), scan, TAU, 10.0, hyp[:2000])
        relo = np.abs(a[:2000] - o) / np.maximum(o, 1e-3)
        assert np.mean(relo <= 1e-5) > 0.95
        # against the FP64 reference CPU path: same optimum region
        o64 = oracle.caer(g, 0.05, (0, 0), scan.astype(np.float64), TAU, 10.0,
                          hyp[:2000].astype(np.float64))
        assert np.median(np.abs(a[:2000] - o64) / np.maximum(o64, 1e-3)) < 1e-3
    finally:
        ours.close()
        theirs.close()


def test_topk_from_scores_bit_exact(kernels, ref):
    rng = np.random.default_rng(9)
    n = 300_000
    s = rng.integers(0, 5000, size=n).astype(np.float32) * np.float32(0.25)  # many ties
    s[rng.integers(0, n, 50)] = np.inf
    g = sim.room_grid()
    ours, theirs = Gl(kernels, g, n), Gl(ref, g, n)
    try:
        for k in (1, 64, 1000, 5000):
            idx = np.zeros(k, np.int32)
            assert kernels.pfgl_topk_from_scores(ours.h, f32p(s), n, k, i32p(idx)) == k
            assert np.array_equal(idx, oracle.topk_from_scores(s, k))
        assert ref.ref_gl_set_caer(theirs.h, f32p(s), n) == 0
        out = np.zeros(3 * 64, np.float32)
        assert ref.pfgl_topk(theirs.h, 64, f32p(out)) == 64
        vals = np.zeros(64, np.int32)
        assert ref.ref_gl_get_sorted(theirs.h, i32p(vals), 64) == 0
        idx = np.zeros(64, np.int32)
        kernels.pfgl_topk_from_scores(ours.h, f32p(s), n, 64, i32p(idx))
        assert np.array_equal(idx, vals)
    finally:
        ours.close()
        theirs.close()


def test_topk_full_path_and_clamps(kernels):
    g, truth, scan, hyp = _scene(seed=4, n_hyp=4096)
    n = len(hyp)
    gl = Gl(kernels, g, n)
    try:
        flat = np.ascontiguousarray(hyp.reshape(-1))
        kernels.pfgl_set_hyps(gl.h, f32p(flat), n)
        assert kernels.pfgl_score(gl.h, f32p(scan), scan.size, 10.0, TAU) == 0
        caer = np.zeros(n, np.float32)
        kernels.pfgl_get_caer(gl.h, f32p(caer))
        out = np.zeros(3 * n, np.float32)
        cs = np.zeros(n, np.float32)
        idx = np.zeros(n, np.int32)
        assert kernels.pfgl_topk_ex(gl.h, n + 50, f32p(out), f32p(cs), i32p(idx)) == n
        assert np.array_equal(idx, oracle.topk_from_scores(caer, n))
        assert np.array_equal(out.reshape(-1, 3), hyp[idx])
        assert np.array_equal(cs, caer[idx])
        assert kernels.pfgl_topk(gl.h, 0, f32p(out)) == -1
        top3 = np.zeros(9, np.float32)
        assert kernels.pfgl_topk(gl.h, 3, f32p(top3)) == 3
        assert np.array_equal(top3.reshape(-1, 3), hyp[idx[:3]])
    finally:
        gl.close()


# 200k (two chunks) and 1M (four) run the pruned scorer in chunks with the
# bound tightened between them (k <= 128); k = 200 keeps the seed batch's
# bound throughout.
@pytest.mark.parametrize("n_hyp,k", [(20_000, 64), (200_000, 64), (200_000, 10),
                                     (1_000_000, 64), (1_000_000, 200)])
def test_pruned_localize_equals_exhaustive(kernels, n_hyp, k):
    g, truth, scan, _ = _scene(seed=6)
    gl = Gl(kernels, g, n_hyp)
    try:
        assert kernels.pfgl_generate_yaws(gl.h, n_hyp // 16, 16, 31) == 0
        o1 = np.zeros(3 * k, np.float32)
        c1 = np.zeros(k, np.float32)
        i1 = np.zeros(k, np.int32)
        assert kernels.pfgl_localize(gl.h, f32p(scan), scan.size, 10.0, TAU, k, f32p(o1),
                                     f32p(c1), i32p(i1)) == k
        assert kernels.pfgl_score(gl.h, f32p(scan), scan.size, 10.0, TAU) == 0
        o2 = np.zeros(3 * k, np.float32)
        c2 = np.zeros(k, np.float32)
        i2 = np.zeros(k, np.int32)
        assert kernels.pfgl_topk_ex(gl.h, k, f32p(o2), f32p(c2), i32p(i2)) == k
        assert np.array_equal(i1, i2)
        assert np.array_equal(c1, c2)
        assert np.array_equal(o1, o2)
    finally:
        gl.close()


def test_cuda_matches_cpu_ranking():
    # crates/pf_core/tests/global_loc.rs:69-129 through the host layer
    g = sim.room_grid()
    truth = (6.0, 7.0, 0.8)
    scan64 = oracle.map_scan(g, 0.05, (0, 0), *truth, 360, TAU, 10.0)
    gl = pkg.GlobalLoc(g, hypotheses=30_000, topk=10, seed=42)
    assert gl.free_cells() > 0
    gpu_top = gl.localize(scan64.astype(np.float32))
    cpu_top = oracle.gl_localize(g, 0.05, (0, 0), scan64, TAU, 10.0, 30_000, 10, 42)
    best = min(math.hypot(a[0] - b[0], a[1] - b[1]) for a in gpu_top for b in cpu_top)
    assert best < 0.5
    b = gpu_top[0]
    assert math.hypot(b[0] - truth[0], b[1] - truth[1]) < 0.5
    assert all(math.isnan(h[3]) for h in gpu_top)
    gl.close()


def test_start_outside_map_scores_rmax(kernels):
    g = sim.room_grid()
    gl = Gl(kernels, g, 4)
    try:
        hyp = np.array([[-1.0, 5.0, 0.0], [5.0, 11.0, 0.0], [5.0, 5.0, 0.0], [5.0, 5.0, 1.0]],
                       np.float32).reshape(-1)
        assert kernels.pfgl_set_hyps(gl.h, f32p(hyp), 4) == 0
        scan = np.full(8, 10.0, np.float32)
        assert kernels.pfgl_score(gl.h, f32p(scan), 8, 10.0, TAU) == 0
        c = np.zeros(4, np.float32)
        kernels.pfgl_get_caer(gl.h, f32p(c))
        assert c[0] == 0.0 and c[1] == 0.0  # outside: every ray returns rmax
        assert c[2] > 0.0
        # nrays == 1: a single ray along theta
        assert kernels.pfgl_score(gl.h, f32p(scan), 1, 10.0, TAU) == 0
        kernels.pfgl_get_caer(gl.h, f32p(c))
        d = oracle.cast_ray(g, 0.05, (0, 0), 5.0, 5.0, 1.0, 0.0, 10.0)
        assert abs(c[2] - (10.0 - d)) < 1e-4
    finally:
        gl.close()


@pytest.mark.parametrize("n", [1, 100, 2048, 2049, 20_000, 65_536])
def test_small_bottom_k_select_equals_full_sort(kernels, n):
    """pfgl_topk_ex picks the block select for n <= 65536 and k <= 128 and
    the radix sort otherwise; both must return the same (CAER, index) order,
    ties included (each hypothesis appears three times, so equal CAERs are
    common and the lower index must come first)."""
    g, _, scan, hyp = _scene(seed=9, n_hyp=max(16, (n + 2) // 3 + 16))
    fed = np.repeat(hyp[: (n + 2) // 3], 3, axis=0)[:n]
    gl = Gl(kernels, g, 70_000)
    try:
        assert kernels.pfgl_set_hyps(gl.h, f32p(np.ascontiguousarray(fed, np.float32)), n) == 0
        assert kernels.pfgl_score(gl.h, f32p(scan), 360, 10.0, TAU) == 0
        caer = np.zeros(n, np.float32)
        assert kernels.pfgl_get_caer(gl.h, f32p(caer)) == 0
        for k in (1, 7, 64, 128, 129):
            kk = min(k, n)
            out = np.zeros(3 * kk, np.float32)
            cs = np.zeros(kk, np.float32)
            idx = np.zeros(kk, np.int32)
            assert kernels.pfgl_topk_ex(gl.h, k, f32p(out), f32p(cs), i32p(idx)) == kk
            ref = np.zeros(kk, np.int32)
            assert kernels.pfgl_topk_from_scores(gl.h, f32p(caer), n, kk, i32p(ref)) == kk
            assert np.array_equal(idx, ref), (n, k)
            assert np.array_equal(cs, caer[ref])
            assert np.array_equal(out.reshape(-1, 3), fed[ref].astype(np.float32))
            # pfgl_topk_from_scores left caller scores in place of the CAERs
            assert kernels.pfgl_score(gl.h, f32p(scan), 360, 10.0, TAU) == 0
    finally:
        gl.close()


def test_large_map_scoring_reads_grid_from_global_memory(kernels, ref):
    """A 30 x 30 m room (600 x 600 cells, 356 KB padded) does not fit the
    scorers' shared-memory grid copy, so they read the grid from global
    memory: CAERs against the reference on fed hypotheses (1e-5 relative,
    as on the small map) and the pruned localizer against exhaustive
    scoring there."""
    g = sim.rooms_grid(21, n_boxes=120, size_m=30.0)
    rng = np.random.default_rng(21)
    x, y, th = sim.free_pose(g, rng)
    scan = oracle.map_scan(g, 0.05, (0, 0), x, y, th, 360, TAU, 10.0)
    scan = (scan + rng.normal(0, 0.01, scan.size)).astype(np.float32)
    hyp = oracle.gl_generate(g, 0.05, (0, 0), 4000 // 16, 16, 77)
    n = len(hyp)
    ours, theirs = Gl(kernels, g, 40_000), Gl(ref, g, n)
    try:
        flat = np.ascontiguousarray(hyp.reshape(-1))
        assert kernels.pfgl_set_hyps(ours.h, f32p(flat), n) == 0
        assert ref.ref_gl_set_hyps(theirs.h, f32p(flat), n) == 0
        assert kernels.pfgl_score(ours.h, f32p(scan), scan.size, 10.0, TAU) == 0
        assert ref.pfgl_score(theirs.h, f32p(scan), scan.size, 10.0, TAU) == 0
        a = np.zeros(n, np.float32)
        b = np.zeros(n, np.float32)
        assert kernels.pfgl_get_caer(ours.h, f32p(a)) == 0
        assert ref.ref_gl_get_caer(theirs.h, f32p(b)) == 0
        rel = np.abs(a.astype(np.float64) - b) / np.maximum(np.abs(b), 1e-3)
        assert rel.max() <= 1e-5, rel.max()
        # pruned localizer (small-set path: seed batch, bound, survivors)
        # against exhaustive scoring on 40 000 hypotheses of this map
        k = 64
        assert kernels.pfgl_generate_yaws(ours.h, 40_000 // 16, 16, 5) == 0
        o1 = np.zeros(3 * k, np.float32)
        c1 = np.zeros(k, np.float32)
        i1 = np.zeros(k, np.int32)
        assert kernels.pfgl_localize(ours.h, f32p(scan), scan.size, 10.0, TAU, k, f32p(o1),
                                     f32p(c1), i32p(i1)) == k
        assert kernels.pfgl_score(ours.h, f32p(scan), scan.size, 10.0, TAU) == 0
        c2 = np.zeros(k, np.float32)
        i2 = np.zeros(k, np.int32)
        assert kernels.pfgl_topk_ex(ours.h, k, None, f32p(c2), i32p(i2)) == k
        assert np.array_equal(i1, i2) and np.array_equal(c1, c2)
    finally:
        ours.close()
        theirs.close()


def _select_cases(rng, n):
    """Score arrays that stress the radix select's range narrowing: spread,
    all equal (ties resolved by the index word alone), two values, 60 decades,
    infinities, negative scores."""
    yield "uniform", rng.uniform(50, 3000, n)
    yield "equal", np.full(n, 7.0)
    yield "two", rng.choice([1.0, 2.0], n)
    yield "decades", 10.0 ** rng.uniform(-30, 30, n)
    c = rng.uniform(0, 1, n)
    c[::7] = np.inf
    yield "inf", c
    yield "signed", rng.normal(0, 100, n)


@pytest.mark.parametrize("n", [1, 2, 100, 2048, 2049, 20_000, 65_536])
def test_select_from_scores_equals_oracle_order(kernels, n):
    """pfgl_select_from_scores (the one-block radix select of the fused
    localizers) against the oracle's stable sort of the same scores, with and
    without dropped (negative) scores sorted last."""
    g, _, _, _ = _scene(seed=9, n_hyp=16)
    gl = Gl(kernels, g, 70_000)
    rng = np.random.default_rng(n)
    try:
        for name, c in _select_cases(rng, n):
            s = np.ascontiguousarray(c, np.float32)
            for k in (1, 64, 128):
                kk = min(k, n)
                got = np.zeros(kk, np.int32)
                assert kernels.pfgl_select_from_scores(gl.h, f32p(s), n, k, 0, i32p(got)) == kk
                assert np.array_equal(got, oracle.topk_from_scores(s, k)), (name, n, k)
        # dropped last: the oracle sees a dropped score as NaN (after +inf)
        for frac in (0.0, 0.5, 0.97):
            s = rng.uniform(50, 3000, n).astype(np.float32)
            s[rng.random(n) < frac] = -1.0
            if n >= 3:
                s[: n // 3] = np.where(s[: n // 3] < 0, -1.0, 9.0)  # ties among valid
            ref_s = np.where(s < 0, np.float32(np.nan), s).astype(np.float32)
            for k in (1, 64, 128):
                kk = min(k, n)
                got = np.zeros(kk, np.int32)
                assert kernels.pfgl_select_from_scores(gl.h, f32p(s), n, k, 1, i32p(got)) == kk
                assert np.array_equal(got, oracle.topk_from_scores(ref_s, k)), (frac, n, k)
        # k above the select's limit of 128 is refused
        if n >= 129:
            big = np.zeros(129, np.int32)
            assert kernels.pfgl_select_from_scores(gl.h, f32p(s), n, 129, 0, i32p(big)) == -1
    finally:
        gl.close()


def test_visit_count_matches_oracle_dda(kernels):
    """pfgl_count_visits replays the scorer's DDA: its count of cell steps
    agrees with the oracle's f32 DDA.  The oracle takes its ray directions
    from host cos/sin, which can differ from the device's sincosf in the last
    bit and so, rarely, send a ray through a different cell; the bar is
    1e-3 of the total."""
    g, _, scan, hyp = _scene(seed=13, n_hyp=2000)
    n = len(hyp)
    gl = Gl(kernels, g, 4000)
    try:
        assert kernels.pfgl_set_hyps(gl.h, f32p(np.ascontiguousarray(hyp, np.float32)), n) == 0
        got = kernels.pfgl_count_visits(gl.h, 360, TAU)
        ref = oracle.dda_visits(g, 0.05, (0, 0), hyp, 360, TAU)
        print(f"\nDDA visits: device {got}, oracle {ref}")
        assert ref > 0 and abs(got - ref) <= 1e-3 * ref
    finally:
        gl.close()
