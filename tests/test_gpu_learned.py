"""Learned proposal on the GPU: the tcgen05 GEMM against a torch fp32
reference, the network's loss and gradients against the FP64 oracle, and what
the trained proposal gains over uniform dispersion at equal hypothesis budget.
"""
import math

import numpy as np
import pytest
import torch

import cuda_pf_localization_b200 as pkg
from cuda_pf_localization_b200 import sim
from oracle import mlp_oracle as M

pytestmark = pytest.mark.gpu


def _bf16_bits(a: np.ndarray) -> np.ndarray:
    t = torch.from_numpy(np.ascontiguousarray(a, np.float32)).to(torch.bfloat16)
    return t.view(torch.int16).numpy().view(np.uint16)


def _bits_to_f32(b: np.ndarray) -> np.ndarray:
    return (b.astype(np.uint32) << 16).view(np.float32)


# the last two shapes give at least 148 tiles of 128 x 256 and so run the
# wide-tile kernel; the others the 128 x 128 one
@pytest.mark.parametrize("M_, N_, K_", [(128, 128, 64), (256, 384, 320), (512, 1024, 1024),
                                         (1024, 384, 2048), (8192, 1024, 128),
                                         (9472, 512, 64)])
def test_gemm_matches_torch_fp32(kernels, M_, N_, K_):
    rng = np.random.default_rng(M_ + N_ + K_)
    a = _bf16_bits(rng.normal(0, 1, (M_, K_)))
    b = _bf16_bits(rng.normal(0, 1, (N_, K_)))
    d = pkg.learned_gemm(a, b)
    ref = (torch.from_numpy(_bits_to_f32(a)) @ torch.from_numpy(_bits_to_f32(b)).T).numpy()
    # products of bf16 values are exact in f32; only the summation order
    # differs: |err| <= K * 2^-23 * sum |a||b| bounds it comfortably.
    bound = K_ * 2.0 ** -23 * (np.abs(_bits_to_f32(a)) @ np.abs(_bits_to_f32(b)).T)
    assert np.all(np.abs(d - ref) <= bound + 1e-6), np.max(np.abs(d - ref))
    # every tile of the output is written (catches skipped tiles)
    assert np.count_nonzero(d == 0.0) < d.size // 1000 + 1


def _gl(seed=3, cap=1 << 16):
    lib = pkg.kernels()
    g = np.ascontiguousarray(sim.rooms_grid(seed))
    h = lib.pfgl_create(200, 200, 0.05, 0.0, 0.0, pkg.u8ptr(g), cap)
    assert h
    return lib, g, h


def _batch(rng, b):
    x = np.zeros((b, M.IN), np.float32)
    x[:, :360] = rng.uniform(0.02, 1.0, (b, 360))
    th = rng.uniform(0, 2 * np.pi, b)
    y = np.stack([rng.uniform(-0.9, 0.9, b), rng.uniform(-0.9, 0.9, b), np.cos(th),
                  np.sin(th)], 1).astype(np.float32)
    return x, y


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


# batch 8192 (the training batch) runs the forward and input-gradient GEMMs
# on 128 x 256 tiles over every SM, batch 128 on 128 x 128 tiles
@pytest.mark.parametrize("batch", [128, 8192])
def test_learned_grad_matches_fp64_oracle(kernels, batch):
    lib, _, h = _gl()
    lp = pkg.LearnedProposal(h, batch=batch, seed=5)
    try:
        rng = np.random.default_rng(11)
        flat = lp.params()
        # nonzero biases everywhere so every bias gradient path is exercised
        layers = M.unflatten(flat)
        for l, (w, b) in enumerate(layers):
            n_used = M.USED if l == M.LAYERS - 1 else len(b)
            b[:n_used] += rng.normal(0, 0.05, n_used).astype(np.float32)
        flat = M.flatten(layers).astype(np.float32)
        lp.set_params(flat)
        assert np.array_equal(lp.params(), flat)
        x, y = _batch(rng, batch)
        loss, g = lp.grad(x, y)
        ref_loss, ref = M.loss_and_grad(M.unflatten(flat.astype(np.float64)),
                                        x.astype(np.float64), y.astype(np.float64))
        assert abs(loss - ref_loss) <= 1e-4 * abs(ref_loss), (loss, ref_loss)
        gl = M.unflatten(g.astype(np.float64))
        # Tolerance: the back-propagated gradient is rounded to bf16 after each
        # input-gradient GEMM, so f32-vs-f64 accumulation order flips some
        # roundings.  The oracle evaluated once with f32 and once with f64
        # accumulation differs by ~5e-3 (norm-relative) in layers 0-3 and
        # ~5e-4 in layer 4 on this kind of input; the bars are 3x that.
        errs = []
        for l in range(M.LAYERS):
            tol = 3e-3 if l == M.LAYERS - 1 else 1.5e-2
            rw = _rel(gl[l][0], ref[l][0])
            rb = _rel(gl[l][1], ref[l][1])
            errs.append((l, rw, rb))
            assert rw <= tol and rb <= tol, errs
        # padding rows of the output layer receive no gradient
        assert np.all(gl[-1][0][M.USED:] == 0) and np.all(gl[-1][1][M.USED:] == 0)
        # forward output against the oracle's Z4: f32 accumulation order plus
        # the bf16 roundings of the hidden activations it flips (measured
        # 2.9e-4 norm-relative)
        z = lp.forward(x[:7])
        _, z_ref = M.forward(M.unflatten(flat.astype(np.float64)), x[:7].astype(np.float64))
        assert _rel(z, z_ref[:, :M.USED]) <= 1e-3
    finally:
        lp.close()
        lib.pfgl_destroy(h)


def test_training_step_matches_oracle_adam(kernels):
    """One Adam step on device pairs equals the FP64 Adam update of the
    device's own gradient (moments start at zero, so the first step moves
    every weight with a nonzero gradient by lr * sign(g) (1 - tiny))."""
    lib, _, h = _gl()
    lp = pkg.LearnedProposal(h, batch=128, seed=9)
    try:
        lp.make_data(128, seed=4)
        before = lp.params()
        loss = lp.train(1, total_steps=1, lr=1e-3)
        after = lp.params()
        assert np.isfinite(loss[0]) and loss[0] != 0
        step = after - before
        moved = np.abs(step) > 0
        assert moved.mean() > 0.5
        # |step| = lr * |g| / (|g| + eps) <= lr (warm-up of one step: lr_t = lr)
        assert np.max(np.abs(step)) <= 1e-3 * (1 + 1e-5)
    finally:
        lp.close()
        lib.pfgl_destroy(h)


def _err(top, truth):
    dp = math.hypot(top[0] - truth[0], top[1] - truth[1])
    dth = abs((top[2] - truth[2] + math.pi) % (2 * math.pi) - math.pi)
    return dp, dth


def test_learned_proposal_beats_uniform_at_equal_budget(kernels):
    """Trained per-map proposal vs uniform dispersion, both scoring 20k
    hypotheses with plain CAER on unseen poses."""
    lib, g, h = _gl(seed=21, cap=200_000)
    lp = pkg.LearnedProposal(h, batch=1024, seed=3)
    try:
        lp.make_data(524_288, seed=17)
        losses = lp.train(2500, lr=1e-3)
        assert np.all(np.isfinite(losses))
        assert losses[-100:].mean() < losses[:100].mean() - 1.0
        tau, held_out = lp.calibrate(n_queries=100, n_samples=20000, seed=123)
        rng = np.random.default_rng(77)
        poses = np.array([sim.free_pose(g, rng) for _ in range(100)], np.float32)
        scans = pkg.render_scans(h, poses, noise=0.01, seed=555)
        ok_l = ok_u = 0
        out = np.zeros(3, np.float32)
        for q in range(len(poses)):
            top, caer, _, _ = lp.localize(scans[q], n_samples=20000, n_fallback=0, k=1)
            dp, dth = _err(top[0], poses[q])
            ok_l += dp <= 0.5 and dth <= 0.1
            assert lib.pfgl_generate_yaws(h, 1250, 16, 1000 + q) == 0
            assert lib.pfgl_localize(h, pkg.fptr(scans[q]), 360, 10.0, 2 * np.pi, 1,
                                     pkg.fptr(out), None, None) == 1
            dp, dth = _err(out, poses[q])
            ok_u += dp <= 0.5 and dth <= 0.1
        print(f"\nlearned {ok_l}/100 uniform {ok_u}/100 held-out {held_out:.2f} tau {tau:.1f}"
              f" loss {losses[:50].mean():.2f}->{losses[-50:].mean():.2f}")
        assert ok_l >= 85
        assert ok_l >= ok_u + 20
    finally:
        lp.close()
        lib.pfgl_destroy(h)


def test_learned_query_graph_equals_direct(kernels):
    """A learned query replayed from its CUDA graph gives the same poses,
    CAERs and indices as the same query launched kernel by kernel (two
    proposals with identical weights, seed and query counter), including
    after a change of sample count and k (re-capture)."""
    lib, g, h = _gl(seed=21, cap=200_000)
    lp1 = pkg.LearnedProposal(h, batch=1024, seed=3)
    lp2 = None
    try:
        lp1.make_data(65_536, seed=17)
        lp1.train(200, lr=1e-3)
        lp2 = pkg.LearnedProposal(h, batch=1024, seed=3)
        lp2.set_params(lp1.params())
        lp2.use_graph(False)
        rng = np.random.default_rng(5)
        poses = np.array([sim.free_pose(g, rng) for _ in range(6)], np.float32)
        scans = pkg.render_scans(h, poses, noise=0.01, seed=99)
        for n_samples, k in ((20_000, 64), (5_000, 8)):
            for q in range(len(poses)):
                a = lp1.localize(scans[q], n_samples=n_samples, n_fallback=0, k=k)
                b = lp2.localize(scans[q], n_samples=n_samples, n_fallback=0, k=k)
                for x, y in zip(a[:3], b[:3]):
                    assert np.array_equal(x, y), (n_samples, k, q)
                assert a[3] == b[3]
    finally:
        if lp2 is not None:
            lp2.close()
        lp1.close()
        lib.pfgl_destroy(h)
