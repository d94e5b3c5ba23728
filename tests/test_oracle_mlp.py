"""CPU checks of the learned-proposal oracle (oracle/mlp_oracle.py).

The oracle is the FP64 checker of the device's forward/backward kernels, so
its own gradient is pinned here by central finite differences of the exact
FP64 loss, and its bf16 rounding by torch's bf16 conversion.
"""
import numpy as np
import pytest
import torch

from oracle import mlp_oracle as M


def _params(rng, bias_scale=0.05):
    layers = []
    for l in range(M.LAYERS):
        o, i = M.layer_dims(l)
        bound = np.sqrt(6.0 / i) * (0.1 if l == M.LAYERS - 1 else 1.0)
        layers.append((rng.uniform(-bound, bound, (o, i)), rng.normal(0, bias_scale, o)))
    return layers


def _batch(rng, b):
    x = np.zeros((b, M.IN))
    x[:, :360] = rng.uniform(0, 1, (b, 360))
    th = rng.uniform(0, 2 * np.pi, b)
    y = np.stack([rng.uniform(-1, 1, b), rng.uniform(-1, 1, b), np.cos(th), np.sin(th)], 1)
    return x, y


def test_param_count_matches_layout():
    assert M.num_params() == (1024 * 384 + 1024) + 3 * (1024 * 1024 + 1024) + (384 * 1024 + 384)
    flat = np.arange(M.num_params(), dtype=np.float64)
    assert np.array_equal(M.flatten(M.unflatten(flat)), flat)


def test_bf16_rounding_matches_torch():
    rng = np.random.default_rng(0)
    v = np.concatenate([rng.normal(0, 1, 10000), rng.normal(0, 1e-30, 100),
                        np.array([0.0, -0.0, 1.0, 3.0039062, 1e38, -2.5e-3])])
    v = v.astype(np.float32)
    ref = torch.from_numpy(v).to(torch.bfloat16).to(torch.float32).numpy()
    assert np.array_equal(M.bf16_round(v).astype(np.float32), ref)


def test_mixture_gradient_finite_differences():
    rng = np.random.default_rng(1)
    z = rng.normal(0, 1, (6, M.OUT))
    _, y = _batch(rng, 6)
    loss, g = M.mixture_loss_grad(z, y)
    assert np.isfinite(loss)
    assert np.all(g[:, M.USED:] == 0)
    for _ in range(40):
        b, c = rng.integers(0, 6), rng.integers(0, M.USED)
        h = 1e-6
        zp, zm = z.copy(), z.copy()
        zp[b, c] += h
        zm[b, c] -= h
        fd = (M.mixture_loss_grad(zp, y)[0] - M.mixture_loss_grad(zm, y)[0]) / (2 * h)
        assert abs(fd - g[b, c]) <= 1e-6 * max(1.0, abs(g[b, c])) + 1e-8


def test_network_gradient_finite_differences():
    rng = np.random.default_rng(2)
    layers = _params(rng)
    x, y = _batch(rng, 4)
    loss, grads = M.loss_and_grad(layers, x, y, bf16=False)
    checked = 0
    for _ in range(30):
        l = int(rng.integers(0, M.LAYERS))
        which = int(rng.integers(0, 2))
        arr = layers[l][which]
        o = int(rng.integers(0, M.USED if l == M.LAYERS - 1 else arr.shape[0]))
        idx = (o, int(rng.integers(0, 360 if l == 0 else arr.shape[1]))) if which == 0 else (o,)
        h = 1e-5
        old = arr[idx]
        arr[idx] = old + h
        lp = M.loss_and_grad(layers, x, y, bf16=False)[0]
        arr[idx] = old - h
        lm = M.loss_and_grad(layers, x, y, bf16=False)[0]
        arr[idx] = old
        fd = (lp - lm) / (2 * h)
        an = grads[l][which][idx]
        assert abs(fd - an) <= 1e-5 * max(1e-3, abs(an)) + 1e-9, (l, which, idx, fd, an)
        checked += 1
    assert checked == 30


def test_bf16_emulation_close_to_exact():
    rng = np.random.default_rng(3)
    layers = _params(rng)
    x, y = _batch(rng, 16)
    l_exact, g_exact = M.loss_and_grad(layers, x, y, bf16=False)
    l_bf, g_bf = M.loss_and_grad(layers, x, y, bf16=True)
    assert abs(l_exact - l_bf) <= 2e-2 * abs(l_exact)
    for (gw, gb), (ew, eb) in zip(g_bf, g_exact):
        assert np.linalg.norm(gw - ew) <= 0.1 * np.linalg.norm(ew)
