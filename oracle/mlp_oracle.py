"""FP64 CPU oracle of the learned-proposal network — TEST INFRASTRUCTURE ONLY.

Imported only by tests/ (and __graft_entry__.smoke()) as the checker of the
library's tcgen05 forward/backward kernels; never by the product.

The network and loss restate the library's definition (the learned proposal
has no counterpart in the reference project):

    Z_l = H_{l-1} W_l^T + b_l,  H_l = relu(Z_l)   (l = 0..3, H_{-1} = X)
    Z_4 = H_3 W_4^T + b_4                          (288 of 384 outputs used)
    mixture of 32 diagonal Gaussians over (x_n, y_n, cos, sin):
      log pi = logits - LSE(logits)
      log sigma = LS_LO + (LS_HI - LS_LO) * sigmoid(raw)
      loss = mean_b -LSE_c(log pi_c - sum_d [z^2/2 + log sigma + log(2 pi)/2])

``loss_and_grad(..., bf16=True)`` evaluates in FP64 but rounds to bf16 at the
points where the device stores bf16 (weights, inputs, activations and the
back-propagated gradients), so the remaining difference to the device is the
f32 accumulation order only.  ``bf16=False`` is the exact FP64 function used
by the finite-difference self-check.
"""
from __future__ import annotations

import numpy as np

IN, HID, OUT, COMP, LAYERS = 384, 1024, 384, 32, 5
USED = COMP * 9
MEAN_OFF, SIG_OFF = COMP, COMP + 4 * COMP
LS_LO, LS_HI = -5.5, 0.0
HALF_LOG_2PI = 0.5 * np.log(2.0 * np.pi)


def layer_dims(l: int) -> tuple[int, int]:
    """(out, in) of layer l over the padded widths."""
    return (OUT if l == LAYERS - 1 else HID), (IN if l == 0 else HID)


def num_params() -> int:
    return sum(o * i + o for o, i in (layer_dims(l) for l in range(LAYERS)))


def unflatten(flat: np.ndarray) -> list[tuple[np.ndarray, np.ndarray]]:
    out, off = [], 0
    for l in range(LAYERS):
        o, i = layer_dims(l)
        w = flat[off:off + o * i].reshape(o, i)
        off += o * i
        b = flat[off:off + o]
        off += o
        out.append((w, b))
    return out


def flatten(layers) -> np.ndarray:
    return np.concatenate([np.concatenate([w.ravel(), b.ravel()]) for w, b in layers])


def bf16_round(x: np.ndarray) -> np.ndarray:
    """Round to the nearest bf16 (ties to even) through f32, as float64."""
    f = np.ascontiguousarray(x, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def mixture_loss_grad(z: np.ndarray, y: np.ndarray):
    """Mean loss over rows and dloss/dz (rows x OUT; padding columns zero)."""
    B = z.shape[0]
    logit = z[:, :COMP]
    mu = z[:, MEAN_OFF:MEAN_OFF + 4 * COMP].reshape(B, COMP, 4)
    raw = z[:, SIG_OFF:SIG_OFF + 4 * COMP].reshape(B, COMP, 4)
    mx = logit.max(axis=1, keepdims=True)
    lse_l = mx + np.log(np.exp(logit - mx).sum(axis=1, keepdims=True))
    logpi = logit - lse_l
    pi = np.exp(logpi)
    s = 1.0 / (1.0 + np.exp(-raw))
    ls = LS_LO + (LS_HI - LS_LO) * s
    sig = np.exp(ls)
    zz = (y[:, None, :] - mu) / sig
    nll = (0.5 * zz * zz + ls).sum(axis=2) + 4 * HALF_LOG_2PI
    a = logpi - nll
    amx = a.max(axis=1, keepdims=True)
    logp = amx + np.log(np.exp(a - amx).sum(axis=1, keepdims=True))
    r = np.exp(a - logp)
    loss = float(-logp.mean())
    g = np.zeros_like(z)
    g[:, :COMP] = (pi - r) / B
    g[:, MEAN_OFF:MEAN_OFF + 4 * COMP] = (-r[:, :, None] * zz / sig / B).reshape(B, -1)
    g[:, SIG_OFF:SIG_OFF + 4 * COMP] = (
        r[:, :, None] * (1 - zz * zz) * (LS_HI - LS_LO) * s * (1 - s) / B).reshape(B, -1)
    return loss, g


def forward(layers, x: np.ndarray, bf16: bool = True):
    """Activations [X, H0..H3] and Z4 (rounded as the device stores them)."""
    rnd = bf16_round if bf16 else (lambda v: np.asarray(v, np.float64))
    hs = [rnd(x)]
    for l in range(LAYERS - 1):
        w, b = layers[l]
        hs.append(rnd(np.maximum(hs[-1] @ rnd(w).T + b, 0.0)))
    w, b = layers[-1]
    z4 = hs[-1] @ rnd(w).T + b
    return hs, z4


def loss_and_grad(layers, x: np.ndarray, y: np.ndarray, bf16: bool = True):
    """Mean mixture loss and the gradients [(dW_l, db_l)] of all layers."""
    rnd = bf16_round if bf16 else (lambda v: np.asarray(v, np.float64))
    hs, z4 = forward(layers, x, bf16)
    loss, g = mixture_loss_grad(z4, y)
    dz = rnd(g)
    grads = [None] * LAYERS
    for l in range(LAYERS - 1, -1, -1):
        w, _ = layers[l]
        grads[l] = (dz.T @ hs[l], dz.sum(axis=0))
        if l > 0:
            dz = rnd((dz @ rnd(w)) * (hs[l] > 0))
    return loss, grads


def mixture_pose_density(z_row: np.ndarray):
    """(pi, mu, sigma) of one output row: mixture weights, means and standard
    deviations over (x_n, y_n, cos, sin)."""
    logit = z_row[:COMP].astype(np.float64)
    pi = np.exp(logit - logit.max())
    pi /= pi.sum()
    mu = z_row[MEAN_OFF:MEAN_OFF + 4 * COMP].reshape(COMP, 4).astype(np.float64)
    raw = z_row[SIG_OFF:SIG_OFF + 4 * COMP].reshape(COMP, 4).astype(np.float64)
    sig = np.exp(LS_LO + (LS_HI - LS_LO) / (1.0 + np.exp(-raw)))
    return pi, mu, sig
