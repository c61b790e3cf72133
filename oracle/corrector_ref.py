"""CPU restatement of the learned corrector -- TEST INFRASTRUCTURE ONLY.

Float64 numpy forward and backward passes of the 3-layer 3x3 corrector
(4 -> 16 -> 16 -> 1 channels, bias-free, ReLU between layers) that
libfomo_b200 runs on BF16 tensor cores.  There is no reference counterpart
(the corrector is new); the restatement is pinned by finite differences in the
CPU tests and is the checker of the GPU gradients.

``bf16=True`` rounds, as the GPU path stores them, the weights, the stored
activations (h1, h2) and the propagated gradients (dy3, dh2, dh1) to bfloat16
(round to nearest even), so the remaining difference to the GPU is FP32
accumulation order only.

Layout: images (n, h, w, c) with x fastest; parameters flat
W1[9][6][16], W2[9][16][16], W3[9][16]; tap = 3*(dz+1) + (dx+1) reads the
input at (z+dz, x+dx) with zero padding.
"""
from __future__ import annotations

import numpy as np

CIN, HID = 6, 16
N1, N2, N3 = 9 * CIN * HID, 9 * HID * HID, 9 * HID
NPARAM = N1 + N2 + N3


def bf16_round(a: np.ndarray) -> np.ndarray:
    """Round to bfloat16 (nearest even), returned as float64."""
    f = np.asarray(a, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return r.view(np.float32).astype(np.float64)


def split(params):
    p = np.asarray(params, dtype=np.float64)
    w1 = p[:N1].reshape(9, CIN, HID)
    w2 = p[N1:N1 + N2].reshape(9, HID, HID)
    w3 = p[N1 + N2:].reshape(9, HID, 1)
    return w1, w2, w3


def conv(x, w):
    """y[p, co] = sum_tap sum_ci x[p + off(tap), ci] w[tap, ci, co]."""
    n, h, ww, _ = x.shape
    xp = np.pad(x, ((0, 0), (1, 1), (1, 1), (0, 0)))
    y = np.zeros((n, h, ww, w.shape[2]))
    for tap in range(9):
        dz, dx = tap // 3, tap % 3
        y += xp[:, dz:dz + h, dx:dx + ww, :] @ w[tap]
    return y


def conv_wgrad(x, dy):
    """dW[tap, ci, co] = sum_p x[p + off(tap), ci] dy[p, co]."""
    n, h, ww, ci = x.shape
    xp = np.pad(x, ((0, 0), (1, 1), (1, 1), (0, 0)))
    d = dy.reshape(-1, dy.shape[-1])
    out = np.zeros((9, ci, dy.shape[-1]))
    for tap in range(9):
        dz, dx = tap // 3, tap % 3
        out[tap] = xp[:, dz:dz + h, dx:dx + ww, :].reshape(-1, ci).T @ d
    return out


def conv_dgrad(dy, w):
    """dx[p, ci] = sum_tap sum_co dy[p - off(tap), co] w[tap, ci, co]."""
    n, h, ww, _ = dy.shape
    dp = np.pad(dy, ((0, 0), (1, 1), (1, 1), (0, 0)))
    dx = np.zeros((n, h, ww, w.shape[1]))
    for tap in range(9):
        dz, dxx = 2 - tap // 3, 2 - tap % 3
        dx += dp[:, dz:dz + h, dxx:dxx + ww, :] @ w[tap].T
    return dx


def forward(feat, params, bf16=False):
    """feat (n, h, w, 4) -> y (n, h, w) plus the saved activations."""
    r = bf16_round if bf16 else (lambda a: np.asarray(a, dtype=np.float64))
    w1, w2, w3 = (r(w) for w in split(params))
    x = r(feat)
    h1 = r(np.maximum(conv(x, w1), 0.0))
    h2 = r(np.maximum(conv(h1, w2), 0.0))
    y = conv(h2, w3)[..., 0]
    return y, (x, h1, h2, w1, w2, w3)


def loss_and_grad(feat, target, params, mask=None, bf16=False):
    """Mean over pixels of (mask * (y - target))^2 and its parameter gradient."""
    r = bf16_round if bf16 else (lambda a: np.asarray(a, dtype=np.float64))
    y, (x, h1, h2, w1, w2, w3) = forward(feat, params, bf16)
    m = 1.0 if mask is None else np.asarray(mask, dtype=np.float64)
    res = m * (y - np.asarray(target, dtype=np.float64))
    count = y.size
    loss = float(np.sum(res * res) / count)
    dy3 = r(2.0 * res / count)[..., None]
    g3 = conv_wgrad(h2, dy3)
    dh2 = r(conv_dgrad(dy3, w3) * (h2 > 0))
    g2 = conv_wgrad(h1, dh2)
    dh1 = r(conv_dgrad(dh2, w2) * (h1 > 0))
    g1 = conv_wgrad(x, dh1)
    grad = np.concatenate([g1.ravel(), g2.ravel(), g3.ravel()])
    return loss, grad, y


def features(u, u_prev, c2, s_next=None, s_prev=None):
    """(u, u_prev, c2 u, c2^2 u, s_next, s_prev) stacked on the last axis;
    s_* are images of the injected values (0 away from the sources)."""
    u, up, c = (np.asarray(a, dtype=np.float64) for a in (u, u_prev, c2))
    z = np.zeros_like(u)
    sn = z if s_next is None else np.asarray(s_next, dtype=np.float64)
    sp = z if s_prev is None else np.asarray(s_prev, dtype=np.float64)
    return np.stack([u, up, c * u, c * c * u, sn, sp], axis=-1)
