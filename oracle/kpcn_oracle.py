"""CPU oracle of the learned denoiser's arithmetic (test infrastructure only:
tests and smoke() call it to check the CUDA kernels; the product never does).

The reference has no learned part, so there is no reference code to follow:
these are restatements of the mathematics, in float64 numpy, with BF16
rounding (round to nearest even) applied at exactly the points where the GPU
stores BF16 tensors, so that the only GPU/oracle difference left is the
order of FP32 additions.

Layouts match the C ABI: activations NHWC (n, h, w, c); 3x3 weights
(9, cout, cin) with tap t = 3 * (dy + 1) + (dx + 1); stride 1, zero padding 1.
"""
from __future__ import annotations

import numpy as np

TAPS = [(t // 3 - 1, t % 3 - 1) for t in range(9)]


# ---------------------------------------------------------------------------
# BF16
# ---------------------------------------------------------------------------

def bf16_bits(x) -> np.ndarray:
    """float32 -> BF16 bit patterns (uint16), round to nearest even."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    r = ((u >> 16) & 1) + 0x7FFF
    return ((u + r) >> 16).astype(np.uint16)


def from_bf16_bits(b) -> np.ndarray:
    return (np.asarray(b, dtype=np.uint16).astype(np.uint32) << 16).view(np.float32)


def bf16_round(x) -> np.ndarray:
    """Values rounded to BF16, as float32."""
    return from_bf16_bits(bf16_bits(x))


# ---------------------------------------------------------------------------
# 3x3 convolution and its gradients (float64)
# ---------------------------------------------------------------------------

def _shift(a, dy, dx):
    """out[:, y, x] = a[:, y + dy, x + dx] (zero outside)."""
    n, h, w, c = a.shape
    p = np.zeros((n, h + 2, w + 2, c), dtype=np.float64)
    p[:, 1:h + 1, 1:w + 1] = a
    return p[:, 1 + dy:1 + dy + h, 1 + dx:1 + dx + w]


def conv3x3_forward(x, w, bias=None, relu=False):
    """sum_{t, c} x[p + off(t), c] * w[t][o][c] (+ bias, ReLU)."""
    x = np.asarray(x, dtype=np.float64)
    w = np.asarray(w, dtype=np.float64)
    out = np.zeros(x.shape[:3] + (w.shape[1],), dtype=np.float64)
    for t, (dy, dx) in enumerate(TAPS):
        out += _shift(x, dy, dx) @ w[t].T
    if bias is not None:
        out += np.asarray(bias, dtype=np.float64)
    if relu:
        out = np.maximum(out, 0.0)
    return out


def conv3x3_backward_data(g, w, mask=None):
    """grad_x[q, c] = sum_{t, o} g[q - off(t), o] * w[t][o][c], times
    (mask[q, c] > 0) when a mask (the layer input, a ReLU output) is given."""
    g = np.asarray(g, dtype=np.float64)
    w = np.asarray(w, dtype=np.float64)
    out = np.zeros(g.shape[:3] + (w.shape[2],), dtype=np.float64)
    for t, (dy, dx) in enumerate(TAPS):
        out += _shift(g, -dy, -dx) @ w[t]
    if mask is not None:
        out = out * (np.asarray(mask) > 0)
    return out


def conv3x3_backward_weights(x, g):
    """grad_w[t][o][c] = sum_p x[p + off(t), c] * g[p, o]."""
    x = np.asarray(x, dtype=np.float64)
    g = np.asarray(g, dtype=np.float64)
    gf = g.reshape(-1, g.shape[-1])
    return np.stack([gf.T @ _shift(x, dy, dx).reshape(-1, x.shape[-1]) for dy, dx in TAPS])


def transpose_taps(w):
    """(9, o, c) -> (9, c, o): the weights of the data-gradient convolution."""
    return np.ascontiguousarray(np.transpose(np.asarray(w), (0, 2, 1)))
