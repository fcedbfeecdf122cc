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


# ---------------------------------------------------------------------------
# The kernel-predicting U-Net (forward, relMSE loss, backward)
# ---------------------------------------------------------------------------

# (cin, cout, relu) per layer: e0a e0b e1a e1b e2a e2b d1a d1b d0a d0b out
SPEC = [(16, 32, True), (32, 32, True), (32, 64, True), (64, 64, True), (64, 96, True), (96, 96, True),
        (160, 64, True), (64, 64, True), (96, 32, True), (32, 32, True), (32, 32, False)]
TAPS5 = 25
REL_EPS = 0.01


def unflatten(params):
    """Flat FP32 parameter vector -> [(w (9, cout, cin), b (cout,))] per layer."""
    out, off = [], 0
    for cin, cout, _ in SPEC:
        nw = 9 * cout * cin
        w = np.asarray(params[off:off + nw], dtype=np.float64).reshape(9, cout, cin)
        off += nw
        out.append((w, np.asarray(params[off:off + cout], dtype=np.float64)))
        off += cout
    assert off == len(params)
    return out


def flatten(layers):
    return np.concatenate([np.concatenate([w.ravel(), b.ravel()]) for w, b in layers])


def avgpool2(x, rnd=bf16_round):
    return rnd((x[:, 0::2, 0::2] + x[:, 0::2, 1::2] + x[:, 1::2, 0::2] + x[:, 1::2, 1::2]) * 0.25)


def up2(x):
    return np.repeat(np.repeat(x, 2, axis=1), 2, axis=2)


def down_sum(g):
    return g[:, 0::2, 0::2] + g[:, 0::2, 1::2] + g[:, 1::2, 0::2] + g[:, 1::2, 1::2]


def _gather5(noisy):
    """(n, h, w, 25, 3): the 5x5 neighbourhood, coordinates clamped."""
    n, h, w, _ = noisy.shape
    ys, xs = np.arange(h), np.arange(w)
    out = np.empty((n, h, w, TAPS5, 3), dtype=np.float64)
    for k in range(TAPS5):
        sy = np.clip(ys + k // 5 - 2, 0, h - 1)
        sx = np.clip(xs + k % 5 - 2, 0, w - 1)
        out[:, :, :, k, :] = noisy[:, sy][:, :, sx][..., :3]
    return out


def _softmax25(logits):
    l = np.asarray(logits, dtype=np.float64)[..., :TAPS5]
    e = np.exp(l - l.max(axis=-1, keepdims=True))
    return e / e.sum(axis=-1, keepdims=True)


def kpcn_forward(params, feat, noisy, rnd=bf16_round):
    """Activations (BF16-rounded where the GPU stores BF16), FP32-path filter
    logits (here float64) and the filtered radiance (n, h, w, 3). `rnd` is
    the BF16 rounding (identity for an exact float64 network)."""
    L = unflatten(params)
    a = {}

    def conv(i, x):
        w, b = L[i]
        return rnd(conv3x3_forward(x, rnd(w), b, relu=SPEC[i][2]))

    a["e0a"] = conv(0, feat)
    a["e0b"] = conv(1, a["e0a"])
    a["pool0"] = avgpool2(a["e0b"], rnd)
    a["e1a"] = conv(2, a["pool0"])
    a["e1b"] = conv(3, a["e1a"])
    a["pool1"] = avgpool2(a["e1b"], rnd)
    a["e2a"] = conv(4, a["pool1"])
    a["e2b"] = conv(5, a["e2a"])
    a["cat1"] = np.concatenate([up2(a["e2b"]), a["e1b"]], axis=-1)
    a["d1a"] = conv(6, a["cat1"])
    a["d1b"] = conv(7, a["d1a"])
    a["cat0"] = np.concatenate([up2(a["d1b"]), a["e0b"]], axis=-1)
    a["d0a"] = conv(8, a["cat0"])
    a["d0b"] = conv(9, a["d0a"])
    w, b = L[10]
    logits = conv3x3_forward(a["d0b"], rnd(w), b)
    out = np.einsum("...k,...kc->...c", _softmax25(logits), _gather5(noisy))
    return a, logits, out


def relmse(out, ref):
    ref = np.asarray(ref, dtype=np.float64)[..., :3]
    return float(np.mean((np.asarray(out)[..., :3] - ref) ** 2 / (ref ** 2 + REL_EPS)))


def filter_loss_grad(logits, noisy, ref):
    """relMSE loss of the filtered radiance and its gradient w.r.t. the
    logits ((n, h, w, 32), channels 25..31 zero)."""
    wgt = _softmax25(logits)
    nb = _gather5(noisy)
    o = np.einsum("...k,...kc->...c", wgt, nb)
    r = np.asarray(ref, dtype=np.float64)[..., :3]
    den = r ** 2 + REL_EPS
    P = o.shape[0] * o.shape[1] * o.shape[2]
    loss = float(np.sum((o - r) ** 2 / den) / (3 * P))
    go = 2 * (o - r) / den / (3 * P)
    dw = np.einsum("...c,...kc->...k", go, nb)
    dl = wgt * (dw - np.sum(wgt * dw, axis=-1, keepdims=True))
    g = np.zeros(logits.shape[:3] + (32,), dtype=np.float64)
    g[..., :TAPS5] = dl
    return loss, g


def kpcn_backward(params, a, feat, dlogits, rnd=bf16_round):
    """Parameter gradients (flat, same order as the parameters), with the
    GPU's BF16 rounding of every stored gradient tensor."""
    L = unflatten(params)
    grads = [None] * len(SPEC)

    def lb(i, x, g, mask, want_in=True):
        w, _ = L[i]
        grads[i] = (conv3x3_backward_weights(x, g), g.sum(axis=(0, 1, 2)))
        if not want_in:
            return None
        return rnd(conv3x3_backward_data(g, rnd(w), mask))

    gl = rnd(dlogits)
    ga = lb(10, a["d0b"], gl, a["d0b"])
    gb = lb(9, a["d0a"], ga, a["d0a"])
    gcat = lb(8, a["cat0"], gb, a["cat0"])
    g_d1b = rnd(down_sum(gcat[..., :64]))
    gsk0 = gcat[..., 64:96]
    gb = lb(7, a["d1a"], g_d1b, a["d1a"])
    gcat1 = lb(6, a["cat1"], gb, a["cat1"])
    g_e2b = rnd(down_sum(gcat1[..., :96]))
    gb = lb(5, a["e2a"], g_e2b, a["e2a"])
    gpool1 = lb(4, a["pool1"], gb, None)
    g_e1b = rnd((gcat1[..., 96:] + 0.25 * up2(gpool1)) * (a["e1b"] > 0))
    gb = lb(3, a["e1a"], g_e1b, a["e1a"])
    gpool0 = lb(2, a["pool0"], gb, None)
    g_e0b = rnd((gsk0 + 0.25 * up2(gpool0)) * (a["e0b"] > 0))
    gb = lb(1, a["e0a"], g_e0b, a["e0a"])
    lb(0, feat, gb, None, want_in=False)
    return flatten(grads)
