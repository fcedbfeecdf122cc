"""The CPU oracle of the denoiser's convolutions checks itself: its data and
weight gradients are the derivatives of its forward pass (finite
differences in float64), and BF16 rounding is round-to-nearest-even."""
import numpy as np

from oracle import kpcn_oracle as K


def test_bf16_rounding_is_nearest_even():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, -2.5, 0.0, 3.3e38, 1e-40], dtype=np.float32)
    r = K.bf16_round(x)
    assert r[0] == 1.0 and r[1] == 1.0  # tie rounds to even
    assert r[2] == np.float32(1.0 + 4 * 2 ** -8)
    assert r[3] == -2.5 and r[4] == 0.0
    b = K.bf16_bits(np.float32(1.0))
    assert int(np.asarray(b).reshape(-1)[0]) == 0x3F80
    np.testing.assert_array_equal(K.from_bf16_bits(K.bf16_bits(r)), r)


def test_conv_gradients_match_finite_differences():
    rng = np.random.default_rng(0)
    x = rng.normal(size=(2, 5, 4, 3))
    w = rng.normal(size=(9, 2, 3))
    g = rng.normal(size=(2, 5, 4, 2))
    # loss = sum(conv(x, w) * g): d/dx = backward_data(g, w), d/dw = backward_weights(x, g)
    gx = K.conv3x3_backward_data(g, w)
    gw = K.conv3x3_backward_weights(x, g)
    eps = 1e-6
    for idx in [(0, 0, 0, 0), (1, 4, 3, 2), (0, 2, 1, 1), (1, 0, 3, 0)]:
        d = np.zeros_like(x)
        d[idx] = eps
        num = ((K.conv3x3_forward(x + d, w) - K.conv3x3_forward(x - d, w)) * g).sum() / (2 * eps)
        assert abs(num - gx[idx]) < 1e-6 * max(1.0, abs(num))
    for idx in [(0, 0, 0), (4, 1, 2), (8, 0, 1), (3, 1, 0)]:
        d = np.zeros_like(w)
        d[idx] = eps
        num = ((K.conv3x3_forward(x, w + d) - K.conv3x3_forward(x, w - d)) * g).sum() / (2 * eps)
        assert abs(num - gw[idx]) < 1e-6 * max(1.0, abs(num))


def test_backward_data_with_relu_mask():
    rng = np.random.default_rng(1)
    g = rng.normal(size=(1, 3, 3, 2))
    w = rng.normal(size=(9, 2, 4))
    m = rng.normal(size=(1, 3, 3, 4))
    np.testing.assert_allclose(K.conv3x3_backward_data(g, w, m), K.conv3x3_backward_data(g, w) * (m > 0))


def test_network_gradient_matches_finite_differences():
    """Exact (float64, no BF16 rounding) U-Net: backward == d loss / d params."""
    rng = np.random.default_rng(2)
    n, h, w = 1, 8, 8
    nparams = sum(9 * co * ci + co for ci, co, _ in K.SPEC)
    params = rng.normal(size=nparams) * 0.1
    feat = np.zeros((n, h, w, 16))
    feat[..., :12] = rng.normal(size=(n, h, w, 12))
    noisy = np.abs(rng.normal(size=(n, h, w, 4)))
    ref = np.abs(rng.normal(size=(n, h, w, 4)))
    ident = lambda x: np.asarray(x, dtype=np.float64)

    def loss(p):
        a, logits, _ = K.kpcn_forward(p, feat, noisy, rnd=ident)
        return K.filter_loss_grad(logits, noisy, ref)[0]

    a, logits, _ = K.kpcn_forward(params, feat, noisy, rnd=ident)
    _, dl = K.filter_loss_grad(logits, noisy, ref)
    g = K.kpcn_backward(params, a, feat, dl, rnd=ident)
    # offsets of each layer's weights and bias
    offs, off = [], 0
    for ci, co, _ in K.SPEC:
        offs.append((off, off + 9 * co * ci))
        off += 9 * co * ci + co
    idx = []
    for wo, bo in offs:
        idx += [wo + int(rng.integers(0, bo - wo)), bo]
    eps = 1e-6
    for i in idx:
        d = np.zeros_like(params)
        d[i] = eps
        num = (loss(params + d) - loss(params - d)) / (2 * eps)
        assert abs(num - g[i]) <= 1e-5 * max(1e-3, abs(num)) + 1e-9, (i, num, g[i])
