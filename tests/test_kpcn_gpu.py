"""The learned denoiser on the GPU: forward activations, filter logits, loss
and every parameter gradient against the CPU oracle (float64 with the GPU's
BF16 rounding points); training reduces the loss; features from a render."""
import numpy as np
import pytest

from oracle import kpcn_oracle as K

pytestmark = pytest.mark.gpu


def bf16_dev(a):
    import torch

    return torch.from_numpy(K.bf16_bits(a).view(np.int16)).view(torch.bfloat16).cuda()


def f32_dev(a):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).cuda()


def bf16_host(a):
    return K.from_bf16_bits(np.asarray(a).view(np.uint16))


def layer_slices():
    out, off = [], 0
    for ci, co, _ in K.SPEC:
        out.append((slice(off, off + 9 * co * ci), slice(off + 9 * co * ci, off + 9 * co * ci + co)))
        off += 9 * co * ci + co
    return out


def synthetic_batch(rng, n, h, w):
    feat = np.zeros((n, h, w, 16), np.float32)
    feat[..., :12] = rng.normal(size=(n, h, w, 12))
    feat = K.bf16_round(feat)
    noisy = np.abs(rng.normal(size=(n, h, w, 4))).astype(np.float32)
    ref = np.abs(rng.normal(size=(n, h, w, 4))).astype(np.float32)
    return feat, noisy, ref


def test_forward_loss_and_gradients_match_oracle(crt_ctx):
    from cudaraytracer_b200.kpcn import Kpcn

    rng = np.random.default_rng(11)
    n, h, w = 2, 16, 12
    feat, noisy, ref = synthetic_batch(rng, n, h, w)
    net = Kpcn(crt_ctx, seed=3)
    params = net.get_params()
    params[-32:-7] = rng.normal(size=25) * 0.3  # output bias: a non-uniform filter
    net.set_params(params)
    loss = net.train_step(bf16_dev(feat), f32_dev(noisy), f32_dev(ref), lr=0.0)
    grads = net.get_grads()
    logits = net.debug_tensor(10, (n, h, w, 32), np.float32)
    e0b = bf16_host(net.debug_tensor(1, (n, h, w, 32), np.int16))
    net.close()

    a, ref_logits, _ = K.kpcn_forward(params, feat, noisy)
    ref_loss, dl = K.filter_loss_grad(ref_logits, noisy, ref)
    ref_grads = K.kpcn_backward(params, a, feat, dl)

    # activations: BF16 values equal up to rare one-ulp rounding flips (and
    # ReLU kinks, where FP32 accumulation error decides the sign)
    assert np.mean(e0b != a["e0b"]) < 0.02
    assert np.allclose(e0b, a["e0b"], rtol=2 ** -7, atol=1e-4)
    err = np.linalg.norm(logits[..., :25] - ref_logits[..., :25]) / np.linalg.norm(ref_logits[..., :25])
    assert err < 5e-3
    assert not logits[..., 25:].any()
    assert abs(loss - ref_loss) <= 2e-3 * ref_loss
    # Weight gradients: relative error < 2e-2. Bias gradients are sums over
    # all pixels of a gradient that changes sign, so the same per-element
    # differences (FP32 order, rare BF16 rounding flips upstream) give a
    # larger relative error after cancellation: < 5e-2.
    for i, (ws, bs) in enumerate(layer_slices()):
        for sl, bound in ((ws, 2e-2), (bs, 5e-2)):
            r = ref_grads[sl]
            e = np.linalg.norm(grads[sl] - r) / max(np.linalg.norm(r), 1e-12)
            assert e < bound, (i, sl, e)


def test_training_reduces_loss(crt_ctx):
    """A denoising task the network can learn: targets are a smooth field,
    inputs that field times per-pixel noise; 150 Adam steps on the GPU."""
    import torch

    from cudaraytracer_b200.kpcn import Kpcn

    rng = np.random.default_rng(4)
    n, h, w = 4, 32, 32
    yy, xx = np.meshgrid(np.linspace(0, 1, h), np.linspace(0, 1, w), indexing="ij")
    base = np.stack([0.5 + 0.4 * np.sin(6 * xx + k) * np.cos(4 * yy - k) for k in range(3)], -1)
    ref = np.zeros((n, h, w, 4), np.float32)
    ref[..., :3] = base
    noisy = ref * rng.exponential(size=(n, h, w, 1)).astype(np.float32)
    feat = np.zeros((n, h, w, 16), np.float32)
    feat[..., :3] = np.log1p(noisy[..., :3])
    feat[..., 3:6] = base
    dfeat, dnoisy, dref = bf16_dev(feat), f32_dev(noisy), f32_dev(ref)
    net = Kpcn(crt_ctx, seed=1)
    first = net.train_step(dfeat, dnoisy, dref, lr=0.0)
    for _ in range(150):
        last = net.train_step(dfeat, dnoisy, dref, lr=2e-3)
    out = net.forward(dfeat, dnoisy)
    torch.cuda.synchronize()
    net.close()
    assert last < 0.5 * first
    assert K.relmse(out.cpu().numpy(), ref) < 0.6 * K.relmse(noisy, ref)


def test_features_from_a_render(tmp_path, crt_ctx):
    import torch

    from cudaraytracer_b200 import Scene, scenes
    from cudaraytracer_b200.kpcn import make_features

    sc = Scene.load(crt_ctx, scenes.cornell_box(width=32, height=24).write(str(tmp_path), "cb"))
    d = torch.zeros((24, 32, 4), device="cuda")
    i = torch.zeros_like(d)
    sc.render_device(d, i, 2)
    g = sc.gbuffer()
    feat, noisy = make_features(sc, g, d, i, 2, depth_scale=5.0)
    torch.cuda.synchronize()
    f = bf16_host(feat.view(torch.int16).cpu().numpy())
    nz = noisy.cpu().numpy()
    np.testing.assert_allclose(nz[..., :3], ((d + i) / 2).cpu().numpy()[..., :3], rtol=1e-6)
    np.testing.assert_allclose(f[..., :3], K.bf16_round(np.log1p(nz[..., :3])), rtol=1e-2, atol=1e-3)
    hit = g["bary_mesh"].cpu().numpy()[..., 3] != 0
    assert hit.all()  # the closed box fills the view
    nrm = np.linalg.norm(f[..., 6:9], axis=-1)
    assert np.all(np.abs(nrm - 1) < 0.02)
    assert np.all((f[..., 3:6] >= 0) & (f[..., 3:6] <= 1))
    assert np.all(f[..., 9] > 0) and not f[..., 13:].any()
    assert np.all(f[..., 12] == K.bf16_round(np.array([2 ** -0.5], np.float32))[0])
    sc.close()
