"""Tensor-core 3x3 convolutions (forward, data gradient, weight gradient)
against the float64 CPU oracle on the same BF16 inputs. The GPU accumulates
in FP32, so the bound is the FP32 accumulation error of the sum of |terms|
(plus half a BF16 ulp for BF16 outputs)."""
import numpy as np
import pytest

from oracle import kpcn_oracle as K

pytestmark = pytest.mark.gpu

CASES = [  # n, h, w, cin, cout
    (2, 19, 23, 16, 32),
    (1, 33, 17, 32, 64),
    (1, 16, 24, 96, 96),
    (1, 12, 13, 160, 64),
    (1, 9, 11, 64, 16),
    (3, 7, 5, 32, 160),
    # wider than 256: 256-pixel tiles, the last x tile partial
    (1, 6, 300, 64, 64),    # row ring, one 128 B channel chunk
    (2, 5, 520, 32, 96),    # row ring, two images, three x tiles
    (1, 4, 280, 96, 64),    # three-row stages with resident weights
    # smallest images and the channel limits
    (1, 1, 1, 16, 16),
    (4, 2, 3, 16, 32),
    (1, 3, 20, 256, 256),   # weights streamed with the stages, two 128-row M blocks
]


def to_dev(a, dtype):
    import torch

    if dtype == "bf16":
        return torch.from_numpy(K.bf16_bits(a).view(np.int16)).view(torch.bfloat16).cuda()
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).cuda()


def from_dev(t):
    import torch

    if t.dtype == torch.bfloat16:
        return K.from_bf16_bits(t.view(torch.int16).cpu().numpy().view(np.uint16))
    return t.cpu().numpy()


@pytest.mark.parametrize("n,h,w,cin,cout", CASES)
def test_conv3x3_forward_and_gradients(crt_ctx, n, h, w, cin, cout):
    import torch

    from cudaraytracer_b200 import kpcn

    rng = np.random.default_rng(cin * 1000 + cout + h)
    x = K.bf16_round(rng.normal(size=(n, h, w, cin)).astype(np.float32))
    wt = K.bf16_round((rng.normal(size=(9, cout, cin)) / np.sqrt(9 * cin)).astype(np.float32))
    b = rng.normal(size=cout).astype(np.float32)
    g = K.bf16_round(rng.normal(size=(n, h, w, cout)).astype(np.float32))

    dx, dw, db, dg = to_dev(x, "bf16"), to_dev(wt, "bf16"), to_dev(b, "f32"), to_dev(g, "bf16")
    f32 = torch.zeros((n, h, w, cout), device="cuda")
    out = kpcn.conv3x3_forward(crt_ctx, dx, dw, db, relu=True, out_f32=f32,
                               out=torch.empty((n, h, w, cout), dtype=torch.bfloat16, device="cuda"))
    gin = kpcn.conv3x3_backward_data(crt_ctx, dg, to_dev(K.transpose_taps(wt), "bf16"), mask=dx)
    gw = kpcn.conv3x3_backward_weights(crt_ctx, dx, dg)
    torch.cuda.synchronize()
    kpcn.check_device_errors(crt_ctx)

    ref = K.conv3x3_forward(x, wt, b, relu=True)
    bound = K.conv3x3_forward(np.abs(x), np.abs(wt)) + np.abs(b)
    tol = 2e-5 * bound + 1e-6
    assert np.all(np.abs(from_dev(f32) - ref) <= tol)
    assert np.all(np.abs(from_dev(out) - ref) <= tol + np.abs(ref) * 2.0 ** -8)

    ref_gx = K.conv3x3_backward_data(g, wt, mask=x)
    bound_gx = K.conv3x3_backward_data(np.abs(g), np.abs(wt))
    assert np.all(np.abs(from_dev(gin) - ref_gx) <= 2e-5 * bound_gx + 1e-6 + np.abs(ref_gx) * 2.0 ** -8)

    ref_gw = K.conv3x3_backward_weights(x, g)
    bound_gw = K.conv3x3_backward_weights(np.abs(x), np.abs(g))
    assert np.all(np.abs(from_dev(gw) - ref_gw) <= 2e-5 * bound_gw + 1e-6)


def test_forward_512_input_channels(crt_ctx):
    """The widest input accepted (512 channels): streamed weights, two-stage pipeline."""
    from cudaraytracer_b200 import kpcn

    rng = np.random.default_rng(512)
    x = K.bf16_round(rng.normal(size=(1, 3, 20, 512)).astype(np.float32))
    wt = K.bf16_round((rng.normal(size=(9, 256, 512)) / np.sqrt(9 * 512)).astype(np.float32))
    out = kpcn.conv3x3_forward(crt_ctx, to_dev(x, "bf16"), to_dev(wt, "bf16"))
    ref = K.conv3x3_forward(x, wt)
    bound = K.conv3x3_forward(np.abs(x), np.abs(wt))
    assert np.all(np.abs(from_dev(out) - ref) <= 2e-5 * bound + 1e-6 + np.abs(ref) * 2.0 ** -8)


def test_weight_gradient_accumulates(crt_ctx):
    import torch

    from cudaraytracer_b200 import kpcn

    rng = np.random.default_rng(5)
    x = K.bf16_round(rng.normal(size=(1, 20, 30, 32)).astype(np.float32))
    g = K.bf16_round(rng.normal(size=(1, 20, 30, 16)).astype(np.float32))
    dw = torch.ones((9, 16, 32), device="cuda")
    kpcn.conv3x3_backward_weights(crt_ctx, to_dev(x, "bf16"), to_dev(g, "bf16"), dw=dw)
    torch.cuda.synchronize()
    ref = K.conv3x3_backward_weights(x, g) + 1.0
    bound = K.conv3x3_backward_weights(np.abs(x), np.abs(g)) + 1.0
    assert np.all(np.abs(dw.cpu().numpy() - ref) <= 2e-5 * bound)


def test_bad_channel_counts_are_refused(crt_ctx):
    import torch

    from cudaraytracer_b200 import CrtError, kpcn

    x = torch.zeros((1, 4, 4, 12), dtype=torch.bfloat16, device="cuda")
    w = torch.zeros((9, 16, 12), dtype=torch.bfloat16, device="cuda")
    with pytest.raises(CrtError, match="INVALID"):
        kpcn.conv3x3_forward(crt_ctx, x, w)
