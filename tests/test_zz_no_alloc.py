"""crt_render_device_noalloc: the render pass for hosts that cannot let the
tracer allocate device memory during a frame (engines and plugins that own
the GPU memory pool). Its path queues live in a fixed scratch area of the
library's device image. Checked through the C ABI against the allocating
entry point crt_render_device on the same samples, on two calls in a row
(the scratch keeps the previous call's contents, so the second call shows
the per-call reset works)."""
import numpy as np
import pytest

from cudaraytracer_b200 import Context, CrtError, Scene, scenes

pytestmark = pytest.mark.gpu


def test_noalloc_render_matches_allocating_entry_point(tmp_path):
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    ctx = Context(0)
    sc = Scene.load(ctx, scenes.cornell_box(width=64, height=64, max_bounces=8).write(str(tmp_path), "cb"))
    sc.set_render_params(seed=13)
    rp = sc.render_params()
    shape = (rp["height"], rp["width"], 4)
    for first in (0, 4):  # two calls in a row, different sample ranges
        ref_d = torch.zeros(shape, device="cuda")
        ref_i = torch.zeros(shape, device="cuda")
        sc.render_device(ref_d, ref_i, 4, first_sample=first)
        d = torch.zeros(shape, device="cuda")
        i = torch.zeros(shape, device="cuda")
        sc.render_device_noalloc(d, i, 4, first_sample=first)
        torch.cuda.synchronize()
        assert float(ref_d.sum()) > 0.0
        np.testing.assert_allclose(d.cpu().numpy(), ref_d.cpu().numpy(), rtol=1e-5, atol=1e-5)
        np.testing.assert_allclose(i.cpu().numpy(), ref_i.cpu().numpy(), rtol=1e-5, atol=1e-5)
    # images beyond the fixed scratch are rejected with a clear error
    sc.set_render_params(width=512, height=512)
    big = torch.zeros((512, 512, 4), device="cuda")
    with pytest.raises(CrtError, match="CRT_ERR_CAPACITY"):
        sc.render_device_noalloc(big, big.clone(), 1)
    sc.close()
    ctx.close()
