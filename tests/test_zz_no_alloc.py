"""crt_render_device_noalloc: the render pass for hosts that cannot let the
tracer allocate device memory during a frame (engines and plugins that own
the GPU memory pool). Its path queues live in a fixed scratch area of the
library's device image. Checked through the C ABI against the allocating
entry point crt_render_device on the same samples:

* two calls in a row on one wavefront (the scratch keeps the previous
  call's contents, and the second call must not read them);
* several wavefronts per call (128x128 at 10 spp runs passes of 4, 4 and 2
  samples; 256x256, exactly the 65,536-pixel limit, runs one sample per
  pass), which exercises the pass loop, its short last pass and the reuse of
  the scratch queues across passes;
* an explicit spp_per_pass below the scratch limit and a 64-thread stage
  block, which the entry point honours as crt_render_device does;
* 65,537 pixels, one beyond the limit, rejected with CRT_ERR_CAPACITY;
* a scene with all four materials and an environment light, whose shade
  order has all three regions (hits, subsurface hits, misses)."""
import numpy as np
import pytest

from cudaraytracer_b200 import Context, CrtError, Scene, scenes

pytestmark = pytest.mark.gpu


def _pair(sc, spp, first):
    import torch

    rp = sc.render_params()
    shape = (rp["height"], rp["width"], 4)
    ref_d = torch.zeros(shape, device="cuda")
    ref_i = torch.zeros(shape, device="cuda")
    sc.render_device(ref_d, ref_i, spp, first_sample=first)
    d = torch.zeros(shape, device="cuda")
    i = torch.zeros(shape, device="cuda")
    sc.render_device_noalloc(d, i, spp, first_sample=first)
    torch.cuda.synchronize()
    assert float(ref_d.sum()) > 0.0
    np.testing.assert_allclose(d.cpu().numpy(), ref_d.cpu().numpy(), rtol=1e-5, atol=1e-5)
    np.testing.assert_allclose(i.cpu().numpy(), ref_i.cpu().numpy(), rtol=1e-5, atol=1e-5)


@pytest.fixture()
def ctx():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    c = Context(0)
    yield c
    c.close()


def test_noalloc_render_matches_allocating_entry_point(ctx, tmp_path):
    sc = Scene.load(ctx, scenes.cornell_box(width=64, height=64, max_bounces=8).write(str(tmp_path), "cb"))
    sc.set_render_params(seed=13)
    for first in (0, 4):  # two calls in a row, different sample ranges
        _pair(sc, 4, first)
    sc.close()


def test_noalloc_render_all_materials(ctx, tmp_path):
    spec = scenes.icosphere_field(n_spheres=8, level=2, width=48, height=48, env_size=(256, 128), spp=4,
                                  max_bounces=6)
    sc = Scene.load(ctx, spec.write(str(tmp_path), "ico"))
    sc.set_render_params(seed=17)
    _pair(sc, 4, 0)
    sc.close()


def test_noalloc_several_wavefronts_per_call(ctx, tmp_path):
    sc = Scene.load(ctx, scenes.cornell_box(width=128, height=128, max_bounces=8).write(str(tmp_path), "cb"))
    sc.set_render_params(seed=21)
    _pair(sc, 10, 0)  # passes of 4, 4 and 2 samples
    _pair(sc, 10, 10)
    sc.set_render_params(spp_per_pass=3, stage_block=64)  # passes of 3, 3, 3, 1
    _pair(sc, 10, 20)
    sc.set_render_params(spp_per_pass=0, stage_block=0, width=256, height=256)  # exactly 65,536 pixels
    _pair(sc, 3, 0)  # three wavefronts of 65,536 paths
    sc.close()


def test_noalloc_rejects_images_beyond_the_scratch(ctx, tmp_path):
    import torch

    sc = Scene.load(ctx, scenes.cornell_box(width=64, height=64, max_bounces=8).write(str(tmp_path), "cb"))
    sc.set_render_params(width=65537, height=1)
    big = torch.zeros((1, 65537, 4), device="cuda")
    with pytest.raises(CrtError, match="CRT_ERR_CAPACITY"):
        sc.render_device_noalloc(big, big.clone(), 1)
    sc.set_render_params(width=512, height=512)
    big = torch.zeros((512, 512, 4), device="cuda")
    with pytest.raises(CrtError, match="CRT_ERR_CAPACITY"):
        sc.render_device_noalloc(big, big.clone(), 1)
    sc.close()
