"""Batched multi-view rendering (shared wavefronts, CUDA graph per pass) and
its autotuner, through the C ABI."""
import numpy as np
import pytest

from cudaraytracer_b200 import Scene, scenes
from cudaraytracer_b200.autotune import autotune_paths_per_pass, orbit_views

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cornell(tmp_path_factory, crt_ctx):
    d = tmp_path_factory.mktemp("batch")
    return Scene.load(crt_ctx, scenes.cornell_box(width=64, height=64, max_bounces=6).write(str(d), "cb"))


def test_single_view_batch_equals_render_device(cornell):
    import torch

    cornell.set_render_params(seed=21, paths_per_pass=1 << 14)
    rp = cornell.render_params()
    shape = (rp["height"], rp["width"], 4)
    d = torch.zeros(shape, device="cuda")
    i = torch.zeros(shape, device="cuda")
    cornell.render_device(d, i, 8)
    bd = torch.zeros((1,) + shape, device="cuda")
    bi = torch.zeros((1,) + shape, device="cuda")
    cornell.render_views([cornell.camera()], bd, bi, 8)
    torch.cuda.synchronize()
    np.testing.assert_allclose(bd[0].cpu().numpy(), d.cpu().numpy(), rtol=1e-5, atol=1e-5)
    np.testing.assert_allclose(bi[0].cpu().numpy(), i.cpu().numpy(), rtol=1e-5, atol=1e-5)


def test_graph_and_direct_launch_agree(cornell):
    import torch

    cornell.set_render_params(seed=5, paths_per_pass=20000)  # several passes, a partial last one
    views = orbit_views(cornell, 5, radius=2.5)
    rp = cornell.render_params()
    shape = (len(views), rp["height"], rp["width"], 4)
    out = []
    for g in (True, False):
        d = torch.zeros(shape, device="cuda")
        i = torch.zeros(shape, device="cuda")
        cornell.render_views(views, d, i, 4, use_graph=g)
        torch.cuda.synchronize()
        out.append((d.cpu().numpy(), i.cpu().numpy()))
    np.testing.assert_allclose(out[0][0], out[1][0], rtol=1e-5, atol=1e-5)
    np.testing.assert_allclose(out[0][1], out[1][1], rtol=1e-5, atol=1e-5)
    # every view was rendered (non-empty), and views differ
    s = out[0][0].sum(axis=(1, 2, 3)) + out[0][1].sum(axis=(1, 2, 3))
    assert (s > 0).all() and len(set(np.round(s, 3))) == len(views)


def test_batched_view_statistics_match_single_view(cornell):
    """A view rendered inside a batch converges to the same image as the
    same camera rendered alone (different PCG32 streams)."""
    import torch

    cornell.set_render_params(seed=9, paths_per_pass=0)
    cam = cornell.camera()
    views = orbit_views(cornell, 3, radius=2.5)
    views[1] = cam
    rp = cornell.render_params()
    shape = (3, rp["height"], rp["width"], 4)
    d = torch.zeros(shape, device="cuda")
    i = torch.zeros(shape, device="cuda")
    cornell.render_views(views, d, i, 256)
    sd, si = cornell.render(256)
    torch.cuda.synchronize()
    a = (d[1] + i[1])[..., :3].cpu().numpy() / 256
    b = (sd + si)[..., :3] / 256
    assert abs(a.mean() - b.mean()) < 0.01 * b.mean()
    assert np.mean((a - b) ** 2 / (b ** 2 + 1e-2)) < 5e-3


def test_autotuner_picks_and_caches(cornell, tmp_path):
    views = orbit_views(cornell, 4, radius=2.5)
    cache = str(tmp_path / "tune.json")
    r = autotune_paths_per_pass(cornell, views, candidates=(1 << 14, 1 << 16), cache_path=cache)
    assert not r["cached"] and r["paths_per_pass"] in (1 << 14, 1 << 16)
    assert cornell.render_params()["paths_per_pass"] == r["paths_per_pass"]
    assert r["stage_block"] in (64, 128, 256) and cornell.render_params()["stage_block"] == r["stage_block"]
    assert r["stage_traversal"] in (1, 2, 3, 4, 5, 6) and len(r["traversal_timings_ms"]) == 6
    assert cornell.render_params()["stage_traversal"] == r["stage_traversal"]
    cornell.set_render_params(stage_traversal=0)
    r2 = autotune_paths_per_pass(cornell, views, candidates=(1 << 14, 1 << 16), cache_path=cache)
    assert r2["cached"] and r2["paths_per_pass"] == r["paths_per_pass"]
    assert r2["stage_block"] == r["stage_block"]
    assert cornell.render_params()["stage_traversal"] == r["stage_traversal"]
    cornell.set_render_params(stage_traversal=0, stage_block=0, paths_per_pass=0)


def test_stage_block_size_does_not_change_the_image(cornell):
    """The stage kernels' block size only changes scheduling: per-path work
    is keyed by (seed, pixel, sample), so the frame is the same up to the
    order of the accumulators' float additions."""
    import pytest

    from cudaraytracer_b200 import CrtError

    frames = []
    for b in (64, 256):
        cornell.set_render_params(stage_block=b, seed=23)
        d, i = cornell.render(4)
        frames.append((d, i))
    cornell.set_render_params(stage_block=0)
    for a, b in zip(frames[0], frames[1]):
        np.testing.assert_allclose(a, b, rtol=1e-5, atol=1e-6)
    with pytest.raises(CrtError):
        cornell.set_render_params(stage_block=96)


def test_stage_traversal_param_does_not_change_the_image(cornell):
    """Each stage traversal (stack in local or shared memory, float or
    quantised nodes) set through the render parameters gives the frame of
    the default, up to the order of float additions and ties between
    equal-t triangles; out-of-range values are refused."""
    import pytest

    from cudaraytracer_b200 import CrtError

    cornell.set_render_params(stage_traversal=0, seed=29)
    d0, i0 = cornell.render(4)
    for t in (1, 2, 3, 4, 5, 6):
        cornell.set_render_params(stage_traversal=t)
        d1, i1 = cornell.render(4)
        for a, b in ((d1, d0), (i1, i0)):
            err = np.abs(a - b)[..., :3] / np.maximum(np.abs(b[..., :3]), 1e-3)
            assert (err > 1e-4).any(-1).mean() <= 0.002, t
    cornell.set_render_params(stage_traversal=0)
    for bad in (-1, 7):
        with pytest.raises(CrtError):
            cornell.set_render_params(stage_traversal=bad)
