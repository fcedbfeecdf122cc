"""Statistical parity of converged renders with the reference's own
renderer. tests/golden/render_ref_*.npz hold images rendered by the
reference's code (headless CUDA build of its scene loader and RenderLoop,
tests/golden/make_render_golden.py) with per-pixel sums of squares. The
samplers differ (curand per compacted slot vs PCG32 per path), so images
agree in distribution: relMSE against the reference must sit at the noise
floor measured between two independent renders of ours, and per-pixel
z-scores must stay within what sampling noise allows."""
import os

import numpy as np
import pytest

from cudaraytracer_b200 import Scene, scenes
from conftest import GOLDEN

pytestmark = pytest.mark.gpu

import sys

sys.path.insert(0, GOLDEN)
import make_render_golden as mg  # noqa: E402


# relMSE bound per fixture. The Cornell-box renders (4096 spp) are held to
# the converged-image bar of 1e-3. The icosphere fixture (64x64 at 16384 spp,
# glass and subsurface spheres lit by a sun lobe) keeps heavier-tailed noise
# from caustic paths; its bound sits above its measured noise floor.
ABS_RELMSE = {"cornell": 1e-3, "cornell_256": 1e-3, "cornell_tex2": 1e-3, "cornell_jpg": 1e-3, "icospheres": 1e-3}


def stats(sum_a, sq_a, na, sum_b, sq_b, nb):
    ma, mb = sum_a / na, sum_b / nb
    va = np.maximum(sq_a / na - ma * ma, 0)
    vb = np.maximum(sq_b / nb - mb * mb, 0)
    relmse = float(np.mean((ma - mb) ** 2 / (mb * mb + 1e-2)))
    z = (ma - mb) / np.sqrt(va / na + vb / nb + 1e-12)
    return relmse, z


@pytest.mark.parametrize("name", sorted(mg.SCENES))
def test_converged_render_matches_reference(crt_ctx, tmp_path, name):
    gpath = os.path.join(GOLDEN, f"render_ref_{name}.npz")
    if not os.path.exists(gpath):
        pytest.skip("reference render fixture missing")
    g = np.load(gpath)
    fn, kw, spp, wkw = mg.scene_entry(name)
    sc = Scene.load(crt_ctx, getattr(scenes, fn)(**kw).write(str(tmp_path), name, **wkw))
    c = sc.camera()
    np.testing.assert_allclose(np.array(c["position"] + c["left_down"] + c["du"] + c["dv"]), g["camera"], atol=1e-6)
    ref_sum = (g["direct"] + g["indirect"])[..., :3].astype(np.float64)
    ref_sq = g["sumsq"][..., :3].astype(np.float64)
    runs = []
    for seed in (1, 2):
        sc.set_render_params(seed=seed)
        d, i, q = sc.render(spp, with_sumsq=True)
        runs.append(((d + i)[..., :3].astype(np.float64), q[..., :3].astype(np.float64)))
    rel_ref, z = stats(runs[0][0], runs[0][1], spp, ref_sum, ref_sq, spp)
    rel_self, _ = stats(runs[0][0], runs[0][1], spp, runs[1][0], runs[1][1], spp)
    # no bias beyond sampling noise: relMSE vs the reference is at the floor
    # set by two independent renders of ours (same spp)
    print(f"{name}: relMSE vs reference {rel_ref:.3e}, between our two renders {rel_self:.3e}, "
          f"mean z^2 {np.mean(z * z):.3f}, |z|>4 {np.mean(np.abs(z) > 4):.4f}")
    assert rel_ref <= 1.5 * rel_self + 1e-5, (rel_ref, rel_self)
    # absolute bound on the converged images' relMSE against the reference
    assert rel_ref <= ABS_RELMSE[name], (rel_ref, ABS_RELMSE[name])
    assert np.mean(np.abs(z) > 4) <= 0.005
    assert np.mean(z * z) <= 1.5
