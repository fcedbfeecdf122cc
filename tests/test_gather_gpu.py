"""Display resolve and debug views (crt_gather) against the CPU restatement
of the reference's GatherKernel on the same accumulators and G-buffer."""
import numpy as np
import pytest

from oracle import display

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("mode", [0, 1, 2, 3, 4])
def test_gather_modes(tmp_path, crt_ctx, mode):
    import torch

    from cudaraytracer_b200 import Scene, scenes

    sc = Scene.load(crt_ctx, scenes.cornell_box(width=40, height=30).write(str(tmp_path), "cb"))
    d = torch.zeros((30, 40, 4), device="cuda")
    i = torch.zeros_like(d)
    sc.render_device(d, i, 8)
    g = sc.gbuffer()
    out = sc.gather(mode, 8, d, i, g).cpu().numpy()
    info, cam = sc.info(), sc.camera()
    gh = {k: (v.view(torch.uint16) if v.dtype == torch.int16 else v).cpu().numpy() for k, v in g.items()}
    ref = display.gather(mode, 8, d.cpu().numpy(), i.cpu().numpy(), gh, info["bounds_min"], info["bounds_max"],
                         cam["position"])
    diff = np.abs(out.astype(int) - ref.astype(int))
    assert diff.max() <= 1  # float rounding at byte boundaries (powf, divisions)
    assert np.mean(diff > 0) < 0.02
    if mode == 3:
        assert len(np.unique(out[..., 0])) >= 3  # several meshes visible
    sc.close()
