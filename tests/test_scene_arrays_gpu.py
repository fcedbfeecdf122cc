"""crt_scene_from_arrays (Scene.from_spec) builds the scene crt_scene_load_json
builds from the same generator written as JSON/OBJ/HDR files."""
import numpy as np
import pytest

from cudaraytracer_b200 import CrtError, Scene, scenes

pytestmark = pytest.mark.gpu

SPECS = {
    "cornell": lambda: scenes.cornell_box(width=40, height=40, max_bounces=5),
    "icospheres": lambda: scenes.icosphere_field(n_spheres=10, level=2, width=36, height=28, max_bounces=8,
                                                 env_size=(96, 48), sun_peak=40.0, sun_sigma=0.1),
    "cornell_tex2": lambda: scenes.cornell_box(width=32, height=32, max_bounces=5, textured=True, lights=2),
}


@pytest.mark.parametrize("name", sorted(SPECS))
def test_from_spec_matches_json_load(tmp_path, crt_ctx, name):
    import torch

    spec = SPECS[name]()
    a = Scene.load(crt_ctx, spec.write(str(tmp_path), name))
    b = Scene.from_spec(crt_ctx, spec)
    ia, ib = a.info(), b.info()
    for k in ("num_triangles", "num_meshes", "num_materials", "num_lights", "width", "height", "spp", "max_bounces",
              "has_env", "num_bvh_nodes", "bvh_depth"):
        assert ia[k] == ib[k], k
    assert a.render_params() == b.render_params()
    assert a.camera() == b.camera()
    ga, gb = a.export_geometry(), b.export_geometry()
    for x, y in zip(ga, gb):
        np.testing.assert_array_equal(x, y)
    ta, tb = a.export_tables(), b.export_tables()
    for x, y in zip(ta, tb):
        np.testing.assert_array_equal(x, y)
    shape = (ia["height"], ia["width"], 4)
    out = []
    for sc in (a, b):
        sc.set_render_params(seed=4)
        d = torch.zeros(shape, device="cuda")
        i = torch.zeros(shape, device="cuda")
        sc.render_device(d, i, 4)
        torch.cuda.synchronize()
        out.append((d.cpu().numpy(), i.cpu().numpy()))
    np.testing.assert_allclose(out[0][0], out[1][0], rtol=2e-5, atol=2e-6)
    np.testing.assert_allclose(out[0][1], out[1][1], rtol=2e-5, atol=2e-6)
    a.close()
    b.close()


def test_from_spec_rejects_bad_tables(crt_ctx):
    spec = scenes.cornell_box(width=8, height=8)
    spec.meshes[0].material = "no-such-material"
    with pytest.raises(KeyError):
        Scene.from_spec(crt_ctx, spec)
    spec = scenes.cornell_box(width=8, height=8)
    spec.camera["resolution"] = [0, 8]
    with pytest.raises(CrtError, match="INVALID"):
        Scene.from_spec(crt_ctx, spec)
