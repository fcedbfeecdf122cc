"""GPU render path (raygen, extend, shade with NEE/MIS, shadow, queue
compaction, accumulation) against the oracle renderer, called through the C
ABI. Both use the same per-path PCG32 streams, so images agree pixel by
pixel except where a float rounding flips a random branch; the bound is
written in each test."""
import numpy as np
import pytest

import oracle
from oracle import scene as osc
from cudaraytracer_b200 import Scene, scenes

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cornell_json(tmp_path_factory):
    d = tmp_path_factory.mktemp("cornell")
    return scenes.cornell_box(width=64, height=64, spp=4, max_bounces=8).write(str(d), "cb")


@pytest.fixture(scope="module")
def ico_json(tmp_path_factory):
    d = tmp_path_factory.mktemp("ico")
    spec = scenes.icosphere_field(n_spheres=8, level=2, width=48, height=48, env_size=(256, 128), spp=4,
                                  max_bounces=6)
    return spec.write(str(d), "ico")


def cam_vectors(sc):
    c = sc.camera()
    return {"position": c["position"], "left_down": c["left_down"], "du": c["du"], "dv": c["dv"]}


def compare(gpu, ora, rel_tol, max_bad_frac):
    g = gpu[..., :3].astype(np.float64)
    o = ora[..., :3].astype(np.float64)
    err = np.abs(g - o) / np.maximum(np.abs(o), 1e-3)
    bad = (err > rel_tol).any(-1)
    assert bad.mean() <= max_bad_frac, f"{bad.mean():.4f} of pixels differ by more than {rel_tol}"
    return bad.mean()


def test_loader_matches_oracle_loader(crt_ctx, cornell_json, ico_json):
    for path in (cornell_json, ico_json):
        sc = Scene.load(crt_ctx, path)
        ref = osc.load_scene(path)
        v, n, uv, pm = sc.export_geometry()
        np.testing.assert_array_equal(v, ref.verts)
        np.testing.assert_array_equal(n, ref.normals)
        np.testing.assert_array_equal(uv, ref.uvs)
        np.testing.assert_array_equal(pm, ref.prim_mesh)
        m, me, li = sc.export_tables()
        np.testing.assert_array_equal(m, ref.materials)
        np.testing.assert_array_equal(me, ref.meshes)
        np.testing.assert_array_equal(li, ref.lights)
        info = sc.info()
        assert (info["width"], info["height"], info["spp"], info["max_bounces"]) == (ref.width, ref.height, ref.spp,
                                                                                      ref.max_bounces)
        assert info["has_env"] == (ref.env_light >= 0)


def test_orbit_camera_matches_formula(crt_ctx, cornell_json, ico_json):
    for path in (cornell_json, ico_json):
        sc = Scene.load(crt_ctx, path)
        c = sc.camera()
        ref = osc.orbit_camera(osc.load_scene(path))
        for k in ("position", "u", "v", "w", "du", "dv", "left_down"):
            np.testing.assert_allclose(c[k], ref[k], rtol=1e-5, atol=1e-5)


def test_cornell_render_matches_oracle(crt_ctx, cornell_json):
    sc = Scene.load(crt_ctx, cornell_json)
    sc.set_render_params(seed=7)
    d, i, q = sc.render(4, with_sumsq=True)
    ref = osc.load_scene(cornell_json)
    od, oi, oq = oracle.render(ref, cam_vectors(sc), spp=4, seed=7)
    assert np.isfinite(d).all() and np.isfinite(i).all()
    compare(d, od, 1e-3, 0.02)
    compare(i, oi, 1e-3, 0.02)
    # q[..., 3] counts the sample values added into each pixel; it differs
    # only where a rounding flip changed a path's random branch, the same
    # 2% of pixels that the radiance bound above allows
    cnt_bad = q[..., 3] != oq[..., 3]
    assert cnt_bad.mean() <= 0.02, f"{cnt_bad.mean():.4f} of pixels differ in sample count"
    assert abs(q[..., 3].mean() - oq[..., 3].mean()) < 0.05


def test_icospheres_render_matches_oracle(crt_ctx, ico_json):
    """All four materials (diffuse, GGX, dielectric, subsurface with probe
    rays) under an importance-sampled environment map; the environment is
    fetched by the texture unit on the GPU and by an emulation of its 8-bit
    filter weights in the oracle, hence the looser bound."""
    sc = Scene.load(crt_ctx, ico_json)
    sc.set_render_params(seed=3)
    d, i = sc.render(4)
    ref = osc.load_scene(ico_json)
    od, oi, _ = oracle.render(ref, cam_vectors(sc), spp=4, seed=3)
    assert np.isfinite(d).all() and np.isfinite(i).all()
    compare(d, od, 2e-2, 0.03)
    compare(i, oi, 2e-2, 0.05)
    assert np.abs(d + i - od - oi)[..., :3].mean() < 2e-2 * max(1e-3, (od + oi)[..., :3].mean())


def test_device_render_accumulates_in_chunks(crt_ctx, cornell_json):
    import torch

    sc = Scene.load(crt_ctx, cornell_json)
    sc.set_render_params(seed=11)
    d8, i8 = sc.render(8)
    rp = sc.render_params()
    shape = (rp["height"], rp["width"], 4)
    dd = torch.zeros(shape, device="cuda")
    di = torch.zeros(shape, device="cuda")
    sc.render_device(dd, di, 4, first_sample=0)
    sc.render_device(dd, di, 4, first_sample=4)
    torch.cuda.synchronize()
    np.testing.assert_allclose(dd.cpu().numpy(), d8, rtol=1e-5, atol=1e-5)
    np.testing.assert_allclose(di.cpu().numpy(), i8, rtol=1e-5, atol=1e-5)


def test_max_bounces_and_survivor_drop(crt_ctx, cornell_json):
    """Paths alive after max_bounces are dropped (not accumulated), as the
    reference's bounce loop does: with rr = 1 every path that hits a wall
    survives its shading step, so one bounce leaves only the pixels that
    see the light directly or miss the box."""
    sc = Scene.load(crt_ctx, cornell_json)
    sc.set_render_params(max_bounces=1, rr=1.0, seed=5)
    d, i, q = sc.render(4, with_sumsq=True)
    ref = osc.load_scene(cornell_json)
    od, oi, oq = oracle.render(ref, cam_vectors(sc), spp=4, seed=5, max_bounces=1, rr=1.0)
    np.testing.assert_array_equal(q[..., 3], oq[..., 3])
    assert np.abs(i).max() == 0.0
    compare(d, od, 1e-5, 0.001)


@pytest.fixture(scope="module")
def textured_json(tmp_path_factory):
    d = tmp_path_factory.mktemp("tex")
    return scenes.cornell_box(width=48, height=48, spp=4, max_bounces=6, textured=True, lights=2).write(str(d), "ct")


def test_textured_two_light_render_matches_oracle(crt_ctx, textured_json):
    """Diffuse textures (PNG decoded by the library; by a separate Python
    decoder for the oracle) on a diffuse and a PBR material, two area lights
    (uniform light selection). Texels are filtered by the texture unit on the
    GPU and by an emulation of its 8-bit weights in the oracle."""
    sc = Scene.load(crt_ctx, textured_json)
    ref = osc.load_scene(textured_json)
    assert len(ref.textures) == 2 and sc.info()["num_lights"] == 2
    m, _, _ = sc.export_tables()
    np.testing.assert_array_equal(m, ref.materials)
    assert sorted(m[:, 14].tolist()) == [-1, -1, -1, -1, 0, 1]
    sc.set_render_params(seed=11)
    d, i = sc.render(4)
    od, oi, _ = oracle.render(ref, cam_vectors(sc), spp=4, seed=11)
    assert np.isfinite(d).all() and np.isfinite(i).all()
    compare(d, od, 2e-2, 0.03)
    compare(i, oi, 2e-2, 0.05)
    # the textures show: the back wall is not uniform
    back = (d + i)[..., :3][24:40, 16:32].reshape(-1, 3)
    assert back.std(0).max() > 0.02


@pytest.mark.parametrize("mode", ["local", "local-quant", "shared-quant", "warp", "refill"])  # against "shared"
def test_stage_traversal_modes_agree(crt_ctx, ico_json, monkeypatch, mode):
    """The extend and shadow stages give the same frame in every traversal
    mode (the whole stack in local memory, the default, or its top in
    shared memory; float nodes or their 16-bit quantised copy; primary rays
    as warp-coherent packets; later rays with per-lane refill), up to the
    order of the float atomics that add paths into pixels and the rare tie between equal-t triangles, and no traversal records an
    out-of-range index."""
    sc = Scene.load(crt_ctx, ico_json)
    sc.set_render_params(seed=4)
    monkeypatch.setenv("CRT_STAGE_TRAVERSAL", "shared")
    d0, i0 = sc.render(4)
    monkeypatch.setenv("CRT_STAGE_TRAVERSAL", mode)
    d1, i1 = sc.render(4)
    crt_ctx.check_device_errors()
    compare(d1, d0, 1e-4, 0.002)
    compare(i1, i0, 1e-4, 0.002)


@pytest.mark.parametrize("min_blocks", ["4", "6", "10"])
def test_shade_register_caps_agree(crt_ctx, ico_json, monkeypatch, min_blocks):
    """The shade stage compiled for 4 (no cap), 6 or 10 resident blocks per
    SM gives the frame of the default build (8 blocks, 64 registers), up to
    the order of the float atomics that add paths into pixels."""
    sc = Scene.load(crt_ctx, ico_json)
    sc.set_render_params(seed=9)
    monkeypatch.delenv("CRT_SHADE_MIN_BLOCKS", raising=False)
    d0, i0 = sc.render(4)
    monkeypatch.setenv("CRT_SHADE_MIN_BLOCKS", min_blocks)
    d1, i1 = sc.render(4)
    crt_ctx.check_device_errors()
    compare(d1, d0, 1e-4, 0.002)
    compare(i1, i0, 1e-4, 0.002)
