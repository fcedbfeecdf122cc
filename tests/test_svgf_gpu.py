"""SVGF and the primary-hit G-buffer on the GPU, through the C ABI.

* The G-buffer has the reference raster pass's encodings and agrees with the
  closest-hit query of the same pixel-centre rays.
* SVGF on identical inputs (noisy 1-spp frames and G-buffers of an orbiting
  camera) agrees with the reference's own SVGF kernels (headless CUDA build
  of TemporalDenoiseKernel, ComputeVarianceKernel and AtrousKernel) within
  1e-3 absolute, frame after frame."""
import numpy as np
import pytest

import oracle
from cudaraytracer_b200 import Scene, Svgf, scenes, hit_prims

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cornell(tmp_path_factory, crt_ctx):
    d = tmp_path_factory.mktemp("svgf")
    return Scene.load(crt_ctx, scenes.cornell_box(width=64, height=48, max_bounces=4).write(str(d), "cb"))


def frames_of(sc, n, dphi=1.5):
    """n frames of an orbiting camera: noisy 1-spp direct/indirect and
    G-buffers (numpy), G-buffer motion against the previous frame."""
    import torch

    rp = sc.render_params()
    shape = (rp["height"], rp["width"], 4)
    cam0 = sc.camera()
    out = {k: [] for k in ("nd", "ni", "pos_tri", "normal_mat", "bary_mesh", "motion_depth")}
    prev = None
    for f in range(n):
        sc.set_camera_orbit(cam0["target"], cam0["distance"], cam0["theta_deg"], cam0["phi_deg"] + dphi * f,
                            cam0["fovy_deg"])
        d = torch.zeros(shape, device="cuda")
        i = torch.zeros(shape, device="cuda")
        sc.render_device(d, i, 1, first_sample=f)
        g = sc.gbuffer(prev_camera=prev)
        torch.cuda.synchronize()
        prev = sc.camera()
        out["nd"].append(d.cpu().numpy())
        out["ni"].append(i.cpu().numpy())
        for k in ("pos_tri", "motion_depth"):
            out[k].append(g[k].cpu().numpy())
        for k in ("normal_mat", "bary_mesh"):
            out[k].append(g[k].cpu().numpy().view(np.uint16))
    sc.set_camera_orbit(cam0["target"], cam0["distance"], cam0["theta_deg"], cam0["phi_deg"], cam0["fovy_deg"])
    return {k: np.stack(v) for k, v in out.items()}


def test_gbuffer_encodings_and_hits(cornell):
    import torch

    g = cornell.gbuffer()
    torch.cuda.synchronize()
    pt = g["pos_tri"].cpu().numpy()
    nm = g["normal_mat"].cpu().numpy().view(np.uint16)
    bm = g["bary_mesh"].cpu().numpy().view(np.uint16)
    md = g["motion_depth"].cpu().numpy()
    hit = bm[..., 3] > 0
    assert hit.mean() > 0.5
    # background is all zeros, as the raster pass clears it
    assert np.all(pt[~hit] == 0) and np.all(md[~hit] == 0) and np.all(nm[~hit] == 0)
    # static camera: no motion; depth positive on hits
    assert np.all(md[hit, :2] == 0) and np.all(md[hit, 2] > 0)
    # decoded normals are unit vectors; barycentrics sum to ~65535
    n = nm[hit, :3] / 65535.0 * 2 - 1
    assert np.allclose(np.linalg.norm(n, axis=1), 1.0, atol=1e-3)
    assert np.all(np.abs(bm[hit, :3].astype(np.int64).sum(1) - 65535) <= 3)
    # positions equal the closest hits of pixel-centre rays (front faces here)
    c = cornell.camera()
    rp = cornell.render_params()
    H, W = rp["height"], rp["width"]
    jj, ii = np.mgrid[0:H, 0:W]
    ld, du, dv, pos = (np.array(c[k], np.float32) for k in ("left_down", "du", "dv", "position"))
    pp = ld + (ii[..., None] + 0.5) * du + (jj[..., None] + 0.5) * dv
    dirs = (pp - pos) / np.linalg.norm(pp - pos, axis=-1, keepdims=True)
    rays = np.zeros((H * W, 8), np.float32)
    rays[:, 0:3] = pos
    rays[:, 4:7] = dirs.reshape(-1, 3)
    rays[:, 7] = 1e8
    h = cornell.trace_closest(rays)
    th = hit_prims(h) >= 0
    agree = th.reshape(H, W) == hit
    assert agree.mean() > 0.99
    both = (th.reshape(H, W) & hit).reshape(-1)
    pts = rays[both, 0:3] + h[both, 0:1] * rays[both, 4:7]
    assert np.abs(pts - pt.reshape(-1, 4)[both, :3]).max() < 1e-4


def test_svgf_matches_reference_kernels(crt_ctx, cornell):
    import torch

    if not oracle.ref_render_available():
        pytest.skip("reference build absent")
    F = 5
    fr = frames_of(cornell, F)
    rp = cornell.render_params()
    sv = Svgf(crt_ctx, rp["width"], rp["height"])
    dev = torch.device("cuda")
    mine_d, mine_i = [], []
    to = lambda a, dt=torch.float32: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    gbs = []
    for f in range(F):
        gbs.append({"pos_tri": to(fr["pos_tri"][f]), "motion_depth": to(fr["motion_depth"][f]),
                    "normal_mat": to(fr["normal_mat"][f].view(np.int16)), "bary_mesh": to(fr["bary_mesh"][f].view(np.int16))})
    zero = {k: torch.zeros_like(v) for k, v in gbs[0].items()}
    for f in range(F):
        od = torch.empty_like(to(fr["nd"][f]))
        oi = torch.empty_like(od)
        sv.frame(gbs[f], gbs[f - 1] if f else zero, to(fr["nd"][f]), to(fr["ni"][f]), od, oi)
        torch.cuda.synchronize()
        mine_d.append(od.cpu().numpy())
        mine_i.append(oi.cpu().numpy())
    ref_d, ref_i = oracle.ref_svgf(fr["nd"], fr["ni"], fr["pos_tri"], fr["normal_mat"], fr["bary_mesh"],
                                   fr["motion_depth"])
    mine_d, mine_i = np.stack(mine_d), np.stack(mine_i)
    assert np.isfinite(mine_d).all() and np.isfinite(mine_i).all()
    for f in range(F):
        np.testing.assert_allclose(mine_d[f], ref_d[f], atol=1e-3, rtol=0, err_msg=f"direct, frame {f}")
        np.testing.assert_allclose(mine_i[f], ref_i[f], atol=1e-3, rtol=0, err_msg=f"indirect, frame {f}")
    sv.close()


def test_render_svgf_frame_pipeline(crt_ctx, cornell):
    """The denoised-frame entry point (1 spp + G-buffer + SVGF) runs frame
    after frame and lowers the error against a converged render."""
    import torch

    rp = cornell.render_params()
    shape = (rp["height"], rp["width"], 4)
    cornell.set_render_params(seed=3)
    ref_d, ref_i = cornell.render(1024)
    ref = (ref_d + ref_i)[..., :3] / 1024
    sv = Svgf(crt_ctx, rp["width"], rp["height"])
    od = torch.empty(shape, device="cuda")
    oi = torch.empty(shape, device="cuda")
    for f in range(8):
        cornell.render_svgf_frame(sv, f, od, oi)
    torch.cuda.synchronize()
    den = (od + oi)[..., :3].cpu().numpy()
    nd, ni = cornell.render(1)
    noisy = (nd + ni)[..., :3]
    rel = lambda x: float(np.mean((x - ref) ** 2 / (ref ** 2 + 1e-2)))
    assert np.isfinite(den).all()
    assert rel(den) < 0.5 * rel(noisy)
    sv.close()
