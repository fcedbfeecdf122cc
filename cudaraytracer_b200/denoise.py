"""Training data, training and evaluation of the learned denoiser (kpcn.py)
against SVGF, on seeded Cornell-box variants rendered by the tracer itself.

* A training example is one rendered view: the network input (features of
  a k-spp render and its G-buffer) and the reference radiance of the same
  view from an independent sample range (samples from 2^20 on), many spp.
* Training draws random crops of random examples per step and runs the
  GPU's own forward, backward and Adam step (crt_kpcn_train_step).
* Evaluation measures relMSE = mean((x - ref)^2 / (ref^2 + 0.01)) against a
  4096-spp reference for: the raw k-spp image, the KPCN output at k spp, and
  SVGF (the reference's filter: TemporalDenoising, variance estimate and 5
  a-trous passes) applied to a k-spp image as a two-frame sequence of the
  same image, which runs the variance estimate and the a-trous passes that a
  first frame skips.
"""
from __future__ import annotations

import math
import time
from dataclasses import dataclass

import numpy as np

from .kpcn import Kpcn, make_features
from .tracer import Scene, Svgf

REF_FIRST_SAMPLE = 1 << 20
DEPTH_SCALE = 4.0


@dataclass
class Example:
    feat: object   # (h, w, 16) bfloat16 CUDA tensor
    noisy: object  # (h, w, 4) float32
    ref: object    # (h, w, 4) float32
    spp: int


def view_cameras(scene: Scene, n: int, seed: int):
    """n orbit poses looking into the open side of a Cornell box: elevation
    U[75, 105] deg, azimuth U[-20, 20] deg, distance x U[0.85, 1.1]."""
    rng = np.random.default_rng(seed)
    c = scene.camera()
    out = []
    for _ in range(n):
        out.append({"target": list(c["target"]), "distance": float(c["distance"]) * float(rng.uniform(0.85, 1.1)),
                    "theta_deg": float(rng.uniform(75, 105)), "phi_deg": float(rng.uniform(-20, 20)),
                    "fovy_deg": float(c["fovy_deg"])})
    return out


def render_view(scene: Scene, cam: dict, width: int, height: int, spp: int, seed: int, first_sample: int = 0):
    """(direct, indirect) float32 (h, w, 4) CUDA sums over spp samples."""
    import torch

    scene.set_render_params(width=width, height=height, seed=seed)
    scene.set_camera_orbit(cam["target"], cam["distance"], cam["theta_deg"], cam["phi_deg"], cam["fovy_deg"])
    d = torch.zeros((height, width, 4), device="cuda")
    i = torch.zeros_like(d)
    if spp:
        scene.render_device(d, i, spp, first_sample=first_sample)
    return d, i


def make_example(scene: Scene, cam: dict, width: int, height: int, spp: int, ref_spp: int, seed: int) -> Example:
    d, i = render_view(scene, cam, width, height, spp, seed)
    g = scene.gbuffer()
    feat, noisy = make_features(scene, g, d, i, spp, DEPTH_SCALE)
    rd, ri = render_view(scene, cam, width, height, ref_spp, seed, first_sample=REF_FIRST_SAMPLE)
    ref = (rd + ri) / ref_spp
    return Example(feat, noisy, ref, spp)


def build_dataset(ctx, scene_seeds, views_per_scene: int, width: int, height: int, spp_choices, ref_spp: int,
                  seed: int = 0):
    """Examples over seeded Cornell variants; each view's spp drawn from
    spp_choices."""
    from . import scenes

    rng = np.random.default_rng(seed)
    out = []
    for s in scene_seeds:
        sc = Scene.from_spec(ctx, scenes.cornell_box(width=width, height=height, seed=int(s)))
        for v, cam in enumerate(view_cameras(sc, views_per_scene, int(s) * 7 + 1)):
            spp = int(spp_choices[int(rng.integers(len(spp_choices)))])
            out.append(make_example(sc, cam, width, height, spp, ref_spp, seed=int(s) * 1000 + v))
        sc.close()
    return out


def train(net: Kpcn, data, steps: int, batch: int = 8, crop: int = 128, lr: float = 1e-3, seed: int = 0):
    """Adam steps on random crops (crop x crop, multiple of 4) of random
    examples. The learning rate ramps up linearly over the first 10% of the
    steps (at most 30), then decays by cosine to 5% of lr: at the full rate from the
    first step the loss overshoots (0.013 -> about 0.15 within 30 steps) and
    some runs never recover, depending only on the order of the GPU's
    floating-point atomic additions. Returns the per-step losses."""
    import torch

    rng = np.random.default_rng(seed)
    losses = []
    for k in range(steps):
        fs, ns, rs = [], [], []
        for _ in range(batch):
            ex = data[int(rng.integers(len(data)))]
            h, w = ex.feat.shape[0], ex.feat.shape[1]
            y = int(rng.integers(0, h - crop + 1)) // 4 * 4
            x = int(rng.integers(0, w - crop + 1)) // 4 * 4
            fs.append(ex.feat[y:y + crop, x:x + crop])
            ns.append(ex.noisy[y:y + crop, x:x + crop])
            rs.append(ex.ref[y:y + crop, x:x + crop])
        f = torch.stack(fs).contiguous()
        nz = torch.stack(ns).contiguous()
        rf = torch.stack(rs).contiguous()
        warm = max(1, min(30, steps // 10))
        cur = lr * min(1.0, (k + 1) / warm) * (0.05 + 0.95 * 0.5 * (1 + math.cos(math.pi * k / max(1, steps))))
        losses.append(net.train_step(f, nz, rf, cur))
    return losses


def relmse(x, ref) -> float:
    """mean over pixels and RGB of (x - ref)^2 / (ref^2 + 0.01) (CUDA tensors)."""
    a, r = x[..., :3].double(), ref[..., :3].double()
    return float(((a - r) ** 2 / (r * r + 0.01)).mean())


def svgf_denoise(ctx, gbuffer: dict, d, i, spp: int, state: Svgf | None = None):
    """SVGF (the reference's filter) on one spp-sample image: two frames of
    the same image and G-buffer, so the variance estimate and the a-trous
    passes run. `state` (an Svgf of the image's size, reset here) is reused
    when given. Returns the radiance (h, w, 4)."""
    import torch

    h, w = d.shape[0], d.shape[1]
    sv = state if state is not None else Svgf(ctx, w, h)
    sv.reset()
    nd, ni = (d / spp).contiguous(), (i / spp).contiguous()
    od, oi = torch.zeros_like(nd), torch.zeros_like(ni)
    for _ in range(2):
        sv.frame(gbuffer, gbuffer, nd, ni, od, oi)
    if state is None:
        sv.close()
    return od + oi


def evaluate(ctx, net: Kpcn, scene_seeds, width: int, height: int, spp_list, svgf_spp: int = 64,
             ref_spp: int = 4096):
    """relMSE vs a ref_spp reference per test scene (one view each): raw and
    KPCN at every spp of spp_list, SVGF at svgf_spp. Returns a dict of mean
    relMSE values."""
    import torch

    from . import scenes

    acc = {f"raw_{k}": [] for k in spp_list}
    acc.update({f"kpcn_{k}": [] for k in spp_list})
    acc[f"svgf_{svgf_spp}"] = []
    acc[f"raw_{svgf_spp}"] = []
    for s in scene_seeds:
        sc = Scene.from_spec(ctx, scenes.cornell_box(width=width, height=height, seed=int(s)))
        cam = view_cameras(sc, 1, int(s) * 7 + 3)[0]
        rd, ri = render_view(sc, cam, width, height, ref_spp, seed=int(s), first_sample=REF_FIRST_SAMPLE)
        ref = (rd + ri) / ref_spp
        for k in sorted(set(list(spp_list) + [svgf_spp])):
            d, i = render_view(sc, cam, width, height, k, seed=int(s))
            g = sc.gbuffer()
            if k in spp_list:
                feat, noisy = make_features(sc, g, d, i, k, DEPTH_SCALE)
                out = net.forward(feat[None].contiguous(), noisy[None].contiguous())[0]
                acc[f"raw_{k}"].append(relmse(noisy, ref))
                acc[f"kpcn_{k}"].append(relmse(out, ref))
            if k == svgf_spp:
                acc[f"svgf_{k}"].append(relmse(svgf_denoise(ctx, g, d, i, k), ref))
                acc[f"raw_{k}"].append(relmse((d + i) / k, ref))
        torch.cuda.synchronize()
        sc.close()
    return {k: float(np.mean(v)) for k, v in acc.items() if v}


def matching_spp(table: dict, spp_list, svgf_spp: int = 64):
    """Smallest k with KPCN relMSE at k spp <= SVGF's at svgf_spp (None if
    none)."""
    target = table[f"svgf_{svgf_spp}"]
    for k in sorted(spp_list):
        if table[f"kpcn_{k}"] <= target:
            return k
    return None


def pipeline_throughput(ctx, net: Kpcn, scene_seeds, width: int, height: int, n_requests: int, learned_spp: int,
                        plain_spp: int = 64, seed: int = 0):
    """Requests/s of two ways to serve n_requests denoised views (scene and
    pose drawn per request): the plain loop, one request at a time, renders
    plain_spp spp and runs SVGF; the learned pipeline submits all requests at
    learned_spp to the multi-scene server (continuous batching), then builds
    features and runs the KPCN on all finished images in one batch. Both
    end with the denoised radiance on the device; GPU work is synchronised
    before the clock stops."""
    import torch

    from . import scenes
    from .serve import RenderRequest, Server

    rng = np.random.default_rng(seed)
    scs = [Scene.from_spec(ctx, scenes.cornell_box(width=width, height=height, seed=int(s))) for s in scene_seeds]
    reqs = []
    for k in range(n_requests):
        si = int(rng.integers(len(scs)))
        cam = view_cameras(scs[si], 1, seed * 1000 + k)[0]
        reqs.append((si, cam, 5000 + k))

    # plain loop (warm once); one SVGF state reused across requests
    sv = Svgf(ctx, width, height)

    def plain_one(si, cam, sd):
        d, i = render_view(scs[si], cam, width, height, plain_spp, sd)
        g = scs[si].gbuffer()
        return svgf_denoise(ctx, g, d, i, plain_spp, state=sv)

    plain_one(*reqs[0])
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for r in reqs:
        plain_one(*r)
    torch.cuda.synchronize()
    plain_s = time.perf_counter() - t0
    sv.close()

    srv = Server(ctx, paths_per_pass=8 << 20)
    for sc in scs:
        srv.add_scene(sc)

    def learned_all():
        ids = [srv.submit(RenderRequest(si, width, height, learned_spp, cam, seed=sd)) for si, cam, sd in reqs]
        srv.drain()
        feats, noisy = [], []
        for rid, (si, cam, sd) in zip(ids, reqs):
            dp, ip = srv.result_device(rid)
            d = torch.empty((height, width, 4), device="cuda")
            i = torch.empty_like(d)
            d.view(-1).copy_(_wrap_device(dp, height * width * 4))
            i.view(-1).copy_(_wrap_device(ip, height * width * 4))
            sc = scs[si]
            sc.set_render_params(width=width, height=height)
            sc.set_camera_orbit(cam["target"], cam["distance"], cam["theta_deg"], cam["phi_deg"], cam["fovy_deg"])
            f, nz = make_features(sc, sc.gbuffer(), d, i, learned_spp, DEPTH_SCALE)
            feats.append(f)
            noisy.append(nz)
            srv.release(rid)
        return net.forward(torch.stack(feats).contiguous(), torch.stack(noisy).contiguous())

    learned_all()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    learned_all()
    torch.cuda.synchronize()
    learned_s = time.perf_counter() - t0
    srv.close()
    for sc in scs:
        sc.close()
    return {"requests": n_requests, "resolution": [width, height],
            "plain": {"spp": plain_spp, "denoiser": "svgf", "wall_s": round(plain_s, 4),
                      "req_per_s": round(n_requests / plain_s, 2)},
            "learned": {"spp": learned_spp, "denoiser": "kpcn", "wall_s": round(learned_s, 4),
                        "req_per_s": round(n_requests / learned_s, 2)},
            "req_per_s_ratio": round(plain_s / learned_s, 3)}


def orbit_sequence(scene: Scene, frames: int, seed: int, dphi_deg: float = 1.5):
    """Cameras of an orbit sequence: a seeded start pose (view_cameras) and
    an azimuth step of dphi_deg per frame."""
    c0 = view_cameras(scene, 1, seed)[0]
    return [dict(c0, phi_deg=c0["phi_deg"] + dphi_deg * f) for f in range(frames)]


def evaluate_sequences(ctx, net: Kpcn, scene_seeds, width: int, height: int, frames: int, spp_list,
                       svgf_spp_list=(1, 64), ref_spp: int = 4096):
    """relMSE against a ref_spp reference of every frame of an orbit
    sequence per test scene: raw and KPCN (per frame) at every spp of
    spp_list, and SVGF run as the reference runs it, temporally over the
    sequence (one Svgf state per sequence carried from frame to frame,
    G-buffer motion against the previous frame), at every spp of
    svgf_spp_list. Returns {method_spp: mean relMSE over all frames} and the
    same over the frames from the fifth on under "steady"."""
    import torch

    from . import scenes

    keys = [f"raw_{k}" for k in spp_list] + [f"kpcn_{k}" for k in spp_list]
    keys += [f"svgf_{k}" for k in svgf_spp_list] + [f"raw_{k}" for k in svgf_spp_list if k not in spp_list]
    acc = {k: [] for k in keys}
    steady = {k: [] for k in keys}
    for s in scene_seeds:
        sc = Scene.from_spec(ctx, scenes.cornell_box(width=width, height=height, seed=int(s)))
        cams = orbit_sequence(sc, frames, int(s) * 7 + 3)
        states = {k: Svgf(ctx, width, height) for k in svgf_spp_list}
        prev = None
        for f, cam in enumerate(cams):
            rd, ri = render_view(sc, cam, width, height, ref_spp, seed=int(s), first_sample=REF_FIRST_SAMPLE)
            ref = (rd + ri) / ref_spp
            g_still = sc.gbuffer()
            g_motion = sc.gbuffer(prev_camera=prev)
            res = {}
            for k in sorted(set(list(spp_list) + list(svgf_spp_list))):
                d, i = render_view(sc, cam, width, height, k, seed=int(s) * 1000 + f)
                if k in spp_list:
                    feat, noisy = make_features(sc, g_still, d, i, k, DEPTH_SCALE)
                    out = net.forward(feat[None].contiguous(), noisy[None].contiguous())[0]
                    res[f"raw_{k}"] = relmse(noisy, ref)
                    res[f"kpcn_{k}"] = relmse(out, ref)
                if k in svgf_spp_list:
                    nd, ni = (d / k).contiguous(), (i / k).contiguous()
                    od, oi = torch.empty_like(nd), torch.empty_like(ni)
                    states[k].frame(g_motion, prev_g if f else g_motion, nd, ni, od, oi)
                    res[f"svgf_{k}"] = relmse(od + oi, ref)
                    if k not in spp_list:
                        res[f"raw_{k}"] = relmse(nd + ni, ref)
            for k2, v in res.items():
                acc[k2].append(v)
                if f >= 4:
                    steady[k2].append(v)
            prev = sc.camera()
            prev_g = g_motion
        torch.cuda.synchronize()
        for st in states.values():
            st.close()
        sc.close()
    out = {k: float(np.mean(v)) for k, v in acc.items() if v}
    out["steady"] = {k: float(np.mean(v)) for k, v in steady.items() if v}
    return out


def sequence_requests(ctx, scene_seeds, width: int, height: int, frames: int, rate_per_s: float, seed: int = 0,
                      scenes_in=None):
    """Requests for the frames of one orbit sequence per scene, interleaved
    by frame (frame f of every sequence before frame f + 1), arriving as a
    Poisson process at rate_per_s (all at t = 0 when rate_per_s is 0).
    Returns (scenes, requests) with requests as dicts (scene index,
    sequence frame, camera, seed, arrival_s). scenes_in: the scenes of an
    earlier call with the same seeds, reused instead of built again."""
    from . import scenes

    scs = scenes_in or [Scene.from_spec(ctx, scenes.cornell_box(width=width, height=height, seed=int(s)))
                        for s in scene_seeds]
    seqs = [orbit_sequence(sc, frames, int(s) * 7 + 3) for sc, s in zip(scs, scene_seeds)]
    rng = np.random.default_rng(seed)
    t = 0.0
    reqs = []
    for f in range(frames):
        for si in range(len(scs)):
            t += rng.exponential(1.0 / rate_per_s) if rate_per_s > 0 else 0.0
            reqs.append({"scene": si, "frame": f, "camera": seqs[si][f], "seed": 7000 + 100 * si + f, "arrival_s": t})
    return scs, reqs


def _lat_summary(lat, wall, n):
    a = np.sort(np.asarray(lat))
    return {"requests": n, "wall_s": round(wall, 4), "req_per_s": round(n / wall, 2),
            "p50_ms": round(float(np.percentile(a, 50)) * 1e3, 2), "p99_ms": round(float(np.percentile(a, 99)) * 1e3, 2),
            "mean_ms": round(float(a.mean()) * 1e3, 2)}


def run_plain_svgf_loop(ctx, scs, reqs, width: int, height: int, spp: int = 64):
    """The plain loop, one request at a time in arrival order: render spp
    samples of the frame, its G-buffer (motion against its sequence's
    previous frame) and one SVGF frame with its sequence's temporal state;
    latency = completion - arrival (host clock, GPU synchronised)."""
    import torch

    states = [Svgf(ctx, width, height) for _ in scs]
    last = [None] * len(scs)
    dev = torch.device("cuda", ctx.device)

    def gbuf():
        return {"pos_tri": torch.empty((height, width, 4), dtype=torch.float32, device=dev),
                "normal_mat": torch.empty((height, width, 4), dtype=torch.int16, device=dev),
                "bary_mesh": torch.empty((height, width, 4), dtype=torch.int16, device=dev),
                "motion_depth": torch.empty((height, width, 4), dtype=torch.float32, device=dev)}

    gbs = [[gbuf(), gbuf()] for _ in scs]  # current / previous G-buffer per sequence
    d = torch.empty((height, width, 4), device=dev)
    i = torch.empty_like(d)
    od, oi = torch.empty_like(d), torch.empty_like(d)
    lat = []
    t0 = time.perf_counter()
    for r in reqs:
        now = time.perf_counter() - t0
        if r["arrival_s"] > now:
            time.sleep(r["arrival_s"] - now)
        si = r["scene"]
        sc = scs[si]
        sc.set_render_params(width=width, height=height, seed=r["seed"])
        c = r["camera"]
        sc.set_camera_orbit(c["target"], c["distance"], c["theta_deg"], c["phi_deg"], c["fovy_deg"])
        d.zero_()
        i.zero_()
        sc.render_device(d, i, spp)
        prev_cam = last[si]
        g, pg = gbs[si]
        sc.gbuffer(prev_camera=prev_cam, out=g)
        d.mul_(1.0 / spp)
        i.mul_(1.0 / spp)
        states[si].frame(g, pg if prev_cam is not None else g, d, i, od, oi)
        torch.cuda.synchronize()
        lat.append(time.perf_counter() - t0 - r["arrival_s"])
        last[si] = sc.camera()
        gbs[si] = [pg, g]
    wall = time.perf_counter() - t0
    for st in states:
        st.close()
    return _lat_summary(lat, wall, len(reqs))


def learned_server(ctx, scs, paths_per_pass: int = 8 << 20):
    """A multi-scene server holding scs (in order) for run_learned_served."""
    from .serve import Server

    srv = Server(ctx, paths_per_pass=paths_per_pass)
    for sc in scs:
        srv.add_scene(sc)
    return srv


def run_learned_served(ctx, net: Kpcn, scs, reqs, width: int, height: int, spp: int, paths_per_pass: int = 8 << 20,
                       server=None):
    """The learned pipeline, open loop: each request is submitted to the
    multi-scene server (continuous batching) at spp when it arrives; the
    requests that finish rendering in a server step get their G-buffer and
    features (built straight from the server's accumulators into one batch)
    and go through one batched KPCN forward together; latency = completion
    of that forward - arrival. server: a long-lived server from
    learned_server(ctx, scs) (its wavefront and accumulator pool stay
    allocated between runs, as in a serving process); without one a server
    is created and closed inside the timed loop."""
    import torch

    from .serve import DONE, RenderRequest

    srv = server or learned_server(ctx, scs, paths_per_pass)
    n = len(reqs)
    lat = [0.0] * n
    ids = {}
    done = 0
    k = 0
    dev = torch.device("cuda", ctx.device)
    g = {"pos_tri": torch.empty((height, width, 4), dtype=torch.float32, device=dev),
         "normal_mat": torch.empty((height, width, 4), dtype=torch.int16, device=dev),
         "bary_mesh": torch.empty((height, width, 4), dtype=torch.int16, device=dev),
         "motion_depth": torch.empty((height, width, 4), dtype=torch.float32, device=dev)}
    feats = torch.empty((n, height, width, 16), dtype=torch.bfloat16, device=dev)
    noisy = torch.empty((n, height, width, 4), dtype=torch.float32, device=dev)
    outb = torch.empty((n, height, width, 4), dtype=torch.float32, device=dev)
    for sc in scs:
        sc.set_render_params(width=width, height=height)
    # size the network's buffers for the largest batch (every request at
    # once); smaller batches reuse them
    net.forward(feats, noisy, out=outb)
    torch.cuda.synchronize()
    tm = {"submit_s": 0.0, "step_s": 0.0, "poll_s": 0.0, "features_s": 0.0, "forward_s": 0.0}
    t0 = time.perf_counter()
    while done < n:
        ta = time.perf_counter()
        now = ta - t0
        while k < n and reqs[k]["arrival_s"] <= now:
            r = reqs[k]
            ids[srv.submit(RenderRequest(r["scene"], width, height, spp, r["camera"], seed=r["seed"]))] = k
            k += 1
        tb = time.perf_counter()
        nd = srv.step(wait=k == n)
        tc = time.perf_counter()
        tm["submit_s"] += tb - ta
        tm["step_s"] += tc - tb
        if nd:
            fin = [(rid, j) for rid, j in ids.items() if srv.poll(rid) == DONE]
            td = time.perf_counter()
            for b, (rid, j) in enumerate(fin):
                r = reqs[j]
                dp, ip = srv.result_device(rid)
                sc = scs[r["scene"]]
                c = r["camera"]
                sc.set_camera_orbit(c["target"], c["distance"], c["theta_deg"], c["phi_deg"], c["fovy_deg"])
                sc.gbuffer(out=g)
                make_features(sc, g, dp, ip, spp, DEPTH_SCALE, out=(feats[b], noisy[b]))
            te = time.perf_counter()
            tm["poll_s"] += td - tc
            tm["features_s"] += te - td
            if fin:
                m = len(fin)
                net.forward(feats[:m], noisy[:m], out=outb[:m])
                # this batch's stream only: the server's next passes keep running
                torch.cuda.current_stream().synchronize()
                for rid, _ in fin:
                    srv.release(rid)
                    del ids[rid]
                now = time.perf_counter() - t0
                tm["forward_s"] += now + t0 - te
                for _, j in fin:
                    lat[j] = now - reqs[j]["arrival_s"]
                done += m
        elif k < n and not ids:
            time.sleep(min(2e-4, max(0.0, reqs[k]["arrival_s"] - (time.perf_counter() - t0))))
    wall = time.perf_counter() - t0
    if server is None:
        srv.close()
    out = _lat_summary(lat, wall, n)
    out["host_time_split_s"] = {k2: round(v, 4) for k2, v in tm.items()}
    return out


def _wrap_device(ptr: int, count: int):
    """A float32 CUDA tensor view of `count` floats at device address ptr
    (server-owned memory, valid until the request is released)."""
    import torch

    class _Arr:
        __cuda_array_interface__ = {"shape": (count,), "typestr": "<f4", "data": (ptr, False), "version": 3}

    return torch.as_tensor(_Arr(), device="cuda")
