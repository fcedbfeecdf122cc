"""Benchmark: extend + shadow ray throughput of the wavefront path tracer on
the traversal-throughput scene (64 level-5 icospheres, 1,310,720 triangles),
16M closest-hit rays + 16M Light::Visible shadow queries per step per GPU.

python bench.py [--gpus N] [--steps K] [--warmup W] [--impl crt|reference]

* value   : (extend + shadow rays) / s over all ranks, device-resident
            inputs, CUDA events on the launching stream, max over ranks.
* e2e     : the same through the public host-buffer API (crt_trace_closest
            / crt_trace_shadow on pinned host arrays; copies inside).
* roofline: the dominant launch of the step (the shadow kernel on this
            workload; the extend kernel if it ever takes longer), its
            algorithmic bytes (shadow 49 B per query: 48 B in + 1 B out;
            extend 48 B per ray: 32 B ray in + 16 B hit out) over its
            event-timed duration, against the measured HBM copy bandwidth.
* cpu_baseline: the reference's own BVH traversal and visibility test
            (oracle/_ref, host-compiled) on the host cores, bounded sample.
--impl reference runs that reference CPU implementation as the timed arm.
Multi-GPU: one process per GPU (torchrun), each traces its own batch
(weak scaling, no data-path collective).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_RAYS = 16 << 20
EXTEND_BYTES = 48  # per ray: 32 B in + 16 B hit out
SHADOW_BYTES = 49  # per query: 48 B in + 1 B out
METRIC = "extend+shadow Mrays/s (icosphere field 1.31M tris, 16M+16M rays/GPU)"


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("LOCAL_RANK", 0)), int(os.environ.get("WORLD_SIZE", 1))


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) per 16M-ray
# launch of each trace kernel, from one ncu capture of an 8M-ray launch of
# the same kernel build on the same batch distribution, scaled x2 (ray bytes
# scale exactly, node visits linearly for uniform random rays). The capture
# and its command are summarised in profiles/ (traversal summary).
TRAFFIC_PER_16M = {"extend": 2 * (564561664 + 132257024), "shadow": 2 * (1538991104 + 26396672)}


def profiled_traffic(kernel: str):
    """Per-launch DRAM bytes (16M-ray launch) of `kernel` ("extend" or
    "shadow"), or None if not captured."""
    return TRAFFIC_PER_16M.get(kernel)


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpus):
        self.gpus = set(gpus)
        self.proc = None
        self.path = os.path.join("/tmp", f"crt_clocks_{os.getpid()}.csv")

    def start(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        self.proc.wait()
        self.f.close()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            c = [x.strip() for x in line.split(",")]
            if len(c) < 9 or not c[0].isdigit() or int(c[0]) not in self.gpus:
                continue
            try:
                sm.append(float(c[1]))
                smax.append(float(c[2]))
            except ValueError:
                continue
            for nm, v in zip(names, c[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def reference_cpu(tris, rays, queries, threads):
    """Times the reference's host-compiled traversal (oracle/_ref) or, if it
    is absent, reports None. Returns (Mrays/s, seconds, kind)."""
    import oracle

    if not oracle.ref_available():
        return None
    ref = oracle.RefScene(tris)
    t0 = time.perf_counter()
    ref.trace_closest(rays, threads)
    ref.visible(queries, threads)
    dt = time.perf_counter() - t0
    ref.close()
    return (len(rays) + len(queries)) / dt / 1e6, dt


def reference_cuda(tris, rays, qs, hits_mine, occ_mine, steps, stream):
    """Times the reference's own traversal built for the GPU (oracle/_ref,
    headless CUDA builds: -rdc, and with device link-time optimisation) on
    the same device batch and checks its hit records against ours. Returns
    the faster build's dict, with both builds' timings under "builds", or
    None when no build is present."""
    import oracle

    runs = {}
    for lto in (False, True):
        if oracle.ref_cuda_available(lto):
            runs["dlto" if lto else "rdc"] = _reference_cuda_build(tris, rays, qs, hits_mine, occ_mine, steps, stream,
                                                                   lto)
    if not runs:
        return None
    best = max(runs.values(), key=lambda r: r["value"])
    return {**best, "builds": {k: {a: r[a] for a in ("value", "extend_ms_per_launch", "shadow_ms_per_launch")}
                               for k, r in runs.items()}}


def _reference_cuda_build(tris, rays, qs, hits_mine, occ_mine, steps, stream, lto):
    import torch

    import oracle

    ref = oracle.RefCudaScene(tris, lto=lto)
    n = rays.shape[0]
    out = torch.empty_like(hits_mine)
    occ = torch.empty_like(occ_mine)
    s = stream.cuda_stream
    ref.trace(rays.data_ptr(), n, out.data_ptr(), s)
    ref.visible(qs.data_ptr(), n, occ.data_ptr(), s)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    ev[0].record(stream)
    for _ in range(steps):
        ref.trace(rays.data_ptr(), n, out.data_ptr(), s)
    ev[1].record(stream)
    for _ in range(steps):
        ref.visible(qs.data_ptr(), n, occ.data_ptr(), s)
    ev[2].record(stream)
    torch.cuda.synchronize()
    ext = ev[0].elapsed_time(ev[1]) / steps
    sh = ev[1].elapsed_time(ev[2]) / steps
    same_prim = (out[:, 1].view(torch.int32) == hits_mine[:, 1].view(torch.int32))
    hit = hits_mine[:, 1].view(torch.int32) >= 0
    rel = ((out[:, 0] - hits_mine[:, 0]).abs() / hits_mine[:, 0].abs().clamp_min(1e-30))
    res = {"value": round(2 * n / ((ext + sh) * 1e-3) / 1e6, 2), "unit": "Mrays/s",
           "extend_ms_per_launch": round(ext, 4), "shadow_ms_per_launch": round(sh, 4),
           "prim_identical_frac": float(same_prim.float().mean().item()),
           "t_bit_identical_frac_of_hits": float((same_prim & hit & (out[:, 0] == hits_mine[:, 0])).sum().item()
                                                 / max(1, int(hit.sum().item()))),
           "t_within_1e-6_rel_frac_of_hits": float((same_prim & hit & (rel <= 1e-6)).sum().item()
                                                   / max(1, int(hit.sum().item()))),
           "note": "the reference's device build contracts multiply-adds (nvcc default), so its t differs "
                   "from its own IEEE host build in the last bits; ours equals the host build bit for bit",
           "occluded_identical_frac": float((occ == occ_mine).float().mean().item()),
           "build": "reference sources, nvcc -O3 -rdc " + ("-dlto " if lto else "") +
                    "-arch sm_100a, BVH built on the host"}
    ref.close()
    return res


def cornell_trace_leg(ctx, stream, reps=20, with_reference=True):
    """Traversal on the Cornell box (36 triangles): 1M fixed closest-hit rays
    (seed 1: origins uniform in the scene box, directions uniform on the
    sphere) + 1M Light::Visible queries (seed 2), device-resident, CUDA
    events over `reps` launches of each after a warm-up; then the reference's
    own traversal built for the GPU on the same device batch, with its hit
    records compared to ours. Returns a dict (Mrays/s of both, their ratio)."""
    import torch

    from cudaraytracer_b200 import Scene, scenes

    n = 1 << 20
    tris = scenes.cornell_box().triangles()
    dev = torch.device("cuda", ctx.device)
    rays = torch.from_numpy(scenes.random_rays(tris, n, seed=1)).to(dev)
    qs = torch.from_numpy(scenes.random_shadow_queries(tris, n, seed=2)).to(dev)
    hits = torch.empty((n, 4), dtype=torch.float32, device=dev)
    occ = torch.empty((n,), dtype=torch.uint8, device=dev)
    sc = Scene.from_triangles(ctx, tris)
    for _ in range(5):
        sc.trace_closest(rays, hits)
        sc.trace_shadow(qs, occ)
    torch.cuda.synchronize()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    ev[0].record(stream)
    for _ in range(reps):
        sc.trace_closest(rays, hits)
    ev[1].record(stream)
    for _ in range(reps):
        sc.trace_shadow(qs, occ)
    ev[2].record(stream)
    torch.cuda.synchronize()
    ext = ev[0].elapsed_time(ev[1]) / reps
    sh = ev[1].elapsed_time(ev[2]) / reps
    out = {"workload": "Cornell box 36 tris; 1M closest-hit rays (seed 1) + 1M shadow queries (seed 2)",
           "value": round(2 * n / ((ext + sh) * 1e-3) / 1e6, 1), "unit": "Mrays/s",
           "extend_ms_per_launch": round(ext, 4), "shadow_ms_per_launch": round(sh, 4),
           "hit_rate": float((hits[:, 1].view(torch.int32) >= 0).float().mean().item()),
           "occluded_frac": float(occ.float().mean().item())}
    if with_reference:
        ref = reference_cuda(tris, rays, qs, hits, occ, reps, stream)
        if ref is not None:
            out["reference_cuda"] = ref
            out["ratio_vs_reference_cuda"] = round(out["value"] / ref["value"], 2)
    sc.close()
    return out


def render_leg(ctx, steps, stream, with_reference=True):
    """Full wavefront render of the traversal scene at 1920x1080 (depth 16,
    2048x1024 sky+sun environment map, the four materials), 4 samples per
    pixel per step, and the same through the reference's own renderer built
    headless (oracle/_ref). Returns a dict (samples/s and spp/s)."""
    import tempfile

    import torch

    from cudaraytracer_b200 import Scene, scenes

    td = tempfile.mkdtemp(prefix="crt_bench_")
    path = scenes.icosphere_field().write(td, "icospheres")
    sc = Scene.load(ctx, path)
    rp = sc.render_params()
    W, H = rp["width"], rp["height"]
    step_spp = 4
    dev = torch.device("cuda", ctx.device)
    d = torch.zeros((H, W, 4), device=dev)
    i = torch.zeros((H, W, 4), device=dev)
    sc.render_device(d, i, step_spp, first_sample=0, stream=stream.cuda_stream)
    torch.cuda.synchronize()
    ext0, sh0 = sc.ray_counts(stream=stream.cuda_stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for k in range(steps):
        sc.render_device(d, i, step_spp, first_sample=step_spp * (k + 1), stream=stream.cuda_stream)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    ext1, sh1 = sc.ray_counts(stream=stream.cuda_stream)
    vertices, shadow_rays = ext1 - ext0, sh1 - sh0
    spp_total = steps * step_spp
    peak, kind = measured_peaks()
    ach = PATH_VERTEX_BYTES * vertices / (ms * 1e-3) / 1e9
    out = {"scene": "icosphere field 1920x1080, depth 16, env 2048x1024", "spp_per_step": step_spp,
           "spp_per_s": round(spp_total / (ms * 1e-3), 2),
           "msamples_per_s": round(W * H * spp_total / (ms * 1e-3) / 1e6, 2),
           "ms_per_spp": round(ms / spp_total, 3),
           "path_vertices": vertices, "shadow_rays": shadow_rays,
           "vertices_per_sample": round(vertices / (W * H * spp_total), 3),
           "mrays_per_s": round((vertices + shadow_rays) / (ms * 1e-3) / 1e6, 1),
           "roofline": {"bound": "hbm", "bytes_per_vertex": PATH_VERTEX_BYTES, "achieved": round(ach, 1),
                        "peak": peak, "unit": "GB/s", "frac": round(ach / peak, 4), "peak_kind": kind}}
    t0 = time.perf_counter()
    sc.render(step_spp)
    out["e2e_ms_per_spp_host_api"] = round((time.perf_counter() - t0) * 1e3 / step_spp, 3)
    if with_reference:
        import oracle

        runs = {}
        for lto in (False, True):  # -rdc and device-LTO builds; the faster one is the reference's number
            if oracle.ref_render_available(lto):
                ref = oracle.RefRenderer(path, lto=lto)
                ref.render(1, with_sumsq=False)
                frames = 2
                _, _, _, rms = ref.render(frames, with_sumsq=False)
                runs["dlto" if lto else "rdc"] = {
                    "msamples_per_s": round(W * H * frames / (rms * 1e-3) / 1e6, 3), "ms_per_spp": round(rms / frames, 2),
                    "build": "reference renderer.cuh + Scene, nvcc -O3 -rdc " + ("-dlto " if lto else "") +
                             "sm_100a, headless"}
        if runs:
            best = min(runs.values(), key=lambda r: r["ms_per_spp"])
            out["reference_cuda"] = {**best, "builds": {k: r["ms_per_spp"] for k, r in runs.items()}}
    sc.close()
    return out


# Algorithmic bytes per path vertex of the wavefront render: extend 48
# (ray in, hit out) + shade (hit 16 + path state 64 in, new ray 32 + path
# state 64 out, shadow record 44) + shadow 36 + accumulation 16.
PATH_VERTEX_BYTES = 48 + 16 + 64 + 32 + 64 + 44 + 36 + 16
SVGF_BYTES_PER_PIXEL = 176 + 112 + 5 * 100  # temporal, variance, 5 a-trous passes (planes read + written once)


def svgf_leg(ctx, stream, frames=4, with_reference=True):
    """SVGF at 1920x1080 on the icosphere field: an orbiting camera
    (0.5 deg per frame), 1-spp noisy direct/indirect and the primary-hit
    G-buffer per frame, then one SVGF frame (temporal reprojection,
    variance, 5 a-trous passes), timed with CUDA events. The reference's
    own SVGF kernels (headless CUDA build) run on the same inputs, timed
    per frame the same way. Frames after the first (which skips the
    a-trous passes) are reported; roofline: 788 B per pixel per frame
    (temporal 176, variance 112, a-trous 5 x 100) over the frame time."""
    import tempfile

    import torch

    from cudaraytracer_b200 import Scene, Svgf, scenes

    td = tempfile.mkdtemp(prefix="crt_svgf_")
    sc = Scene.load(ctx, scenes.icosphere_field().write(td, "icospheres"))
    rp = sc.render_params()
    W, H = rp["width"], rp["height"]
    shape = (H, W, 4)
    dev = torch.device("cuda", ctx.device)
    cam0 = sc.camera()
    sv = Svgf(ctx, W, H)
    ins, gbs = [], []
    prev = None
    for f in range(frames):
        sc.set_camera_orbit(cam0["target"], cam0["distance"], cam0["theta_deg"], cam0["phi_deg"] + 0.5 * f,
                            cam0["fovy_deg"])
        d = torch.zeros(shape, device=dev)
        i = torch.zeros(shape, device=dev)
        sc.render_device(d, i, 1, first_sample=f, stream=stream.cuda_stream)
        g = sc.gbuffer(prev_camera=prev, stream=stream.cuda_stream)
        prev = sc.camera()
        ins.append((d, i))
        gbs.append(g)
    torch.cuda.synchronize()
    zero = {k: torch.zeros_like(v) for k, v in gbs[0].items()}
    outs, ms = [], []
    for f in range(frames):
        od = torch.empty(shape, device=dev)
        oi = torch.empty(shape, device=dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        sv.frame(gbs[f], gbs[f - 1] if f else zero, ins[f][0], ins[f][1], od, oi, stream=stream.cuda_stream)
        e1.record(stream)
        torch.cuda.synchronize()
        ms.append(e0.elapsed_time(e1))
        outs.append((od, oi))
    mine = float(np.median(ms[1:]))
    px = W * H
    from_peak, kind = measured_peaks()
    ach = SVGF_BYTES_PER_PIXEL * px / (mine * 1e-3) / 1e9
    out = {"workload": "icosphere field 1920x1080, 1 spp per frame, orbit 0.5 deg/frame, 5 a-trous passes",
           "ms_per_frame": round(mine, 4), "ms_frames": [round(x, 4) for x in ms],
           "roofline": {"bound": "hbm", "bytes_per_pixel": SVGF_BYTES_PER_PIXEL, "achieved": round(ach, 1),
                        "peak": from_peak, "unit": "GB/s", "frac": round(ach / from_peak, 4), "peak_kind": kind}}
    if with_reference:
        import oracle

        if oracle.ref_render_available():
            host = lambda t: t.cpu().numpy()
            nd = np.stack([host(d) for d, _ in ins])
            ni = np.stack([host(i) for _, i in ins])
            g = {k: np.stack([host(gb[k]) for gb in gbs]) for k in gbs[0]}
            rd, ri, rms = oracle.ref_svgf(nd, ni, g["pos_tri"], g["normal_mat"].view(np.uint16),
                                          g["bary_mesh"].view(np.uint16), g["motion_depth"], timing=True)
            ref_ms = float(np.median(rms[1:]))
            builds = {"rdc": round(ref_ms, 4)}
            build = "reference renderer.cuh SVGF kernels, nvcc -O3 -rdc sm_100a, headless"
            if oracle.ref_render_available(lto=True):  # the device-LTO build; the faster one counts
                _, _, rms_lto = oracle.ref_svgf(nd, ni, g["pos_tri"], g["normal_mat"].view(np.uint16),
                                                g["bary_mesh"].view(np.uint16), g["motion_depth"], timing=True,
                                                lto=True)
                lto_ms = float(np.median(rms_lto[1:]))
                builds["dlto"] = round(lto_ms, 4)
                if lto_ms < ref_ms:
                    ref_ms, rms = lto_ms, rms_lto
                    build = "reference renderer.cuh SVGF kernels, nvcc -O3 -rdc -dlto sm_100a, headless"
            crt_out = np.stack([np.stack([host(od), host(oi)]) for od, oi in outs])[..., :3].astype(np.float64)
            ref = np.stack([np.stack([rd[f], ri[f]]) for f in range(frames)])[..., :3].astype(np.float64)
            dif = np.abs(crt_out - ref)
            out["reference_cuda"] = {"ms_per_frame": round(ref_ms, 4), "ms_frames": [round(float(x), 4) for x in rms],
                                     "build": build, "builds": builds,
                                     "outputs_vs_crt": {
                                         "max_abs_diff": float(dif.max()), "max_abs_value": float(np.abs(ref).max()),
                                         "frac_above_1e-3_abs": float((dif > 1e-3).mean()),
                                         "frac_above_1e-3_rel": float((dif > 1e-3 * np.maximum(1.0, np.abs(ref))).mean()),
                                         "max_rel_diff_where_ref_above_1": float(
                                             (dif / np.maximum(1.0, np.abs(ref))).max())}}
            out["speedup_vs_reference_cuda"] = round(ref_ms / mine, 2)
    sv.close()
    sc.close()
    return out


def batch_leg(ctx, stream):
    """Batched persistent wavefront (the multi-view batch workload): 64 orbit views of
    the Cornell box (radius 3, elevation U[-30, 30] deg, seeded), 512x512,
    16 spp, depth 12, all views in shared wavefronts with a CUDA graph per
    pass and an autotuned wavefront size, stage block size and stage
    traversal (stack placement, node format), against 64 sequential
    single-view renders of the same cameras with the same settings."""
    import tempfile

    import torch

    from cudaraytracer_b200 import Scene, scenes
    from cudaraytracer_b200.autotune import autotune_paths_per_pass, orbit_views

    td = tempfile.mkdtemp(prefix="crt_batch_")
    sc = Scene.load(ctx, scenes.cornell_box(width=512, height=512, spp=16, max_bounces=12).write(td, "cb"))
    views = orbit_views(sc, 64, radius=3.0, max_elev_deg=30.0, seed=1)
    spp = 16
    tune = autotune_paths_per_pass(sc, views, probe_spp=1,
                                   candidates=(2 << 20, 4 << 20, 8 << 20, 16 << 20))
    rp = sc.render_params()
    shape = (len(views), rp["height"], rp["width"], 4)
    d = torch.zeros(shape, device="cuda")
    i = torch.zeros(shape, device="cuda")
    e = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    e[0].record(stream)
    sc.render_views(views, d, i, spp, stream=stream.cuda_stream)
    e[1].record(stream)
    sd = torch.zeros(shape[1:], device="cuda")
    si = torch.zeros(shape[1:], device="cuda")
    torch.cuda.synchronize()
    e[2].record(stream)
    for v in views:
        sc.set_camera_orbit(v["target"], v["distance"], v["theta_deg"], v["phi_deg"], v["fovy_deg"])
        sc.render_device(sd, si, spp, stream=stream.cuda_stream)
    e[3].record(stream)
    torch.cuda.synchronize()
    bms, sms = e[0].elapsed_time(e[1]), e[2].elapsed_time(e[3])
    samples = len(views) * rp["width"] * rp["height"] * spp
    sc.close()
    return {"workload": "64 views x 512x512 x 16 spp, Cornell box, depth 12", "batched_ms": round(bms, 2),
            "sequential_ms": round(sms, 2), "speedup": round(sms / bms, 3),
            "batched_msamples_per_s": round(samples / (bms * 1e-3) / 1e6, 1),
            "sequential_msamples_per_s": round(samples / (sms * 1e-3) / 1e6, 1),
            "paths_per_pass": tune["paths_per_pass"], "stage_block": tune["stage_block"],
            "stage_traversal": tune["stage_traversal"],
            "autotune_ms": tune.get("timings_ms"), "autotune_block_ms": tune.get("block_timings_ms"),
            "autotune_traversal_ms": tune.get("traversal_timings_ms")}


def serve_leg(ctx, quick=False):
    """Serving (the multi-scene request workload) on a bounded sample. 8 resident scenes of
    the icosphere-field generator with {1, 4, 8, 16, 32, 64, 128, 256}
    level-5 spheres (20k to 5.2M triangles, 2048x1024 env each). Requests
    draw resolution from {256^2, 512^2, 1280x720, 1920x1080}, spp from
    {1, 4, 16, 64} and a random orbit pose. Poisson arrivals at 5, 20 and
    80 per second (100, 300 and 320 requests instead of 2,000 per rate) and
    a saturated burst (160 requests at t=0), each served by crt_server
    (continuous batching, HBM budget 150 GiB, 8M-path wavefronts, passes
    filled shortest-remaining-first; at 80/s and in the burst also in
    admission order) and by the one-request-at-a-time loop
    (Scene.render_device per request) over the same requests. Latency =
    completion - arrival (host clock), overall and per request class
    (resolution x spp)."""
    from cudaraytracer_b200 import Scene, scenes
    from cudaraytracer_b200.serve import Server, poisson_requests, run_one_at_a_time, run_served

    counts = (1, 4, 8, 16, 32, 64, 128, 256)
    t0 = time.perf_counter()
    scs = [Scene.from_spec(ctx, scenes.icosphere_field(n_spheres=c, seed=100 + k)) for k, c in enumerate(counts)]
    load_s = time.perf_counter() - t0
    cams = [sc.camera() for sc in scs]
    res = [(256, 256), (512, 512), (1280, 720), (1920, 1080)]
    spps = [1, 4, 16, 64]
    srv = Server(ctx, hbm_budget_bytes=150 << 30, paths_per_pass=8 << 20, passes_in_flight=2)
    fifo = Server(ctx, hbm_budget_bytes=150 << 30, paths_per_pass=8 << 20, passes_in_flight=2,
                  schedule=Server.ADMISSION_ORDER)
    for sc in scs:
        srv.add_scene(sc)
        fifo.add_scene(sc)
    warm = poisson_requests(8, 0.0, cams, res, [1, 4], seed=99)
    run_served(srv, warm)
    run_served(fifo, warm)
    run_one_at_a_time(scs, warm)
    plan = [(5.0, 100), (20.0, 300), (80.0, 320)] if not quick else [(80.0, 48)]
    out = {"workload": "8 resident icosphere-field scenes (1..256 level-5 spheres, 20k-5.2M tris); requests of "
                       "{256^2, 512^2, 1280x720, 1920x1080} x {1, 4, 16, 64} spp, random poses",
           "scenes_tris": [int(sc.info()["num_triangles"]) for sc in scs], "scene_build_s": round(load_s, 2),
           "hbm": {k: v for k, v in srv.stats().items() if k.startswith("bytes")}, "rates": {}}
    for rate, n in plan:
        reqs = poisson_requests(n, rate, cams, res, spps, seed=int(rate))
        served = run_served(srv, reqs)
        leg = {"served": served}
        if rate >= 80.0:
            leg["served_admission_order"] = run_served(fifo, reqs)
        leg["one_at_a_time"] = run_one_at_a_time(scs, reqs)
        out["rates"][f"{rate:g}/s"] = leg
    burst = poisson_requests(160 if not quick else 32, 0.0, cams, res, spps, seed=7)
    served = run_served(srv, burst)
    served_fifo = run_served(fifo, burst)
    plain = run_one_at_a_time(scs, burst)
    out["saturated"] = {"served": served, "served_admission_order": served_fifo, "one_at_a_time": plain,
                        "req_per_s_ratio": round(served["req_per_s"] / plain["req_per_s"], 3)}
    out["schedule"] = "served: shortest remaining paths first (oldest request keeps half of each pass); " \
                      "served_admission_order: first come, first served"
    out["server_stats"] = {k: v for k, v in srv.stats().items() if k in ("passes", "paths")}
    srv.close()
    fifo.close()
    for sc in scs:
        sc.close()
    return out


def conv_leg(ctx, h=1080, w=1920, cin=64, cout=64, reps=10):
    """Tensor-core 3x3 convolution at 1920x1080 with 64 -> 64 channels
    (the denoiser's most common shape): forward (bias + ReLU), data gradient
    and weight gradient, each timed with CUDA events over `reps` launches
    after a warm-up. FLOPs = 2 * 9 * cin * cout * pixels per launch;
    roofline against the measured BF16 peak (burst)."""
    import torch

    from cudaraytracer_b200 import kpcn

    g = torch.Generator(device="cuda").manual_seed(0)
    x = torch.randn((1, h, w, cin), device="cuda", generator=g).to(torch.bfloat16)
    wt = (torch.randn((9, cout, cin), device="cuda", generator=g) / 24).to(torch.bfloat16)
    wtt = wt.permute(0, 2, 1).contiguous()
    b = torch.zeros(cout, device="cuda")
    gy = torch.randn((1, h, w, cout), device="cuda", generator=g).to(torch.bfloat16)
    y = torch.empty((1, h, w, cout), dtype=torch.bfloat16, device="cuda")
    gx = torch.empty((1, h, w, cin), dtype=torch.bfloat16, device="cuda")
    dw = torch.zeros((9, cout, cin), device="cuda")
    ops = {"forward": lambda: kpcn.conv3x3_forward(ctx, x, wt, b, relu=True, out=y),
           "backward_data": lambda: kpcn.conv3x3_backward_data(ctx, gy, wtt, out=gx),
           "backward_weights": lambda: kpcn.conv3x3_backward_weights(ctx, x, gy, dw=dw)}
    pp = os.path.join(ROOT, "MEASURED_PEAKS.json")
    peak, kind = (float(json.load(open(pp))["bf16_tflops"]), "measured") if os.path.exists(pp) else (1590.0, "fallback")
    flops = 2.0 * 9 * cin * cout * h * w
    out = {"shape": f"1x{h}x{w}, {cin}->{cout}", "flops_per_launch": flops, "peak_tflops": peak, "peak_kind": kind}
    for name, fn in ops.items():
        # warm up for at least 200 ms so the timed launches run at boost clocks
        t_end = time.perf_counter() + 0.2
        while time.perf_counter() < t_end:
            for _ in range(3):
                fn()
            torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / reps
        tf = flops / (ms * 1e-3) / 1e12
        out[name] = {"ms_per_launch": round(ms, 4), "tflops": round(tf, 1), "frac": round(tf / peak, 4)}
    kpcn.check_device_errors(ctx)
    return out


def kpcn_layers_leg(ctx, reps=10):
    """The denoiser network at 1920x1080: each of its 11 convolutions
    timed alone at its own resolution (full, 1/2, 1/4) and channel counts
    (forward, bias + ReLU), and the whole forward pass of one frame
    (convolutions, pooling, upsampling, softmax filter). FLOPs per
    convolution = 2 * 9 * cin * cout * pixels."""
    import torch

    from cudaraytracer_b200 import kpcn
    from cudaraytracer_b200.kpcn import Kpcn

    H, W = 1080, 1920
    scale = {"e0a": 1, "e0b": 1, "e1a": 2, "e1b": 2, "e2a": 4, "e2b": 4, "d1a": 2, "d1b": 2, "d0a": 1, "d0b": 1,
             "out": 1}
    pp = os.path.join(ROOT, "MEASURED_PEAKS.json")
    peak = float(json.load(open(pp))["bf16_tflops"]) if os.path.exists(pp) else 1590.0
    g = torch.Generator(device="cuda").manual_seed(1)
    layers, total_ms, total_flop = {}, 0.0, 0.0

    def timed(fn):
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    for name, (cin, cout) in zip(Kpcn.LAYERS, Kpcn.SPEC):
        h, w = H // scale[name], W // scale[name]
        x = torch.randn((1, h, w, cin), device="cuda", generator=g).to(torch.bfloat16)
        wt = (torch.randn((9, cout, cin), device="cuda", generator=g) / 24).to(torch.bfloat16)
        b = torch.zeros(cout, device="cuda")
        y = torch.empty((1, h, w, cout), dtype=torch.bfloat16, device="cuda")
        ms = timed(lambda: kpcn.conv3x3_forward(ctx, x, wt, b, relu=name != "out", out=y))
        flop = 2.0 * 9 * cin * cout * h * w
        total_ms += ms
        total_flop += flop
        layers[name] = {"shape": f"{w}x{h}, {cin}->{cout}", "ms": round(ms, 4),
                        "tflops": round(flop / (ms * 1e-3) / 1e12, 1), "frac": round(flop / (ms * 1e-3) / 1e12 / peak, 4)}
        del x, wt, y
    net = Kpcn(ctx, seed=0)
    feat = torch.randn((1, H, W, 16), device="cuda", generator=g).to(torch.bfloat16)
    noisy = torch.rand((1, H, W, 4), device="cuda", generator=g)
    out = torch.empty((1, H, W, 4), device="cuda")
    fwd = timed(lambda: net.forward(feat, noisy, out=out))
    net.close()
    kpcn.check_device_errors(ctx)
    return {"resolution": [W, H], "layers": layers, "conv_ms_sum": round(total_ms, 4),
            "conv_gflop": round(total_flop / 1e9, 1), "conv_tflops": round(total_flop / (total_ms * 1e-3) / 1e12, 1),
            "conv_frac": round(total_flop / (total_ms * 1e-3) / 1e12 / peak, 4), "forward_ms_per_frame": round(fwd, 4),
            "peak_tflops": peak}


def denoise_leg(ctx, train_steps=6000):
    """Learned denoiser against SVGF (the learned-denoiser workload, at
    256x256 instead of 1920x1080 and 16-frame instead of 60-frame
    sequences so the 4096-spp references fit the bench): the KPCN is
    trained on the GPU on 64 views of seeded Cornell variants (scene seeds
    100-163, one view each, 1-16 spp inputs, 4096-spp references) for
    6000 Adam steps of 8 random 128x128 crops. Test: one 16-frame orbit
    sequence (1.5 deg per frame) per unseen scene (seeds 200-207), relMSE
    of every frame against its 4096-spp reference for raw and KPCN at 1-32
    spp and for SVGF run temporally over the sequence at 1 and 64 spp.
    The smallest spp at which KPCN matches 64 spp + temporal SVGF sets the
    learned pipeline. Serving (same 256x256 frames, same sequences): the
    plain loop (one request at a time: 64 spp render, G-buffer, SVGF frame
    with the sequence's state) against the learned pipeline (requests
    through the multi-scene server at the matching spp, finished requests'
    KPCN batched; a long-lived server warmed by an untimed burst), both for
    a burst of all 128 frames at t = 0 (throughput; the learned pipeline
    also at twice the matching spp, since the match itself moves between
    trainings) and for Poisson arrivals at 70% of the plain loop's
    throughput (latency)."""
    import torch

    from cudaraytracer_b200 import denoise as D
    from cudaraytracer_b200.kpcn import Kpcn

    res = 256
    t0 = time.perf_counter()
    data = D.build_dataset(ctx, range(100, 164), 1, res, res, [1, 2, 4, 8, 16], 4096, seed=0)
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    net = Kpcn(ctx, seed=0)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    losses = D.train(net, data, train_steps, batch=8, crop=128, lr=1e-3)
    e1.record()
    torch.cuda.synchronize()
    t2 = time.perf_counter()
    del data
    spp_list = [1, 2, 4, 8, 16, 32]
    frames = 16
    tab = D.evaluate_sequences(ctx, net, range(200, 208), res, res, frames, spp_list, svgf_spp_list=(1, 64))
    t3 = time.perf_counter()
    k = D.matching_spp(tab, spp_list) or 32
    scs, burst = D.sequence_requests(ctx, range(200, 208), res, res, frames, 0.0)
    # both pipelines keep their state between requests: the plain loop its
    # scenes' wavefronts and SVGF states, the learned one a long-lived server
    # (wavefront, accumulator pool) warmed by one untimed burst at each spp
    srv = D.learned_server(ctx, scs)
    k2 = min(2 * k, 32)
    D.run_plain_svgf_loop(ctx, scs, burst[:8], res, res)  # warm-up
    for kk in sorted({k, k2}):
        D.run_learned_served(ctx, net, scs, burst, res, res, kk, server=srv)
    plain_b = D.run_plain_svgf_loop(ctx, scs, burst, res, res)
    learned_b = D.run_learned_served(ctx, net, scs, burst, res, res, k, server=srv)
    learned_b2 = D.run_learned_served(ctx, net, scs, burst, res, res, k2, server=srv) if k2 != k else None
    rate = 0.7 * plain_b["req_per_s"]
    _, pois = D.sequence_requests(ctx, range(200, 208), res, res, frames, rate, seed=1, scenes_in=scs)
    plain_p = D.run_plain_svgf_loop(ctx, scs, pois, res, res)
    learned_p = D.run_learned_served(ctx, net, scs, pois, res, res, k, server=srv)
    srv.close()
    for sc in scs:
        sc.close()
    px = train_steps * 8 * 128 * 128
    net.close()
    return {"workload": f"Cornell variants at {res}x{res}: train seeds 100-163 (1 view each, 1-16 spp, 4096-spp refs); "
                        f"test: {frames}-frame orbit sequences of seeds 200-207, 4096-spp refs per frame",
            "dataset_s": round(t1 - t0, 2), "train_s": round(t2 - t1, 2), "eval_s": round(t3 - t2, 2),
            "train_steps": train_steps,
            "train_mpix_per_s": round(px / (e0.elapsed_time(e1) * 1e-3) / 1e6, 1),
            "loss_first": round(float(sum(losses[:20]) / 20), 5), "loss_last": round(float(sum(losses[-50:]) / 50), 5),
            "relmse": {k2: (round(v, 6) if not isinstance(v, dict) else {a: round(b, 6) for a, b in v.items()})
                       for k2, v in tab.items()},
            "kpcn_spp_matching_svgf64": k,
            "serving": {"resolution": [res, res], "learned_spp": k, "plain_spp": 64,
                        "burst": {"plain_svgf": plain_b, "learned_kpcn": learned_b,
                                  "req_per_s_ratio": round(learned_b["req_per_s"] / plain_b["req_per_s"], 2),
                                  f"learned_kpcn_at_{k2}spp": learned_b2,
                                  f"req_per_s_ratio_at_{k2}spp": (round(learned_b2["req_per_s"] / plain_b["req_per_s"], 2)
                                                                if learned_b2 else None)},
                        "poisson": {"rate_per_s": round(rate, 1), "plain_svgf": plain_p, "learned_kpcn": learned_p}}}


def bench_config(world):
    """The workload description both arms print (the same dict, so the two
    lines name one configuration)."""
    return {"workload": "icosphere field (64 x level-5 icospheres, 1,310,720 tris); per GPU and step "
                        "16M closest-hit rays + 16M shadow queries (1:1 extend:shadow)",
            "l2": "inputs 1.28 GB per step > 126 MB L2 (no flush needed)",
            "parallelism": f"replicas x{world}"}


def run_reference(args, rank, world):
    """--impl reference: the reference's own CPU implementation of the path
    (rank 0 only), on the same scene, metric and unit."""
    if rank != 0:
        return
    import oracle
    from cudaraytracer_b200 import scenes

    if not oracle.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libcrtref.so not built (needs the reference tree)"}))
        return
    threads = os.cpu_count() or 1
    tris = scenes.icosphere_field(with_env=False).triangles()
    # the same 1:1 extend:shadow mix as the GPU arm, on the first rays and
    # queries of the GPU arm's rank-0 batch
    n_ext = n_sh = 2 << 20
    rays = scenes.random_rays(tris, N_RAYS, seed=5)[:n_ext]
    q = scenes.random_shadow_queries(tris, N_RAYS, seed=1005)[:n_sh]
    ref = oracle.RefScene(tris)
    for _ in range(args.warmup):
        ref.trace_closest(rays[: 1 << 18], threads)
        ref.visible(q[: 1 << 16], threads)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        ref.trace_closest(rays, threads)
        ref.visible(q, threads)
        times.append(time.perf_counter() - t0)
    ref.close()
    dt = sum(times)
    value = args.steps * (n_ext + n_sh) / dt / 1e6
    sample = (f"{n_ext} extend rays + {n_sh} shadow queries per step: the first rays and queries of the "
              f"16M+16M batch, same 1:1 mix")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": round(value, 3), "unit": "Mrays/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1e3 * dt / args.steps, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": bench_config(world), "threads": threads,
        "cpu_baseline": {"value": round(value, 3), "unit": "Mrays/s", "cores": threads, "kind": "reference",
                         "sample": sample},
        "e2e": {"value": round(value, 3), "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


def main():
    global N_RAYS
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="crt", choices=["crt", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-ref-cuda", action="store_true", help="skip timing the reference's own CUDA traversal")
    ap.add_argument("--no-cornell", action="store_true", help="skip the Cornell-box 1M+1M traversal leg")
    ap.add_argument("--train-steps", type=int, default=6000, help="Adam steps of the denoise leg's KPCN training")
    ap.add_argument("--no-render", action="store_true", help="skip the full-frame render leg")
    ap.add_argument("--no-svgf", action="store_true", help="skip the 1080p SVGF leg")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched multi-view leg")
    ap.add_argument("--no-serve", action="store_true", help="skip the multi-scene serving leg")
    ap.add_argument("--no-denoise", action="store_true", help="skip the learned-denoiser leg")
    ap.add_argument("--only", choices=["conv", "kpcn", "svgf", "render", "cornell", "serve", "denoise"], default=None,
                    help="run one leg alone: conv (tensor-core convolutions at 1080p), kpcn (the denoiser's "
                         "layers at 1080p), svgf (1080p SVGF), render (1080p render), cornell (Cornell-box "
                         "traversal), serve (serving), denoise (learned denoiser vs SVGF)")
    ap.add_argument("--rays", type=int, default=N_RAYS, help="rays (and shadow queries) per step per GPU")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    rank, local_rank, world = dist_env()
    N_RAYS = args.rays

    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if args.only is not None:
        import torch

        from cudaraytracer_b200 import Context

        torch.cuda.set_device(local_rank)
        ctx = Context(local_rank)
        stream = torch.cuda.Stream()
        torch.cuda.set_stream(stream)
        legs = {"conv": lambda: conv_leg(ctx, reps=args.steps), "kpcn": lambda: kpcn_layers_leg(ctx),
                "svgf": lambda: svgf_leg(ctx, stream, with_reference=not args.no_ref_cuda),
                "render": lambda: render_leg(ctx, max(2, min(args.steps, 8)), stream,
                                             with_reference=not args.no_ref_cuda),
                "cornell": lambda: cornell_trace_leg(ctx, stream, with_reference=not args.no_ref_cuda),
                "serve": lambda: serve_leg(ctx), "denoise": lambda: denoise_leg(ctx, args.train_steps)}
        print(json.dumps({args.only: legs[args.only]()}))
        ctx.close()
        return

    import torch
    import torch.distributed as dist

    torch.cuda.set_device(local_rank)
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    from cudaraytracer_b200 import Context, Scene, scenes

    tris = scenes.icosphere_field(with_env=False).triangles()
    rays_np = scenes.random_rays(tris, N_RAYS, seed=5 + rank)
    q_np = scenes.random_shadow_queries(tris, N_RAYS, seed=1005 + rank)
    ctx = Context(local_rank)
    scene = Scene.from_triangles(ctx, tris)
    info = scene.info()
    dev = torch.device("cuda", local_rank)
    rays = torch.from_numpy(rays_np).to(dev)
    qs = torch.from_numpy(q_np).to(dev)
    hits = torch.empty((N_RAYS, 4), dtype=torch.float32, device=dev)
    occ = torch.empty((N_RAYS,), dtype=torch.uint8, device=dev)
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)

    def step():
        scene.trace_closest(rays, hits)
        scene.trace_shadow(qs, occ)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    sampler = ClockSampler(range(world) if world > 1 else [local_rank]) if rank == 0 else None
    if sampler:
        sampler.start()
        time.sleep(0.3)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True),
           torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    for k in range(args.steps):
        ev[k][0].record(stream)
        scene.trace_closest(rays, hits)
        ev[k][1].record(stream)
        scene.trace_shadow(qs, occ)
        ev[k][2].record(stream)
    torch.cuda.synchronize()
    ext_ms = sum(e[0].elapsed_time(e[1]) for e in ev)
    sh_ms = sum(e[1].elapsed_time(e[2]) for e in ev)
    total_ms = ev[0][0].elapsed_time(ev[-1][2])
    if world > 1:
        t = torch.tensor([total_ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
        dist.barrier()
    clocks = sampler.stop() if sampler else None
    ref_cuda = None
    if rank == 0 and not args.no_ref_cuda:
        ref_cuda = reference_cuda(tris, rays, qs, hits, occ, max(1, min(args.steps, 3)), stream)
    cornell = None
    if rank == 0 and not args.no_cornell:
        cornell = cornell_trace_leg(ctx, stream, with_reference=not args.no_ref_cuda)
    render = None
    if rank == 0 and not args.no_render:
        render = render_leg(ctx, max(2, min(args.steps, 8)), stream, with_reference=not args.no_ref_cuda)
    svgf = None
    if rank == 0 and not args.no_svgf:
        svgf = svgf_leg(ctx, stream, with_reference=not args.no_ref_cuda)
    batch = None
    if rank == 0 and not args.no_batch:
        batch = batch_leg(ctx, stream)
    serve = None
    if rank == 0 and not args.no_serve:
        serve = serve_leg(ctx)
    denoise = None
    if rank == 0 and not args.no_denoise:
        denoise = denoise_leg(ctx, args.train_steps)
        denoise["conv"] = conv_leg(ctx)
        denoise["kpcn_1080p"] = kpcn_layers_leg(ctx)

    # e2e through the host-buffer API: pinned host inputs, results back.
    pin_r = torch.from_numpy(rays_np).pin_memory()
    pin_q = torch.from_numpy(q_np).pin_memory()
    pin_h = torch.empty((N_RAYS, 4), dtype=torch.float32).pin_memory()
    pin_o = torch.empty((N_RAYS,), dtype=torch.uint8).pin_memory()
    rn, qn, hn, on = pin_r.numpy(), pin_q.numpy(), pin_h.numpy(), pin_o.numpy()
    e2e_steps = 0 if args.no_e2e else max(2, min(args.steps, 5))
    e2e_s = 1.0
    if e2e_steps:
        scene.trace_closest(rn, hn)
        scene.trace_shadow(qn, on)
        if world > 1:
            dist.barrier()
        t0 = time.perf_counter()
        for _ in range(e2e_steps):
            scene.trace_closest(rn, hn)
            scene.trace_shadow(qn, on)
        e2e_s = time.perf_counter() - t0
    if world > 1:
        t = torch.tensor([e2e_s], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e_val = world * e2e_steps * 2 * N_RAYS / e2e_s / 1e6

    if rank == 0:
        value = world * args.steps * 2 * N_RAYS / (total_ms * 1e-3) / 1e6
        peak, peak_kind = measured_peaks()
        ext_launch_ms = ext_ms / args.steps
        sh_launch_ms = sh_ms / args.steps
        kern = {}
        for name, ms, per in (("extend", ext_launch_ms, EXTEND_BYTES), ("shadow", sh_launch_ms, SHADOW_BYTES)):
            ach = per * N_RAYS / (ms * 1e-3) / 1e9
            tr = profiled_traffic(name)
            kern[name] = {"ms_per_launch": round(ms, 4), "mrays_s": round(N_RAYS / (ms * 1e-3) / 1e6, 1),
                          "achieved": round(ach, 1), "frac": round(ach / peak, 4),
                          "algorithmic_bytes_per_launch": per * N_RAYS,
                          "traffic": None if tr is None else round(tr * N_RAYS / (16 << 20))}
        dom = "shadow" if sh_launch_ms > ext_launch_ms else "extend"
        cpu = None
        if not args.no_cpu_baseline:
            threads = os.cpu_count() or 1
            n_ext = n_sh = 2 << 20  # the step's 1:1 extend:shadow mix
            r = reference_cpu(tris, rays_np[:n_ext], q_np[:n_sh], threads)
            if r is not None:
                cpu = {"value": round(r[0], 3), "unit": "Mrays/s", "cores": threads, "kind": "reference",
                       "sample": f"{n_ext} extend rays + {n_sh} shadow queries of the same batch, "
                                 f"{r[1]:.1f} s of CPU work on {threads} threads"}
        out = {
            "metric": METRIC, "value": round(value, 2), "unit": "Mrays/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(total_ms / args.steps, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": bench_config(world),
            "bvh": {"nodes": info["num_bvh_nodes"], "depth": info["bvh_depth"],
                    "build_ms": round(info["build_ms"], 2)},
            "kernels": kern,
            "roofline": {"bound": "hbm", "achieved": kern[dom]["achieved"], "peak": peak, "unit": "GB/s",
                         "frac": kern[dom]["frac"], "traffic": kern[dom]["traffic"],
                         "peak_kind": peak_kind,
                         "kernel": "k_trace_shadow" if dom == "shadow" else "k_trace_closest",
                         "algorithmic_bytes_per_launch": kern[dom]["algorithmic_bytes_per_launch"],
                         "bytes_per_unit": SHADOW_BYTES if dom == "shadow" else EXTEND_BYTES},
            "cpu_baseline": cpu,
            "e2e": {"value": round(e2e_val, 2), "unit": "Mrays/s",
                    "h2d_bytes_per_step": N_RAYS * (32 + 48), "d2h_bytes_per_step": N_RAYS * (16 + 1)},
            "reference_cuda": ref_cuda,
            "cornell_trace": cornell,
            "render": render,
            "svgf": svgf,
            "batch": batch,
            "serve": serve,
            "denoise": denoise,
            "gpu_launches": 2 * args.steps,
            "clocks": clocks,
        }
        print(json.dumps(out))
    del scene
    ctx.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
