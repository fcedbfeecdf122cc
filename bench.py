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
TRAFFIC_PER_16M = {"extend": 1698088448, "shadow": 5904843776}


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
    headless CUDA build) on the same device batch and checks its hit records
    against ours. Returns a dict or None when that build is absent."""
    import torch

    import oracle

    if not oracle.ref_cuda_available():
        return None
    ref = oracle.RefCudaScene(tris)
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
           "build": "reference sources, nvcc -O3 -rdc -arch sm_100a, BVH built on the host"}
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
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for k in range(steps):
        sc.render_device(d, i, step_spp, first_sample=step_spp * (k + 1), stream=stream.cuda_stream)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    spp_total = steps * step_spp
    out = {"scene": "icosphere field 1920x1080, depth 16, env 2048x1024", "spp_per_step": step_spp,
           "spp_per_s": round(spp_total / (ms * 1e-3), 2),
           "msamples_per_s": round(W * H * spp_total / (ms * 1e-3) / 1e6, 2),
           "ms_per_spp": round(ms / spp_total, 3)}
    t0 = time.perf_counter()
    sc.render(step_spp)
    out["e2e_ms_per_spp_host_api"] = round((time.perf_counter() - t0) * 1e3 / step_spp, 3)
    if with_reference:
        import oracle

        if oracle.ref_render_available():
            ref = oracle.RefRenderer(path)
            ref.render(1, with_sumsq=False)
            frames = 2
            _, _, _, rms = ref.render(frames, with_sumsq=False)
            out["reference_cuda"] = {"msamples_per_s": round(W * H * frames / (rms * 1e-3) / 1e6, 3),
                                     "ms_per_spp": round(rms / frames, 2),
                                     "build": "reference renderer.cuh + Scene, nvcc -O3 -rdc sm_100a, headless"}
    sc.close()
    return out


def batch_leg(ctx, stream):
    """Batched persistent wavefront (the multi-view batch workload): 64 orbit views of
    the Cornell box (radius 3, elevation U[-30, 30] deg, seeded), 512x512,
    16 spp, depth 12, all views in shared wavefronts with a CUDA graph per
    pass and an autotuned wavefront size and stage block size, against 64 sequential single-view
    renders of the same cameras."""
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
            "autotune_ms": tune.get("timings_ms"), "autotune_block_ms": tune.get("block_timings_ms")}


def serve_leg(ctx, quick=False):
    """Serving (the multi-scene request workload) on a bounded sample. 8 resident scenes of
    the icosphere-field generator with {1, 4, 8, 16, 32, 64, 128, 256}
    level-5 spheres (20k to 5.2M triangles, 2048x1024 env each). Requests
    draw resolution from {256^2, 512^2, 1280x720, 1920x1080}, spp from
    {1, 4, 16, 64} and a random orbit pose. Poisson arrivals at 5, 20 and
    80 per second (40, 120 and 320 requests instead of 2,000 per rate) and a
    saturated burst (160 requests at t=0), each served by crt_server
    (continuous batching, HBM budget 150 GiB, 8M-path wavefronts) and by the
    one-request-at-a-time loop (Scene.render_device per request) over the
    same requests. Latency = completion - arrival (host clock)."""
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
    for sc in scs:
        srv.add_scene(sc)
    warm = poisson_requests(8, 0.0, cams, res, [1, 4], seed=99)
    run_served(srv, warm)
    run_one_at_a_time(scs, warm)
    plan = [(5.0, 40), (20.0, 120), (80.0, 320)] if not quick else [(80.0, 48)]
    out = {"workload": "8 resident icosphere-field scenes (1..256 level-5 spheres, 20k-5.2M tris); requests of "
                       "{256^2, 512^2, 1280x720, 1920x1080} x {1, 4, 16, 64} spp, random poses",
           "scenes_tris": [int(sc.info()["num_triangles"]) for sc in scs], "scene_build_s": round(load_s, 2),
           "hbm": {k: v for k, v in srv.stats().items() if k.startswith("bytes")}, "rates": {}}
    for rate, n in plan:
        reqs = poisson_requests(n, rate, cams, res, spps, seed=int(rate))
        served = run_served(srv, reqs)
        plain = run_one_at_a_time(scs, reqs)
        out["rates"][f"{rate:g}/s"] = {"served": served, "one_at_a_time": plain}
    burst = poisson_requests(160 if not quick else 32, 0.0, cams, res, spps, seed=7)
    served = run_served(srv, burst)
    plain = run_one_at_a_time(scs, burst)
    out["saturated"] = {"served": served, "one_at_a_time": plain,
                        "req_per_s_ratio": round(served["req_per_s"] / plain["req_per_s"], 3)}
    out["server_stats"] = {k: v for k, v in srv.stats().items() if k in ("passes", "paths")}
    srv.close()
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


def denoise_leg(ctx):
    """Learned denoiser (the learned-denoiser workload on a bounded sample): the KPCN is
    trained on the GPU on 64 views of seeded Cornell variants (scene seeds
    100-131, 256x256, 1-16 spp inputs, 1024-spp references) for 1500 Adam
    steps of 8 random 128x128 crops, then evaluated on unseen scenes (seeds
    200-207, one 256x256 view each) by relMSE against 4096-spp references:
    raw and KPCN at 1-32 spp, SVGF at 64 spp. The smallest spp at which the
    KPCN matches 64 spp + SVGF then sets the learned pipeline of the
    requests/s comparison: 32 requests at 512x512 served through the
    multi-scene server at that spp + KPCN, against the one-request-at-a-time
    loop of 64 spp + SVGF."""
    import torch

    from cudaraytracer_b200 import denoise as D
    from cudaraytracer_b200.kpcn import Kpcn

    t0 = time.perf_counter()
    data = D.build_dataset(ctx, range(100, 132), 2, 256, 256, [1, 2, 4, 8, 16], 1024, seed=0)
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    net = Kpcn(ctx, seed=0)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    losses = D.train(net, data, 1500, batch=8, crop=128, lr=1e-3)
    e1.record()
    torch.cuda.synchronize()
    t2 = time.perf_counter()
    spp_list = [1, 2, 4, 8, 16, 32]
    tab = D.evaluate(ctx, net, range(200, 208), 256, 256, spp_list)
    k = D.matching_spp(tab, spp_list)
    thr = D.pipeline_throughput(ctx, net, range(200, 208), 512, 512, 32, k or 32)
    # training throughput: pixels x (forward + backward) per second
    px = 1500 * 8 * 128 * 128
    net.close()
    return {"workload": "Cornell variants: train seeds 100-131 (64 views, 256^2, 1-16 spp, 1024-spp refs), "
                        "test seeds 200-207 (256^2, 4096-spp refs)",
            "dataset_s": round(t1 - t0, 2), "train_s": round(t2 - t1, 2), "train_steps": 1500,
            "train_mpix_per_s": round(px / (e0.elapsed_time(e1) * 1e-3) / 1e6, 1),
            "loss_first": round(float(sum(losses[:20]) / 20), 5), "loss_last": round(float(sum(losses[-50:]) / 50), 5),
            "relmse": {k2: round(v, 6) for k2, v in tab.items()}, "kpcn_spp_matching_svgf64": k,
            "throughput": thr}


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
    ap.add_argument("--no-render", action="store_true", help="skip the full-frame render leg")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched multi-view leg")
    ap.add_argument("--no-serve", action="store_true", help="skip the multi-scene serving leg")
    ap.add_argument("--no-denoise", action="store_true", help="skip the learned-denoiser leg")
    ap.add_argument("--only", choices=["conv"], default=None,
                    help="run one micro-benchmark alone (conv: the tensor-core convolutions at 1080p)")
    ap.add_argument("--rays", type=int, default=N_RAYS, help="rays (and shadow queries) per step per GPU")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    rank, local_rank, world = dist_env()
    N_RAYS = args.rays

    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if args.only == "conv":
        import torch

        from cudaraytracer_b200 import Context

        torch.cuda.set_device(local_rank)
        ctx = Context(local_rank)
        print(json.dumps({"conv": conv_leg(ctx, reps=args.steps)}))
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
    batch = None
    if rank == 0 and not args.no_batch:
        batch = batch_leg(ctx, stream)
    serve = None
    if rank == 0 and not args.no_serve:
        serve = serve_leg(ctx)
    denoise = None
    if rank == 0 and not args.no_denoise:
        denoise = denoise_leg(ctx)
        denoise["conv"] = conv_leg(ctx)

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
