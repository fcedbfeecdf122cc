"""Autotuner for the batched renderer: picks the wavefront size (paths per
pass, the queue capacity), then the thread-block size of the
extend/shade/shadow stage kernels, then their BVH traversal (stack depth
and placement: a 64-entry stack in local memory or the top 8 entries in
shared memory; node width: 64 B float child boxes or 32 B 16-bit quantised
ones) for Scene.render_views, by timing a short probe render of each
candidate with CUDA events, and caches the choice in a JSON file keyed by
GPU name, scene triangle count (power-of-two bucket), image size and view
count. The branching factor stays binary (the 4- and 8-wide collapses
measured slower). No counterpart in the reference (its wavefront is one
frame of one view)."""
from __future__ import annotations

import json
import math
import os

DEFAULT_CANDIDATES = (1 << 20, 2 << 20, 4 << 20, 8 << 20, 16 << 20)
BLOCK_CANDIDATES = (64, 128, 256)
# crt_render_params.stage_traversal: CRT_STAGE_LOCAL, _SHARED, _LOCAL_QUANT,
# _SHARED_QUANT, _WARP, _REFILL (include/crt.h)
TRAVERSAL_CANDIDATES = {1: "local", 2: "shared", 3: "local-quant", 4: "shared-quant", 5: "warp", 6: "refill"}


def cache_key(scene, n_views: int) -> str:
    import torch

    info = scene.info()
    rp = scene.render_params()
    tris = max(1, int(info["num_triangles"]))
    return (f"{torch.cuda.get_device_name(scene.ctx.device)}|tris2^{int(math.log2(tris))}|"
            f"{rp['width']}x{rp['height']}x{n_views}|bounces{rp['max_bounces']}")


def autotune_paths_per_pass(scene, cameras, probe_spp: int = 1, candidates=DEFAULT_CANDIDATES,
                            cache_path: str | None = None, blocks=BLOCK_CANDIDATES,
                            traversals=tuple(TRAVERSAL_CANDIDATES)) -> dict:
    """Times render_views(cameras, probe_spp) for each candidate wavefront
    size (at the scene's current stage block size and traversal), then for
    each stage block size at the fastest wavefront size, then for each stage
    traversal at both; sets the winners on the scene and returns
    {"paths_per_pass", "stage_block", "stage_traversal", "timings_ms",
    "block_timings_ms", "traversal_timings_ms", "cached"}."""
    import torch

    key = cache_key(scene, len(cameras))
    if cache_path and os.path.exists(cache_path):
        with open(cache_path) as f:
            cache = json.load(f)
        if key in cache:
            scene.set_render_params(paths_per_pass=int(cache[key]["paths_per_pass"]),
                                    stage_block=int(cache[key].get("stage_block", 0)),
                                    stage_traversal=int(cache[key].get("stage_traversal", 0)))
            return {**cache[key], "cached": True}
    rp = scene.render_params()
    shape = (len(cameras), rp["height"], rp["width"], 4)
    d = torch.zeros(shape, device="cuda")
    i = torch.zeros(shape, device="cuda")
    total = len(cameras) * rp["height"] * rp["width"] * probe_spp

    def probe_ms() -> float:
        scene.render_views(cameras, d, i, probe_spp)  # warm-up (allocation, capture)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        scene.render_views(cameras, d, i, probe_spp, first_sample=probe_spp)
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)

    timings = {}
    for c in candidates:
        c = int(min(c, max(total, 1)))
        if c in timings:
            continue
        scene.set_render_params(paths_per_pass=c)
        timings[c] = probe_ms()
    best = min(timings, key=timings.get)
    scene.set_render_params(paths_per_pass=best)
    block_timings = {}
    for b in blocks:
        scene.set_render_params(stage_block=int(b))
        block_timings[int(b)] = probe_ms()
    best_block = min(block_timings, key=block_timings.get)
    scene.set_render_params(stage_block=best_block)
    trav_timings = {}
    for t in traversals:
        scene.set_render_params(stage_traversal=int(t))
        trav_timings[int(t)] = probe_ms()
    best_trav = min(trav_timings, key=trav_timings.get) if trav_timings else 0
    scene.set_render_params(stage_traversal=best_trav)
    entry = {"paths_per_pass": best, "stage_block": best_block, "stage_traversal": best_trav,
             "timings_ms": {str(k): round(v, 3) for k, v in timings.items()},
             "block_timings_ms": {str(k): round(v, 3) for k, v in block_timings.items()},
             "traversal_timings_ms": {TRAVERSAL_CANDIDATES.get(k, str(k)): round(v, 3)
                                      for k, v in trav_timings.items()}}
    if cache_path:
        cache = {}
        if os.path.exists(cache_path):
            with open(cache_path) as f:
                cache = json.load(f)
        cache[key] = entry
        os.makedirs(os.path.dirname(os.path.abspath(cache_path)), exist_ok=True)
        with open(cache_path, "w") as f:
            json.dump(cache, f, indent=1)
    return {**entry, "cached": False}


def orbit_views(scene, n_views: int, radius: float = 3.0, max_elev_deg: float = 30.0, seed: int = 1):
    """n_views orbit cameras around the scene's target: azimuths evenly
    spaced, elevations uniform in [-max_elev, max_elev] (seeded), distance
    `radius`, the scene camera's fov."""
    import numpy as np

    c = scene.camera()
    rng = np.random.default_rng(seed)
    elev = rng.uniform(-max_elev_deg, max_elev_deg, n_views)
    return [{"target": c["target"], "distance": radius, "theta_deg": float(90.0 - elev[v]),
             "phi_deg": float(360.0 * v / n_views), "fovy_deg": c["fovy_deg"]} for v in range(n_views)]
