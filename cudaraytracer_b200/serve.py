"""Render serving over resident scenes: the crt_server C ABI (continuous
batching of requests into shared wavefronts under an HBM budget) and the
open-loop drivers that measure it against a one-request-at-a-time loop.

The reference has no serving layer: Renderer::RenderLoop renders one scene
for one viewer (Src/Core/renderer.cuh:1106-1307). A request here is one
render job (scene, resolution, spp, orbit camera, seed) whose result is the
float4 direct/indirect accumulators, rows bottom-up, as crt_render returns.
"""
from __future__ import annotations

import ctypes as C
import time
from dataclasses import dataclass, field

import numpy as np

from . import _lib

QUEUED, RUNNING, DONE = 0, 1, 2


@dataclass
class RenderRequest:
    """One render job. camera: orbit parameters (target, distance,
    theta_deg, phi_deg, fovy_deg); max_bounces / rr / rr_start_bounce of
    None take the scene's render parameters."""
    scene: int
    width: int
    height: int
    spp: int
    camera: dict
    seed: int = 1
    max_bounces: int | None = None
    rr: float | None = None
    rr_start_bounce: int | None = None
    arrival_s: float = 0.0
    tag: dict = field(default_factory=dict)


class Server:
    """A crt_server on a Context: add scenes, submit requests, step."""

    SHORTEST_FIRST, ADMISSION_ORDER = 0, 1

    def __init__(self, ctx, hbm_budget_bytes: int = 0, paths_per_pass: int = 0, max_requests: int = 0,
                 passes_in_flight: int = 0, schedule: int = 0):
        self.ctx = ctx
        cfg = _lib.ServerConfig(int(hbm_budget_bytes), int(paths_per_pass), int(max_requests), int(passes_in_flight),
                                int(schedule))
        h = C.c_void_p()
        _lib.call("crt_server_create", ctx._h, C.byref(cfg), C.byref(h))
        self._h = h
        self._scenes = []
        ctx._adopt(self)

    def close(self):
        if self._h:
            _lib.lib().crt_server_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add_scene(self, scene) -> int:
        """Makes a loaded Scene resident; returns its id. The Scene must
        stay open while the server lives."""
        sid = C.c_int32()
        _lib.call("crt_server_add_scene", self._h, scene._h, C.byref(sid))
        self._scenes.append(scene)
        return sid.value

    def submit(self, req: RenderRequest) -> int:
        sc = self._scenes[req.scene]
        rp = sc.render_params()
        r = _lib.Request()
        r.scene = req.scene
        r.width, r.height, r.spp = int(req.width), int(req.height), int(req.spp)
        r.max_bounces = int(rp["max_bounces"] if req.max_bounces is None else req.max_bounces)
        r.rr = float(rp["rr"] if req.rr is None else req.rr)
        r.rr_start_bounce = int(rp["rr_start_bounce"] if req.rr_start_bounce is None else req.rr_start_bounce)
        r.seed = int(req.seed)
        cam = req.camera
        for k in range(3):
            r.camera.target[k] = cam["target"][k]
        r.camera.distance = cam["distance"]
        r.camera.theta_deg, r.camera.phi_deg, r.camera.fovy_deg = cam["theta_deg"], cam["phi_deg"], cam["fovy_deg"]
        rid = C.c_int64()
        _lib.call("crt_server_submit", self._h, C.byref(r), C.byref(rid))
        return rid.value

    def step(self, wait: bool = False) -> int:
        n = C.c_int32()
        _lib.call("crt_server_step", self._h, 1 if wait else 0, C.byref(n))
        return n.value

    def poll(self, rid: int) -> int:
        s = C.c_int32()
        _lib.call("crt_server_poll", self._h, int(rid), C.byref(s))
        return s.value

    def result(self, rid: int, width: int, height: int):
        d = np.empty((height, width, 4), np.float32)
        i = np.empty_like(d)
        _lib.call("crt_server_result", self._h, int(rid), d.ctypes.data, i.ctypes.data)
        return d, i

    def result_device(self, rid: int):
        """(direct, indirect) device addresses, valid until release."""
        d, i = C.c_void_p(), C.c_void_p()
        _lib.call("crt_server_result_device", self._h, int(rid), C.byref(d), C.byref(i))
        return d.value, i.value

    def release(self, rid: int) -> None:
        _lib.call("crt_server_release", self._h, int(rid))

    def stats(self) -> dict:
        st = _lib.ServerStats()
        _lib.call("crt_server_get_stats", self._h, C.byref(st))
        return {k: getattr(st, k) for k, _ in st._fields_}

    def drain(self) -> None:
        """Steps until nothing is queued or running."""
        while True:
            s = self.stats()
            if s["queued"] == 0 and s["running"] == 0:
                return
            self.step(wait=True)


def poisson_requests(n: int, rate_per_s: float, scene_cameras: list, resolutions, spp_choices, seed: int = 0,
                     max_bounces: int | None = None):
    """n requests with exponential inter-arrival times at rate_per_s; each
    draws a scene, a resolution and an spp uniformly and a random orbit pose
    around that scene's default camera (theta U[30, 150] deg, phi U[0, 360)
    deg, distance x U[0.8, 1.2])."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for k in range(n):
        t += rng.exponential(1.0 / rate_per_s) if rate_per_s > 0 else 0.0
        s = int(rng.integers(len(scene_cameras)))
        base = scene_cameras[s]
        w, h = resolutions[int(rng.integers(len(resolutions)))]
        spp = int(spp_choices[int(rng.integers(len(spp_choices)))])
        cam = {"target": list(base["target"]), "distance": float(base["distance"]) * float(rng.uniform(0.8, 1.2)),
               "theta_deg": float(rng.uniform(30, 150)), "phi_deg": float(rng.uniform(0, 360)),
               "fovy_deg": float(base["fovy_deg"])}
        out.append(RenderRequest(scene=s, width=int(w), height=int(h), spp=spp, camera=cam, seed=1000 + k,
                                 max_bounces=max_bounces, arrival_s=t))
    return out


def _percentiles(lat):
    a = np.sort(np.asarray(lat))
    if a.size == 0:
        return {"p50_ms": None, "p99_ms": None, "mean_ms": None}
    return {"p50_ms": round(float(np.percentile(a, 50)) * 1e3, 2),
            "p99_ms": round(float(np.percentile(a, 99)) * 1e3, 2),
            "mean_ms": round(float(a.mean()) * 1e3, 2)}


def _by_class(requests, lat):
    """Latency percentiles per request class (resolution x spp)."""
    groups = {}
    for r, l in zip(requests, lat):
        groups.setdefault((r.width * r.height, f"{r.width}x{r.height}@{r.spp}spp"), []).append(l)
    out = {}
    for (_, name), ls in sorted(groups.items(), key=lambda kv: (kv[0][0], int(kv[0][1].split("@")[1][:-3]))):
        out[name] = {"n": len(ls), **_percentiles(ls)}
    return out


def run_served(server: Server, requests, keep_results: bool = False, idle_sleep_s: float = 2e-4):
    """Open-loop run: each request is submitted at its arrival time (wall
    clock from the start), the server is stepped continuously, and a request's
    latency is its completion time minus its arrival time. Returns a summary
    dict (and the results by request index when keep_results)."""
    n = len(requests)
    ids = {}
    done_t = {}
    results = {}
    k = 0
    t0 = time.perf_counter()
    pending = set()
    while len(done_t) < n:
        now = time.perf_counter() - t0
        while k < n and requests[k].arrival_s <= now:
            ids[server.submit(requests[k])] = k
            pending.add(k)
            k += 1
        nd = server.step(wait=k == n)  # block for a completion once nothing more arrives
        if nd:
            now = time.perf_counter() - t0
            for rid, j in list(ids.items()):
                if j in pending and server.poll(rid) == DONE:
                    done_t[j] = now
                    pending.discard(j)
                    if keep_results:
                        r = requests[j]
                        results[j] = server.result(rid, r.width, r.height)
                    server.release(rid)
                    del ids[rid]
        if not nd and k < n and not pending:
            time.sleep(min(idle_sleep_s, max(0.0, requests[k].arrival_s - (time.perf_counter() - t0))))
    wall = time.perf_counter() - t0
    lat = [done_t[j] - requests[j].arrival_s for j in range(n)]
    out = {"requests": n, "wall_s": round(wall, 3), "req_per_s": round(n / wall, 3), **_percentiles(lat),
           "samples": int(sum(r.width * r.height * r.spp for r in requests)), "by_class": _by_class(requests, lat)}
    return (out, results) if keep_results else out


def run_one_at_a_time(scenes, requests, keep_results: bool = False):
    """The plain loop: requests in arrival order, each rendered alone with
    Scene.render_device after its arrival and synchronised before the next
    starts; latency = completion - arrival."""
    import torch

    n = len(requests)
    lat = []
    results = {}
    t0 = time.perf_counter()
    for j, r in enumerate(requests):
        now = time.perf_counter() - t0
        if r.arrival_s > now:
            time.sleep(r.arrival_s - now)
        sc = scenes[r.scene]
        rp = sc.render_params()
        sc.set_render_params(width=r.width, height=r.height, seed=r.seed,
                             max_bounces=rp["max_bounces"] if r.max_bounces is None else r.max_bounces,
                             rr=rp["rr"] if r.rr is None else r.rr,
                             rr_start_bounce=rp["rr_start_bounce"] if r.rr_start_bounce is None else r.rr_start_bounce)
        c = r.camera
        sc.set_camera_orbit(c["target"], c["distance"], c["theta_deg"], c["phi_deg"], c["fovy_deg"])
        dev = torch.device("cuda", sc.ctx.device)
        d = torch.zeros((r.height, r.width, 4), device=dev)
        i = torch.zeros_like(d)
        sc.render_device(d, i, r.spp)
        torch.cuda.synchronize(dev)
        lat.append(time.perf_counter() - t0 - r.arrival_s)
        if keep_results:
            results[j] = (d.cpu().numpy(), i.cpu().numpy())
    wall = time.perf_counter() - t0
    out = {"requests": n, "wall_s": round(wall, 3), "req_per_s": round(n / wall, 3), **_percentiles(lat),
           "samples": int(sum(r.width * r.height * r.spp for r in requests)), "by_class": _by_class(requests, lat)}
    return (out, results) if keep_results else out


def scene_hbm_bytes_estimate(num_tris: int) -> int:
    """Device bytes a loaded scene holds per triangle count (BVH nodes at
    most 2n x 64 B, leaf-order triangles 48 B, vertices 36 B, attributes
    64 B, slot map 4 B, 8-wide nodes and links about 24 B), for sizing
    budgets before loading."""
    return int(num_tris * (128 + 48 + 36 + 64 + 4 + 24))
