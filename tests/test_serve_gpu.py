"""Multi-scene render server (crt_server_*): continuous batching of requests of
differing scene, resolution, spp and depth into shared wavefronts, HBM-budget
admission, and the result of each request alone vs in the mix."""
import numpy as np
import pytest

from cudaraytracer_b200 import CrtError, Scene, scenes
from cudaraytracer_b200.serve import DONE, QUEUED, RenderRequest, Server, poisson_requests, run_served

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def resident(tmp_path_factory, crt_ctx):
    d = str(tmp_path_factory.mktemp("serve"))
    cb = Scene.load(crt_ctx, scenes.cornell_box(width=48, height=48, max_bounces=6).write(d, "cb"))
    ico = Scene.load(crt_ctx, scenes.icosphere_field(n_spheres=8, level=2, width=40, height=32, max_bounces=8,
                                                     env_size=(128, 64), sun_peak=40.0, sun_sigma=0.1).write(d, "ico"))
    yield [cb, ico]
    cb.close()
    ico.close()


def orbit(sc, theta, phi, scale=1.0):
    c = sc.camera()
    return {"target": c["target"], "distance": c["distance"] * scale, "theta_deg": theta, "phi_deg": phi,
            "fovy_deg": c["fovy_deg"]}


def mix(resident):
    cb, ico = resident
    return [
        RenderRequest(0, 48, 48, 6, orbit(cb, 80, 10), seed=11),
        RenderRequest(1, 40, 32, 9, orbit(ico, 70, 200, 1.1), seed=12),
        RenderRequest(0, 33, 21, 3, orbit(cb, 100, 350, 0.9), seed=13, max_bounces=3),
        RenderRequest(1, 64, 48, 2, orbit(ico, 120, 30), seed=14, max_bounces=12, rr=0.6),
        RenderRequest(0, 16, 16, 0, orbit(cb, 90, 0), seed=15),
        RenderRequest(1, 17, 19, 5, orbit(ico, 45, 90, 0.8), seed=16, rr_start_bounce=2),
    ]


def render_alone(sc, r):
    import torch

    rp = sc.render_params()
    sc.set_render_params(width=r.width, height=r.height, seed=r.seed,
                         max_bounces=rp["max_bounces"] if r.max_bounces is None else r.max_bounces,
                         rr=rp["rr"] if r.rr is None else r.rr,
                         rr_start_bounce=0 if r.rr_start_bounce is None else r.rr_start_bounce)
    c = r.camera
    sc.set_camera_orbit(c["target"], c["distance"], c["theta_deg"], c["phi_deg"], c["fovy_deg"])
    d = torch.zeros((r.height, r.width, 4), device="cuda")
    i = torch.zeros_like(d)
    sc.render_device(d, i, r.spp)
    torch.cuda.synchronize()
    sc.set_render_params(**{k: rp[k] for k in ("width", "height", "seed", "max_bounces", "rr", "rr_start_bounce")})
    return d.cpu().numpy(), i.cpu().numpy()


@pytest.mark.parametrize("schedule", [Server.SHORTEST_FIRST, Server.ADMISSION_ORDER])
def test_each_request_same_alone_and_in_the_mix(crt_ctx, resident, schedule):
    reqs = mix(resident)
    # small wavefronts so requests straddle passes and passes mix requests
    srv = Server(crt_ctx, paths_per_pass=3000, passes_in_flight=3, schedule=schedule)
    for sc in resident:
        srv.add_scene(sc)
    ids = [srv.submit(r) for r in reqs]
    srv.drain()
    assert srv.stats()["passes"] > 4
    mixed = [srv.result(rid, r.width, r.height) for rid, r in zip(ids, reqs)]
    for rid in ids:
        srv.release(rid)
    # the same requests one at a time through the server
    alone = []
    for r in reqs:
        rid = srv.submit(r)
        srv.drain()
        alone.append(srv.result(rid, r.width, r.height))
        srv.release(rid)
    srv.close()
    for r, (md, mi), (ad, ai) in zip(reqs, mixed, alone):
        pd, pi = render_alone(resident[r.scene], r)
        for got in ((md, mi), (ad, ai)):
            np.testing.assert_allclose(got[0], pd, rtol=2e-5, atol=2e-6)
            np.testing.assert_allclose(got[1], pi, rtol=2e-5, atol=2e-6)
        if r.spp == 0:
            assert not md.any() and not mi.any()
        else:
            assert (md + mi)[..., :3].sum() > 0


def test_budget_admission_and_queueing(crt_ctx, resident):
    cb = resident[0]
    st0 = None
    srv0 = Server(crt_ctx, paths_per_pass=4096)
    srv0.add_scene(cb)
    st0 = srv0.stats()
    srv0.close()
    per_req = 64 * 64 * 32
    budget = st0["bytes_scenes"] + st0["bytes_wavefront"] + per_req + per_req // 2  # one request at a time
    srv = Server(crt_ctx, hbm_budget_bytes=budget, paths_per_pass=4096)
    srv.add_scene(cb)
    reqs = [RenderRequest(0, 64, 64, 2, orbit(cb, 90, 30 * k), seed=k) for k in range(3)]
    ids = [srv.submit(r) for r in reqs]
    srv.step()
    st = srv.stats()
    assert st["running"] == 1 and st["queued"] == 2
    assert st["bytes_requests"] == per_req
    assert srv.poll(ids[2]) == QUEUED
    with pytest.raises(CrtError):
        srv.result(ids[2], 64, 64)
    done = 0
    while done < 3:
        srv.step(wait=True)
        for rid in list(ids):
            if srv.poll(rid) == DONE:
                srv.release(rid)
                ids.remove(rid)
                done += 1
        assert srv.stats()["bytes_requests"] <= per_req
    # a request that can never fit is refused at submit
    with pytest.raises(CrtError, match="CAPACITY"):
        srv.submit(RenderRequest(0, 512, 512, 1, orbit(cb, 90, 0)))
    # a queued request can be released before it runs
    a = srv.submit(reqs[0])
    b = srv.submit(reqs[1])
    srv.step()
    assert srv.poll(b) == QUEUED
    srv.release(b)
    srv.drain()
    assert srv.poll(a) == DONE
    srv.release(a)
    srv.close()


def test_open_loop_driver_reports_latency(crt_ctx, resident):
    cams = [orbit(sc, 90, 0) for sc in resident]
    reqs = poisson_requests(24, 400.0, cams, [(32, 32), (48, 40)], [1, 4], seed=3, max_bounces=5)
    srv = Server(crt_ctx, paths_per_pass=1 << 14)
    for sc in resident:
        srv.add_scene(sc)
    out, res = run_served(srv, reqs, keep_results=True)
    srv.close()
    assert out["requests"] == 24 and out["p99_ms"] >= out["p50_ms"] > 0
    assert len(res) == 24
    j = 5
    pd, pi = render_alone(resident[reqs[j].scene], reqs[j])
    np.testing.assert_allclose(res[j][0], pd, rtol=2e-5, atol=2e-6)
    np.testing.assert_allclose(res[j][1], pi, rtol=2e-5, atol=2e-6)


@pytest.mark.parametrize("schedule", [Server.SHORTEST_FIRST, Server.ADMISSION_ORDER])
def test_shortest_first_finishes_a_small_request_behind_a_large_one(crt_ctx, resident, schedule):
    """A large request (1M paths) admitted first and a small one (2K paths)
    right behind it: filling passes shortest-first finishes the small one
    in the first pass while the large one still runs; in admission order
    the small one waits for the large one's last pass."""
    cb = resident[0]
    srv = Server(crt_ctx, paths_per_pass=1 << 15, passes_in_flight=1, schedule=schedule)
    srv.add_scene(cb)
    big = srv.submit(RenderRequest(0, 128, 128, 64, orbit(cb, 90, 0), seed=21))
    small = srv.submit(RenderRequest(0, 32, 32, 2, orbit(cb, 90, 10), seed=22))
    order = []
    while len(order) < 2:
        srv.step(wait=True)
        for rid in (big, small):
            if rid not in order and srv.poll(rid) == DONE:
                order.append(rid)
    if schedule == Server.SHORTEST_FIRST:
        assert order == [small, big]
        assert srv.stats()["passes"] >= 32  # 1M paths of the large request in passes of 32K
    else:
        assert order == [big, small]
    for rid in (big, small):
        srv.release(rid)
    srv.close()
