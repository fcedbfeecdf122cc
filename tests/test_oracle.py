"""CPU tests of the oracle: the restatement (oracle/crt_oracle.c) against the
reference's own results (golden fixtures generated by running the reference
harness, plus live comparisons where the reference tree is present), against
the FP64 intersector, and on the edge cases of the acceptance predicate."""
import hashlib

import numpy as np
import pytest

import oracle
from cudaraytracer_b200 import scenes


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def prims(h):
    return np.ascontiguousarray(h[:, 1]).view(np.int32)


def test_generators_reproduce_fixture_inputs(golden, cornell_tris, ico_tris):
    assert sha(cornell_tris) == golden["c1_tris_sha"]
    assert sha(ico_tris) == golden["c2_tris_sha"]
    assert cornell_tris.shape == (36, 9)
    assert ico_tris.shape == (64 * 20480, 9)
    assert sha(scenes.random_rays(cornell_tris, 1 << 20, seed=1)) == golden["c1_rays_sha"]
    assert sha(scenes.random_shadow_queries(cornell_tris, 1 << 20, seed=2)) == golden["c1_queries_sha"]


def test_oracle_matches_reference_cornell_1m(golden, cornell_tris):
    rays = scenes.random_rays(cornell_tris, 1 << 20, seed=1)
    h = oracle.trace_brute(cornell_tris, rays)
    np.testing.assert_array_equal(h[:8192], golden["c1_hits_head"])
    assert sha(h[:, 1]) == golden["c1_prim_sha"]
    assert sha(h[:, 0]) == golden["c1_t_sha"]
    assert sha(h[:, 2:]) == golden["c1_uv_sha"]


def test_oracle_matches_reference_icospheres(golden, ico_tris):
    rays = scenes.random_rays(ico_tris, 1 << 20, seed=1)
    assert sha(rays) == golden["c2_rays_sha"]
    sel = golden["c2_sel"]
    sub = np.concatenate([sel[:96], sel[1024:1120]])
    h = oracle.trace_brute(ico_tris, rays[sub])
    ref = dict(zip(sel.tolist(), golden["c2_hits_sel"]))
    np.testing.assert_array_equal(h, np.stack([ref[i] for i in sub.tolist()]))


def test_oracle_visible_matches_reference(golden, cornell_tris, ico_tris):
    q1 = scenes.random_shadow_queries(cornell_tris, 1 << 20, seed=2)
    v1 = oracle.visible(cornell_tris, q1)
    assert sha(v1) == golden["c1_vis_sha"]
    q2 = scenes.random_shadow_queries(ico_tris, 1 << 16, seed=2)
    v2 = oracle.visible(ico_tris, q2[:256])
    np.testing.assert_array_equal(v2, golden["c2_vis"][:256])


@pytest.mark.skipif(not oracle.ref_available(), reason="reference harness not built (no reference tree)")
def test_oracle_vs_reference_live(cornell_tris):
    """Fresh inputs (other seeds) through the live reference harness."""
    rays = scenes.random_rays(cornell_tris, 200_000, seed=11, tmax=1e8)
    ref = oracle.RefScene(cornell_tris)
    np.testing.assert_array_equal(oracle.trace_brute(cornell_tris, rays), ref.trace_closest(rays))
    q = scenes.random_shadow_queries(cornell_tris, 200_000, seed=12)
    np.testing.assert_array_equal(oracle.visible(cornell_tris, q), ref.visible(q))


def test_oracle_agrees_with_fp64(cornell_tris):
    rays = scenes.random_rays(cornell_tris, 1 << 18, seed=3)
    h = oracle.trace_brute(cornell_tris, rays)
    t64, p64 = oracle.trace_fp64(cornell_tris, rays)
    p = prims(h)
    np.testing.assert_array_equal(p, p64)
    hit = p >= 0
    err = np.abs(h[hit, 0].astype(np.float64) - t64[hit])
    # float error of the reference's arithmetic is absolute (a few ulps of the
    # unit-scale operands, more on grazing hits); the relative error exceeds
    # 1e-6 only for origins very close to a surface
    assert err.max() < 1e-5
    rel = err / np.maximum(t64[hit], 1e-30)
    assert np.mean(rel <= 1e-6) > 0.995


# -- edge cases of Triangle::IsIntersect / BVH::IsIntersect semantics -------

TRI = np.array([0, 0, 0, 1, 0, 0, 0, 1, 0], dtype=np.float32)  # normal +z


def test_backface_culled():
    ok, *_ = oracle.tri_isect(TRI, [0.2, 0.2, -1], [0, 0, 1])  # hits from behind
    assert not ok
    ok, t, b1, b2 = oracle.tri_isect(TRI, [0.2, 0.2, 1], [0, 0, -1])
    assert ok and t == 1.0 and b1 == np.float32(0.2) and b2 == np.float32(0.2)


def test_degenerate_and_parallel():
    degenerate = np.array([0, 0, 0, 1, 1, 1, 2, 2, 2], dtype=np.float32)
    assert not oracle.tri_isect(degenerate, [0, 0, 1], [0, 0, -1])[0]
    assert not oracle.tri_isect(TRI, [0.2, 0.2, 1], [1, 0, 0])[0]


def test_t_bounds_and_strict_closest():
    ok, t, *_ = oracle.tri_isect(TRI, [0.2, 0.2, 1], [0, 0, -1], closest=np.float32(1.0))
    assert not ok  # t == closest is rejected (strict <)
    assert not oracle.tri_isect(TRI, [0.2, 0.2, -1], [0, 0, 1])[0]
    assert not oracle.tri_isect(TRI, [0.2, 0.2, 2e8], [0, 0, -1])[0]  # t > 1e8


def test_tie_keeps_first_index():
    # two identical triangles: the ray hits both at the same t, the first wins
    tris = np.stack([TRI, TRI])
    rays = np.array([[0.2, 0.2, 1, 0, 0, 0, -1, 1e8]], dtype=np.float32)
    h = oracle.trace_brute(tris, rays)
    assert prims(h)[0] == 0


def test_empty_batch(cornell_tris):
    h = oracle.trace_brute(cornell_tris, np.zeros((0, 8), np.float32))
    assert h.shape == (0, 4)
