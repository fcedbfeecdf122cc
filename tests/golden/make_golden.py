"""Generates tests/golden/*.npz by running the reference's own code
(oracle/_ref/libcrtref.so: the reference's BVH build, BVH::IsIntersect and
Light::Visible compiled as host C++) on the seeded synthetic inputs.

Run from the repository root where the reference tree is available:
    make -C oracle && python tests/golden/make_golden.py
The fixtures hold small result arrays plus SHA-256 digests of full 1M-ray
results, so the GPU box (which has no reference tree) can check the full
batches without storing them."""
from __future__ import annotations

import hashlib
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from cudaraytracer_b200 import scenes  # noqa: E402

N_RAYS = 1 << 20
HEAD = 8192


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def main() -> None:
    assert oracle.ref_available(), "oracle/_ref/libcrtref.so missing (make -C oracle on a box with the reference)"
    out = {}
    # Cornell box: full 1M rays and 1M shadow queries.
    c1 = scenes.cornell_box().triangles()
    r1 = scenes.random_rays(c1, N_RAYS, seed=1)
    q1 = scenes.random_shadow_queries(c1, N_RAYS, seed=2)
    ref1 = oracle.RefScene(c1)
    h1 = ref1.trace_closest(r1)
    v1 = ref1.visible(q1)
    out.update(
        c1_tris_sha=sha(c1), c1_rays_sha=sha(r1), c1_queries_sha=sha(q1),
        c1_prim_sha=sha(h1[:, 1]), c1_t_sha=sha(h1[:, 0]), c1_uv_sha=sha(h1[:, 2:]),
        c1_hits_head=h1[:HEAD], c1_vis_sha=sha(v1), c1_vis_head=v1[:HEAD],
        c1_hit_frac=np.float64((h1[:, 1].view(np.int32) >= 0).mean()), c1_occ_frac=np.float64(v1.mean()),
    )
    # Icosphere field: 1M rays (digests) + 2048 selected rays (arrays).
    c2 = scenes.icosphere_field(with_env=False).triangles()
    r2 = scenes.random_rays(c2, N_RAYS, seed=1)
    q2 = scenes.random_shadow_queries(c2, 1 << 16, seed=2)
    ref2 = oracle.RefScene(c2)
    h2 = ref2.trace_closest(r2)
    v2 = ref2.visible(q2)
    p2 = h2[:, 1].view(np.int32)
    sel = np.concatenate([np.nonzero(p2 >= 0)[0][:1024], np.nonzero(p2 < 0)[0][:1024]]).astype(np.int64)
    nodes, depth = ref2.stats()
    out.update(
        c2_tris_sha=sha(c2), c2_rays_sha=sha(r2), c2_queries_sha=sha(q2),
        c2_prim_sha=sha(h2[:, 1]), c2_t_sha=sha(h2[:, 0]),
        c2_sel=sel, c2_hits_sel=h2[sel], c2_vis=v2, c2_hit_frac=np.float64((p2 >= 0).mean()),
        c2_ref_nodes=np.int64(nodes), c2_ref_depth=np.int64(depth),
    )
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "trace_golden.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
