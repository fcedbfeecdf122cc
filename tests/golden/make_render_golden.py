"""Generates tests/golden/render_ref_*.npz: converged images rendered by the
reference's own renderer (oracle/_ref/libcrtref_render.so, a headless CUDA
build of its Scene loader and RenderLoop frame body). Needs a GPU and the
prebuilt oracle/_ref libraries; writes to the directory given (default
tests/golden). Each scene renders in a fresh process because the reference
keeps its scene in process-global state.

    python tests/golden/make_render_golden.py [outdir [scene ...]]
"""
from __future__ import annotations

import os
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

# name -> (scene factory kwargs, spp)
SCENES = {
    "cornell": ("cornell_box", dict(width=128, height=128, max_bounces=8), 4096),
    # the Cornell box at its stated render size: 256x256, depth 8, converged at 4096 spp
    "cornell_256": ("cornell_box", dict(width=256, height=256, max_bounces=8), 4096),
    "icospheres": ("icosphere_field", dict(n_spheres=8, level=2, width=64, height=64, env_size=(256, 128),
                                           max_bounces=6, sun_peak=40.0, sun_sigma=0.1), 16384),
    # diffuse textures (PNG, on a diffuse and a PBR material) and two area lights
    "cornell_tex2": ("cornell_box", dict(width=96, height=96, max_bounces=8, textured=True, lights=2), 4096),
    # the same scene with its textures as JPEG files (the reference decodes them with stb_image)
    "cornell_jpg": ("cornell_box", dict(width=96, height=96, max_bounces=8, textured=True, lights=2), 4096,
                    dict(texture_format="jpg")),
}


def scene_entry(name):
    """(factory name, factory kwargs, spp, SceneSpec.write kwargs)."""
    e = SCENES[name]
    return e[0], e[1], e[2], (e[3] if len(e) > 3 else {})


def render_one(name: str, outdir: str) -> None:
    import oracle
    from cudaraytracer_b200 import scenes

    fn, kw, spp, wkw = scene_entry(name)
    spec = getattr(scenes, fn)(**kw)
    with tempfile.TemporaryDirectory() as td:
        path = spec.write(td, name, **wkw)
        rr = oracle.RefRenderer(path)
        d, i, q, ms = rr.render(spp, with_sumsq=True)
    np.savez_compressed(os.path.join(outdir, f"render_ref_{name}.npz"), direct=d, indirect=i, sumsq=q,
                        spp=np.int64(spp), gpu_ms=np.float64(ms), camera=np.asarray(
                            rr.camera["position"] + rr.camera["left_down"] + rr.camera["du"] + rr.camera["dv"],
                            np.float32))
    print(f"{name}: {spp} spp in {ms:.1f} ms")


if __name__ == "__main__":
    if len(sys.argv) > 2 and sys.argv[1] == "--one":
        render_one(sys.argv[2], sys.argv[3])
    else:
        out = sys.argv[1] if len(sys.argv) > 1 else os.path.dirname(os.path.abspath(__file__))
        os.makedirs(out, exist_ok=True)
        for name in (sys.argv[2:] or list(SCENES)):
            subprocess.run([sys.executable, os.path.abspath(__file__), "--one", name, out], check=True)
