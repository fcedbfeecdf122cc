"""CPU restatement of the reference's display resolve (GatherKernel,
Src/Core/renderer.cuh:956-1030), test infrastructure only: arrays are
(H, W, c) with rows bottom-up as the accumulators and G-buffer planes."""
from __future__ import annotations

import numpy as np


def _byte(x):
    return np.clip(np.asarray(x, dtype=np.float32) * np.float32(255.0), 0, 255).astype(np.uint8)


def gather(mode, spp, direct, indirect, gb, bmin, bmax, cam_pos, denoised=False):
    """uchar4 pixels (H, W, 4), indexed like the reference's display buffer
    (pixel (i, j) at row j of the returned array)."""
    d = np.asarray(direct, dtype=np.float32)
    h, w = d.shape[:2]
    out = np.zeros((h, w, 4), np.uint8)
    out[..., 3] = 255
    if mode == 0:
        c = (d[..., :3] + np.asarray(indirect, dtype=np.float32)[..., :3])
        if not denoised:
            c = c / np.float32(spp)
        v = np.clip(np.power(c, np.float32(1 / 2.2)) * np.float32(255.0), 0, 255).astype(np.uint8)
        out[::-1, :, :3] = v  # written to the flipped row
        return out
    flip = lambda a: np.asarray(a)[::-1]  # read at the flipped row
    if mode == 1:
        bmin, bmax = np.asarray(bmin, np.float32), np.asarray(bmax, np.float32)
        diag = np.float32(np.linalg.norm(bmax - bmin))
        far = diag + np.float32(np.linalg.norm(np.asarray(cam_pos, np.float32) - (bmin + bmax) * np.float32(0.5)))
        z = flip(gb["motion_depth"])[..., 2]
        v = _byte((z - np.float32(0.1)) / (far - np.float32(0.1)))
        out[..., 0] = out[..., 1] = out[..., 2] = v
    elif mode == 2:
        n = flip(gb["normal_mat"]).astype(np.float32)
        out[..., :3] = _byte(n[..., :3] / np.float32(65535.0))
    elif mode == 3:
        i = flip(gb["bary_mesh"])[..., 3].astype(np.int64)
        out[..., 0], out[..., 1], out[..., 2] = (i * 37) % 256, (i * 57) % 256, (i * 97) % 256
    else:
        p = flip(gb["pos_tri"])[..., :3].astype(np.float32)
        lo, hi = np.asarray(bmin, np.float32), np.asarray(bmax, np.float32)
        out[..., :3] = _byte((p - lo) / (hi - lo))
    return out
