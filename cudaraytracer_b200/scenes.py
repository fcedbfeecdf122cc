"""Seeded synthetic scenes and ray batches for the benchmark configurations.

The reference's own scene assets are not distributed with it (every scene
JSON points at absent OBJ/HDR files), so the workloads are generated here and
written in the reference's formats (OBJ without normals, Radiance .hdr, scene
JSON with the schema of Src/Core/scene.cpp:129-252) so that the same files
feed both this tracer and the reference.

* Cornell box: 36 triangles, unit box x,y,z in [0,1] open toward +z; walls
  face the interior (the reference culls back faces), boxes face outward.
* Icosphere field: 64 icospheres subdivided 5 times (20,480 triangles each),
  seeded centres/radii/value-noise displacement, 4-way material mix, and a
  procedural sky + sun environment map.
"""
from __future__ import annotations

import json
import math
import os
from dataclasses import dataclass, field

import numpy as np

# --------------------------------------------------------------------------
# geometry helpers
# --------------------------------------------------------------------------


def _quad(p0, p1, p2, p3):
    """Two triangles (p0,p1,p2), (p0,p2,p3): CCW as listed."""
    return [(p0, p1, p2), (p0, p2, p3)]


def _box(center, size, angle_deg):
    """Axis box rotated about +y, 12 triangles with outward normals."""
    cx, cy, cz = center
    sx, sy, sz = (s * 0.5 for s in size)
    a = math.radians(angle_deg)
    ca, sa = math.cos(a), math.sin(a)

    def P(x, y, z):
        return (cx + ca * x + sa * z, cy + y, cz - sa * x + ca * z)

    c = {
        (i, j, k): P(i * sx, j * sy, k * sz)
        for i in (-1, 1)
        for j in (-1, 1)
        for k in (-1, 1)
    }
    tris = []
    # each face listed CCW seen from outside
    tris += _quad(c[1, -1, -1], c[1, 1, -1], c[1, 1, 1], c[1, -1, 1])  # +x
    tris += _quad(c[-1, -1, -1], c[-1, -1, 1], c[-1, 1, 1], c[-1, 1, -1])  # -x
    tris += _quad(c[-1, 1, -1], c[-1, 1, 1], c[1, 1, 1], c[1, 1, -1])  # +y
    tris += _quad(c[-1, -1, -1], c[1, -1, -1], c[1, -1, 1], c[-1, -1, 1])  # -y
    tris += _quad(c[-1, -1, 1], c[1, -1, 1], c[1, 1, 1], c[-1, 1, 1])  # +z
    tris += _quad(c[-1, -1, -1], c[-1, 1, -1], c[1, 1, -1], c[1, -1, -1])  # -z
    return tris


@dataclass
class Mesh:
    name: str
    material: str
    tris: np.ndarray  # (n, 9) float32
    uvs: np.ndarray | None = None  # (n, 6) float32 texture coordinates per corner


@dataclass
class SceneSpec:
    """A generated scene: meshes, materials, lights and camera block."""

    meshes: list
    materials: list
    lights: list
    camera: dict
    env: np.ndarray | None = None  # (H, W, 3) float32
    extra: dict = field(default_factory=dict)
    textures: dict = field(default_factory=dict)  # name -> (h, w, 4) uint8 RGBA, top row first

    def triangles(self) -> np.ndarray:
        return np.concatenate([m.tris for m in self.meshes]).astype(np.float32)

    def write(self, directory: str, name: str = "scene", texture_format: str = "png") -> str:
        """Writes OBJ / HDR / JSON in the reference's schema; returns the
        JSON path. Asset paths are absolute, as in the reference's scenes.
        Textures are written as PNG, or as baseline JPEG (quality 95, 4:4:4
        chroma, through Pillow) with texture_format="jpg"."""
        os.makedirs(directory, exist_ok=True)
        directory = os.path.abspath(directory)
        objects = []
        for m in self.meshes:
            path = os.path.join(directory, f"{name}_{m.name}.obj")
            write_obj(path, m.tris, m.uvs)
            objects.append({"name": m.name, "path": path, "material": m.material})
        textures = []
        for tname, img in self.textures.items():
            if texture_format == "jpg":
                from PIL import Image

                path = os.path.join(directory, f"{name}_tex_{tname}.jpg")
                Image.fromarray(np.ascontiguousarray(img[..., :3], dtype=np.uint8)).save(path, quality=95,
                                                                                         subsampling=0)
            else:
                path = os.path.join(directory, f"{name}_tex_{tname}.png")
                write_png(path, img)
            textures.append({"name": tname, "path": path})
        lights = []
        for l in self.lights:
            l = dict(l)
            if l["type"] == "env":
                path = os.path.join(directory, f"{name}_env.hdr")
                write_hdr(path, self.env)
                l["path"] = path
            lights.append(l)
        doc = {
            "camera": self.camera,
            "textures": textures,
            "materials": self.materials,
            "objects": objects,
            "lights": lights,
        }
        jpath = os.path.join(directory, f"{name}.json")
        with open(jpath, "w") as f:
            json.dump(doc, f, indent=1)
        return jpath


def write_obj(path: str, tris: np.ndarray, uvs: np.ndarray | None = None) -> None:
    """OBJ with one vertex per triangle corner, %.9g so floats round-trip
    exactly, no normals (the reference then uses face normals,
    Src/Utils/objloader.cpp:192-198); texture coordinates (vt) when given."""
    t = np.asarray(tris, dtype=np.float32).reshape(-1, 3, 3)
    lines = []
    for tri in t:
        for v in tri:
            lines.append("v %.9g %.9g %.9g" % (float(v[0]), float(v[1]), float(v[2])))
    n = t.shape[0]
    if uvs is not None:
        u = np.asarray(uvs, dtype=np.float32).reshape(-1, 3, 2)
        for tri in u:
            for c in tri:
                lines.append("vt %.9g %.9g" % (float(c[0]), float(c[1])))
    for i in range(n):
        b = 3 * i + 1
        if uvs is not None:
            lines.append("f %d/%d %d/%d %d/%d" % (b, b, b + 1, b + 1, b + 2, b + 2))
        else:
            lines.append("f %d %d %d" % (b, b + 1, b + 2))
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def write_png(path: str, rgba: np.ndarray) -> None:
    """8-bit RGBA PNG, rows top-down; row filters cycle through the five PNG
    filter types (None, Sub, Up, Average, Paeth) so a decoder meets all."""
    import struct
    import zlib

    img = np.ascontiguousarray(rgba, dtype=np.uint8)
    h, w, _ = img.shape
    bpp = 4
    rows = []
    prev = np.zeros(w * 4, np.int32)
    for y in range(h):
        cur = img[y].reshape(-1).astype(np.int32)
        ft = y % 5
        a = np.concatenate([np.zeros(bpp, np.int32), cur[:-bpp]])
        c = np.concatenate([np.zeros(bpp, np.int32), prev[:-bpp]])
        if ft == 0:
            f = cur
        elif ft == 1:
            f = cur - a
        elif ft == 2:
            f = cur - prev
        elif ft == 3:
            f = cur - ((a + prev) >> 1)
        else:
            p = a + prev - c
            pa, pb, pc = np.abs(p - a), np.abs(p - prev), np.abs(p - c)
            pr = np.where((pa <= pb) & (pa <= pc), a, np.where(pb <= pc, prev, c))
            f = cur - pr
        rows.append(bytes([ft]) + (f & 255).astype(np.uint8).tobytes())
        prev = cur

    def chunk(tag, body):
        return struct.pack(">I", len(body)) + tag + body + struct.pack(">I", zlib.crc32(tag + body) & 0xFFFFFFFF)

    raw = b"".join(rows)
    with open(path, "wb") as f:
        f.write(b"\x89PNG\r\n\x1a\n")
        f.write(chunk(b"IHDR", struct.pack(">IIBBBBB", w, h, 8, 6, 0, 0, 0)))
        f.write(chunk(b"IDAT", zlib.compress(raw, 6)))
        f.write(chunk(b"IEND", b""))


def checker_texture(w=64, h=48, seed=0) -> np.ndarray:
    """A seeded RGBA test texture: a coloured checkerboard over a gradient."""
    rng = np.random.default_rng(seed)
    yy, xx = np.mgrid[0:h, 0:w]
    cols = rng.integers(40, 230, size=(2, 3))
    chk = ((xx // 8 + yy // 8) % 2).astype(np.int32)
    img = np.zeros((h, w, 4), np.uint8)
    img[..., :3] = np.clip(cols[chk] * (0.6 + 0.4 * xx[..., None] / max(1, w - 1)), 0, 255).astype(np.uint8)
    img[..., 3] = 255
    return img


def write_hdr(path: str, img: np.ndarray) -> None:
    """Radiance RGBE (.hdr), flat (non-RLE) scanlines, top row first."""
    img = np.asarray(img, dtype=np.float32)
    h, w, _ = img.shape
    v = img.max(axis=2)
    m, e = np.frexp(v)
    scale = np.where(v > 1e-32, m * 256.0 / np.where(v > 1e-32, v, 1.0), 0.0)
    rgbe = np.zeros((h, w, 4), dtype=np.uint8)
    rgbe[..., :3] = np.clip(img * scale[..., None], 0, 255).astype(np.uint8)
    rgbe[..., 3] = np.where(v > 1e-32, e + 128, 0).astype(np.uint8)
    with open(path, "wb") as f:
        f.write(b"#?RADIANCE\nFORMAT=32-bit_rle_rgbe\n\n")
        f.write(f"-Y {h} +X {w}\n".encode())
        f.write(rgbe.tobytes())


def decode_hdr_rgbe(img: np.ndarray) -> np.ndarray:
    """Float values a Radiance loader produces for the data write_hdr stores
    (stb_image: byte * 2^(e - 136), alpha 1)."""
    img = np.asarray(img, dtype=np.float32)
    v = img.max(axis=2)
    m, e = np.frexp(v)
    scale = np.where(v > 1e-32, m * 256.0 / np.where(v > 1e-32, v, 1.0), 0.0)
    q = np.clip(img * scale[..., None], 0, 255).astype(np.uint8).astype(np.float32)
    ee = np.where(v > 1e-32, e + 128, 0)
    f = np.where(ee > 0, np.ldexp(1.0, (ee - 136).astype(np.int32)), 0.0).astype(np.float32)
    return q * f[..., None]


# --------------------------------------------------------------------------
# Cornell box (36 triangles)
# --------------------------------------------------------------------------

WHITE = [0.725, 0.71, 0.68]
RED = [0.63, 0.065, 0.05]
GREEN = [0.14, 0.45, 0.09]
LIGHT_KE = [17.0, 12.0, 4.0]


def cornell_box(width=256, height=256, spp=16, max_bounces=8, rr=0.8, seed=None, textured=False,
                lights=1) -> SceneSpec:
    """The 36-triangle Cornell box. With a seed, a variant of it: box
    positions, sizes and rotations, wall colours and the light's size and
    emission drawn from ranges around the canonical values (the
    denoiser's training and test scenes). textured=True puts a diffuse
    texture on the back wall (UVs spanning the wall) and a textured PBR
    material on the boxes (planar UVs); lights=2 splits the ceiling light
    into two area lights."""
    P = lambda x, y, z: (float(x), float(y), float(z))
    white, red, green = [], [], []
    wall_l, wall_r, ke = RED, GREEN, LIGHT_KE
    b1 = ((0.33, 0.30, 0.36), (0.28, 0.60, 0.28), 18.0)
    b2 = ((0.67, 0.15, 0.63), (0.28, 0.30, 0.28), -18.0)
    half = 0.125
    if seed is not None:
        rng = np.random.default_rng(seed)
        hue = lambda base: np.clip(np.asarray(base) * rng.uniform(0.6, 1.4, 3), 0.02, 0.9).round(4).tolist()
        wall_l, wall_r = hue(RED), hue(GREEN)
        ke = (np.asarray(LIGHT_KE) * rng.uniform(0.7, 1.3)).round(3).tolist()
        half = float(rng.uniform(0.09, 0.17))
        hgt1, hgt2 = rng.uniform(0.4, 0.7), rng.uniform(0.2, 0.35)
        s1, s2 = rng.uniform(0.22, 0.30, 2)
        b1 = ((rng.uniform(0.27, 0.38), hgt1 / 2, rng.uniform(0.30, 0.42)), (s1, hgt1, s1), rng.uniform(8, 30))
        b2 = ((rng.uniform(0.62, 0.72), hgt2 / 2, rng.uniform(0.58, 0.70)), (s2, hgt2, s2), -rng.uniform(8, 30))
    # floor y=0 (+y), ceiling y=1 (-y), back z=0 (+z): CCW seen from inside
    white += _quad(P(0, 0, 0), P(0, 0, 1), P(1, 0, 1), P(1, 0, 0))
    white += _quad(P(0, 1, 0), P(1, 1, 0), P(1, 1, 1), P(0, 1, 1))
    back = _quad(P(0, 0, 0), P(1, 0, 0), P(1, 1, 0), P(0, 1, 0))
    if not textured:
        white += back
    red += _quad(P(0, 0, 0), P(0, 1, 0), P(0, 1, 1), P(0, 0, 1))  # x=0, +x
    green += _quad(P(1, 0, 0), P(1, 0, 1), P(1, 1, 1), P(1, 1, 0))  # x=1, -x
    boxes = _box(*b1)
    boxes += _box(*b2)
    h = 0.999
    lo, hi = 0.5 - half, 0.5 + half

    def arr(t):
        return np.asarray(t, dtype=np.float32).reshape(-1, 9)

    def planar_uv(t, ax_u, ax_v):
        v = arr(t).reshape(-1, 3, 3)
        return np.stack([v[:, :, ax_u], v[:, :, ax_v]], -1).reshape(-1, 6).astype(np.float32)

    if lights == 2:  # two ceiling lights side by side, same material
        mid = 0.5
        light_meshes = [Mesh("light", "light", arr(_quad(P(lo, h, lo), P(mid - 0.02, h, lo), P(mid - 0.02, h, hi),
                                                         P(lo, h, hi)))),
                        Mesh("light_b", "light", arr(_quad(P(mid + 0.02, h, lo), P(hi, h, lo), P(hi, h, hi),
                                                           P(mid + 0.02, h, hi))))]
    else:
        light_meshes = [Mesh("light", "light", arr(_quad(P(lo, h, lo), P(hi, h, lo), P(hi, h, hi), P(lo, h, hi))))]
    meshes = [
        Mesh("walls_white", "white", arr(white)),
        Mesh("wall_red", "red", arr(red)),
        Mesh("wall_green", "green", arr(green)),
    ]
    materials = [
        {"name": "white", "type": "diffuse", "basecolor": WHITE},
        {"name": "red", "type": "diffuse", "basecolor": wall_l},
        {"name": "green", "type": "diffuse", "basecolor": wall_r},
        {"name": "light", "type": "light", "emission": ke},
    ]
    textures = {}
    if textured:
        meshes.append(Mesh("wall_back", "checker", arr(back), planar_uv(back, 0, 1)))
        meshes.append(Mesh("boxes", "pbr_tex", arr(boxes), planar_uv(boxes, 0, 1)))
        materials.append({"name": "checker", "type": "diffuse", "basecolor": WHITE, "diffuse_texture": "checker"})
        materials.append({"name": "pbr_tex", "type": "pbr", "basecolor": WHITE, "metallic": 0.3, "roughness": 0.45,
                          "diffuse_texture": "stripes"})
        textures["checker"] = checker_texture(64, 48, seed=1)
        stripes = checker_texture(32, 32, seed=2)
        stripes[:, ::4, :3] = 240
        textures["stripes"] = stripes
    else:
        meshes.append(Mesh("boxes", "white", arr(boxes)))
    meshes += light_meshes
    lights = [{"type": "area", "lightMeshName": m.name, "material": "light"} for m in light_meshes]
    camera = {
        "type": "pinhole",
        "resolution": [width, height],
        "fov": 40,
        "max_bounces": max_bounces,
        "rr": rr,
        "spp": spp,
        "direction": [0, 0, 1],
        "denoise": False,
    }
    return SceneSpec(meshes, materials, lights, camera, textures=textures)


# --------------------------------------------------------------------------
# Icosphere field (64 x 20,480 triangles) + environment map
# --------------------------------------------------------------------------


def icosphere(level: int):
    """Unit icosphere: (verts (V,3) float64, faces (F,3) int64), CCW outward."""
    t = (1.0 + 5 ** 0.5) / 2.0
    v = np.array(
        [
            [-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0],
            [0, -1, t], [0, 1, t], [0, -1, -t], [0, 1, -t],
            [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1],
        ],
        dtype=np.float64,
    )
    f = np.array(
        [
            [0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11],
            [1, 5, 9], [5, 11, 4], [11, 10, 2], [10, 7, 6], [7, 1, 8],
            [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8], [3, 8, 9],
            [4, 9, 5], [2, 4, 11], [6, 2, 10], [8, 6, 7], [9, 8, 1],
        ],
        dtype=np.int64,
    )
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    for _ in range(level):
        a, b, c = f[:, 0], f[:, 1], f[:, 2]
        edges = np.stack([np.stack([a, b], 1), np.stack([b, c], 1), np.stack([c, a], 1)], 1).reshape(-1, 2)
        key = np.sort(edges, axis=1)
        uniq, inv = np.unique(key, axis=0, return_inverse=True)
        mids = v[uniq[:, 0]] + v[uniq[:, 1]]
        mids /= np.linalg.norm(mids, axis=1, keepdims=True)
        mid_idx = (np.asarray(inv).reshape(-1, 3) + len(v)).astype(np.int64)
        v = np.concatenate([v, mids])
        ab, bc, ca = mid_idx[:, 0], mid_idx[:, 1], mid_idx[:, 2]
        f = np.concatenate(
            [np.stack([a, ab, ca], 1), np.stack([b, bc, ab], 1), np.stack([c, ca, bc], 1), np.stack([ab, bc, ca], 1)]
        )
    return v, f


def value_noise(p: np.ndarray, rng: np.random.Generator, freq: float = 4.0, lattice: int = 32) -> np.ndarray:
    """Trilinear value noise in [0,1) on a periodic random lattice."""
    table = rng.random((lattice, lattice, lattice))
    q = p * freq
    i0 = np.floor(q).astype(np.int64)
    fr = q - i0
    s = fr * fr * (3 - 2 * fr)
    out = np.zeros(len(p))
    for dx in (0, 1):
        for dy in (0, 1):
            for dz in (0, 1):
                w = (
                    (s[:, 0] if dx else 1 - s[:, 0])
                    * (s[:, 1] if dy else 1 - s[:, 1])
                    * (s[:, 2] if dz else 1 - s[:, 2])
                )
                ix = (i0[:, 0] + dx) % lattice
                iy = (i0[:, 1] + dy) % lattice
                iz = (i0[:, 2] + dz) % lattice
                out += w * table[ix, iy, iz]
    return out


def env_map(width=2048, height=1024, seed=7, sun_peak=5000.0, sun_sigma=0.03):
    """Sky gradient + Gaussian sun lobe. Pixel (x,y) <-> direction with
    theta = (y+.5)/H*pi from +y, phi = (x+.5)/W*2pi, dir = (sin t sin p,
    cos t, sin t cos p): the mapping of Light::Emission
    (Src/Core/light.cu:141-155)."""
    rng = np.random.default_rng(seed)
    th = (np.arange(height) + 0.5) / height * np.pi
    ph = (np.arange(width) + 0.5) / width * 2 * np.pi
    T, Pp = np.meshgrid(th, ph, indexing="ij")
    d = np.stack([np.sin(T) * np.sin(Pp), np.cos(T), np.sin(T) * np.cos(Pp)], -1)
    up = np.clip(d[..., 1], 0, 1)[..., None]
    horizon = np.array([0.8, 0.85, 0.9])
    zenith = np.array([0.2, 0.4, 0.9])
    ground = np.array([0.15, 0.13, 0.10])
    sky = np.where(d[..., 1:2] >= 0, horizon * (1 - up) + zenith * up, ground)
    # seeded sun direction in the upper hemisphere
    z = rng.uniform(0.3, 0.9)
    a = rng.uniform(0, 2 * np.pi)
    r = np.sqrt(1 - z * z)
    sun = np.array([r * np.sin(a), z, r * np.cos(a)])
    ang = np.arccos(np.clip(d @ sun, -1, 1))
    lobe = sun_peak * np.exp(-(ang ** 2) / (2 * sun_sigma ** 2))
    img = sky + lobe[..., None] * np.array([1.0, 0.95, 0.85])
    return img.astype(np.float32)


def icosphere_field(n_spheres=64, level=5, seed=1, width=1920, height=1080, spp=64, max_bounces=16, rr=0.8,
                    env_size=(2048, 1024), with_env=True, sun_peak=5000.0, sun_sigma=0.03) -> SceneSpec:
    rng = np.random.default_rng(seed)
    uv, uf = icosphere(level)
    meshes, materials = [], []
    kinds = rng.choice(4, size=n_spheres, p=[0.4, 0.3, 0.2, 0.1])
    for s in range(n_spheres):
        c = rng.uniform(-1, 1, 3)
        rad = rng.uniform(0.02, 0.1)
        disp = 0.05 * rad * (2 * value_noise(uv + s * 7.31, rng) - 1)
        verts = c + uv * (rad + disp)[:, None]
        tris = verts[uf].reshape(-1, 9).astype(np.float32)
        name = f"sphere{s:03d}"
        k = int(kinds[s])
        if k == 0:
            mat = {"name": name, "type": "diffuse", "basecolor": rng.uniform(0.1, 0.9, 3).round(4).tolist()}
        elif k == 1:
            mat = {"name": name, "type": "pbr", "basecolor": rng.uniform(0.5, 1.0, 3).round(4).tolist(),
                   "metallic": 1.0, "roughness": round(float(rng.uniform(0.05, 0.5)), 4)}
        elif k == 2:
            mat = {"name": name, "type": "dielectric", "basecolor": [1.0, 1.0, 1.0], "ior": 1.5}
        else:
            mfp = round(float(rng.uniform(0.01, 0.1)), 4)
            mat = {"name": name, "type": "subsurface", "basecolor": rng.uniform(0.3, 0.95, 3).round(4).tolist(),
                   "scatter_distance": [mfp, mfp, mfp], "ior": 1.3, "roughness": 0.3}
        materials.append(mat)
        meshes.append(Mesh(name, name, tris))
    camera = {
        "type": "pinhole",
        "resolution": [width, height],
        "fov": 40,
        "max_bounces": max_bounces,
        "rr": rr,
        "spp": spp,
        "direction": [0.3, 0.4, 1.0],
        "denoise": False,
    }
    lights, env = [], None
    if with_env:
        env = env_map(*env_size, seed=seed + 6, sun_peak=sun_peak, sun_sigma=sun_sigma)
        lights = [{"type": "env"}]
    return SceneSpec(meshes, materials, lights, camera, env=env)


# --------------------------------------------------------------------------
# ray and shadow-query batches
# --------------------------------------------------------------------------


def scene_bounds(tris: np.ndarray):
    v = np.asarray(tris, dtype=np.float32).reshape(-1, 3)
    return v.min(0), v.max(0)


def unit_sphere(rng: np.random.Generator, n: int) -> np.ndarray:
    z = rng.uniform(-1.0, 1.0, n)
    phi = rng.uniform(0.0, 2 * np.pi, n)
    r = np.sqrt(np.maximum(0.0, 1 - z * z))
    return np.stack([r * np.cos(phi), r * np.sin(phi), z], 1)


def random_rays(tris: np.ndarray, n: int, seed: int = 1, tmin: float = 0.0, tmax: float = 1e8) -> np.ndarray:
    """n rays (n, 8) float32: origins uniform in the scene AABB, directions
    uniform on the sphere, tmin/tmax as given."""
    rng = np.random.default_rng(seed)
    lo, hi = scene_bounds(tris)
    out = np.empty((n, 8), dtype=np.float32)
    step = 1 << 22
    for b in range(0, n, step):
        m = min(step, n - b)
        out[b:b + m, 0:3] = lo + (hi - lo) * rng.random((m, 3))
        out[b:b + m, 3] = tmin
        out[b:b + m, 4:7] = unit_sphere(rng, m)
        out[b:b + m, 7] = tmax
    return out


def random_shadow_queries(tris: np.ndarray, n: int, seed: int = 2) -> np.ndarray:
    """n Light::Visible queries (n, 12) float32: shading points uniform in the
    AABB with random unit normals, light points uniform on random triangles
    with those triangles' geometric normals."""
    rng = np.random.default_rng(seed)
    t = np.asarray(tris, dtype=np.float32).reshape(-1, 3, 3)
    lo, hi = scene_bounds(tris)
    out = np.empty((n, 12), dtype=np.float32)
    step = 1 << 22
    for b in range(0, n, step):
        m = min(step, n - b)
        out[b:b + m, 0:3] = lo + (hi - lo) * rng.random((m, 3))
        out[b:b + m, 3:6] = unit_sphere(rng, m)
        k = rng.integers(0, len(t), m)
        u = rng.random((m, 2))
        flip = u.sum(1) > 1
        u[flip] = 1 - u[flip]
        v0, v1, v2 = t[k, 0], t[k, 1], t[k, 2]
        p = v0 + u[:, 0:1] * (v1 - v0) + u[:, 1:2] * (v2 - v0)
        nrm = np.cross(v1 - v0, v2 - v0)
        nrm /= np.maximum(np.linalg.norm(nrm, axis=1, keepdims=True), 1e-30)
        out[b:b + m, 6:9] = p
        out[b:b + m, 9:12] = nrm
    return out
