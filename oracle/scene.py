"""Oracle scene loader (test infrastructure): an independent Python
restatement of the reference's scene loading, used to check the library's
C++ loader and to feed the oracle renderer.

Follows Src/Core/scene.cpp (ParseCamera :187, ParseMaterials :254,
ParseObjects :398 with ResolveMaterialName :12 and BuildSceneMeshName :38,
ParseLights :539, InitCameraParam :646) and Src/Utils/objloader.cpp
(LoadObject :66, face normals when a face lacks vn :192-198). Floats are
rounded to float32 where the reference stores them."""
from __future__ import annotations

import json
import math
import os
from dataclasses import dataclass, field

import numpy as np

F = np.float32

TYPES = {"light": 0, "diffuse": 1, "pbr": 2, "dielectric": 3, "glass": 3, "subsurface": 4}


@dataclass
class OracleScene:
    width: int = 0
    height: int = 0
    fovy: float = 40.0
    max_bounces: int = 5
    rr: float = 0.8
    spp: int = 16
    direction: tuple = (0.0, 0.0, -1.0)
    denoise: bool = False
    verts: np.ndarray = None      # (n, 9) float32
    normals: np.ndarray = None    # (n, 9)
    uvs: np.ndarray = None        # (n, 6)
    prim_mesh: np.ndarray = None  # (n,) int32
    materials: np.ndarray = None  # (m, 16) float32
    meshes: np.ndarray = None     # (k, 8) float32
    lights: np.ndarray = None     # (l, 8) float32
    mesh_names: list = field(default_factory=list)
    env_light: int = -1
    env: np.ndarray = None        # (H, W, 4) float32
    textures: list = field(default_factory=list)  # (h, w, 4) uint8 RGBA, top row first


def _f32cross(a, b):
    return np.stack([a[:, 1] * b[:, 2] - a[:, 2] * b[:, 1],
                     a[:, 2] * b[:, 0] - a[:, 0] * b[:, 2],
                     a[:, 0] * b[:, 1] - a[:, 1] * b[:, 0]], 1).astype(F)


def _f32dot(a, b):
    return (a[:, 0] * b[:, 0] + (a[:, 1] * b[:, 1] + a[:, 2] * b[:, 2])).astype(F)


def _f32normalize(v):
    z = _f32dot(v, v)
    s = np.sqrt(z).astype(F)
    out = v.copy()
    ok = z > 0
    out[ok] = (v[ok] / s[ok, None]).astype(F)
    return out


def load_hdr(path: str) -> np.ndarray:
    """Radiance RGBE -> (H, W, 4) float32: byte * 2^(e-136), alpha 1."""
    data = open(path, "rb").read()
    p = 0

    def line():
        nonlocal p
        e = data.index(b"\n", p)
        l = data[p:e].decode("latin1")
        p = e + 1
        return l

    assert line().startswith("#?")
    while line() != "":
        pass
    parts = line().split()
    h, w = int(parts[1]), int(parts[3])
    out = np.zeros((h, w, 4), F)
    raw = np.frombuffer(data, np.uint8, offset=p)
    q = 0
    for y in range(h):
        if 8 <= w < 32768 and raw[q] == 2 and raw[q + 1] == 2 and not (raw[q + 2] & 0x80):
            q += 4
            scan = np.zeros((w, 4), np.uint8)
            for c in range(4):
                x = 0
                while x < w:
                    n = int(raw[q]); q += 1
                    if n > 128:
                        scan[x:x + n - 128, c] = raw[q]; q += 1; x += n - 128
                    else:
                        scan[x:x + n, c] = raw[q:q + n]; q += n; x += n
        else:
            scan = raw[q:q + 4 * w].reshape(w, 4); q += 4 * w
        e = scan[:, 3].astype(np.int32)
        f = np.where(e > 0, np.ldexp(np.float32(1.0), e - 136), 0).astype(F)
        out[y, :, :3] = scan[:, :3].astype(F) * f[:, None]
        out[y, :, 3] = 1.0
    return out


def load_obj(path: str):
    """Meshes of (name, material name, verts (n,9), normals (n,9), uvs (n,6))
    with identity transform, split by (shape, material) in first-face order."""
    P, N, T = [], [], []
    shapes = [{"name": "", "faces": []}]
    mtl_names, cur = [], -1
    base = os.path.dirname(path)
    for raw in open(path):
        s = raw.strip()
        if s.startswith("v "):
            P.append([float(x) for x in s.split()[1:4]])
        elif s.startswith("vn "):
            N.append([float(x) for x in s.split()[1:4]])
        elif s.startswith("vt "):
            T.append([float(x) for x in s.split()[1:3]])
        elif s.startswith("f "):
            cs = []
            for tok in s.split()[1:]:
                f = tok.split("/")
                r = lambda v, n: (int(v) - 1 if int(v) > 0 else n + int(v)) if v else -1
                cs.append((r(f[0], len(P)), r(f[1], len(T)) if len(f) > 1 else -1, r(f[2], len(N)) if len(f) > 2 else -1))
            for k in range(1, len(cs) - 1):
                shapes[-1]["faces"].append(((cs[0], cs[k], cs[k + 1]), cur))
        elif s[:2] in ("o ", "g ") or s in ("o", "g"):
            nm = s[2:] if len(s) > 2 else ""
            if shapes[-1]["faces"]:
                shapes.append({"name": nm, "faces": []})
            else:
                shapes[-1]["name"] = nm
        elif s.startswith("usemtl"):
            nm = s[6:].strip()
            cur = mtl_names.index(nm) if nm in mtl_names else -1
        elif s.startswith("mtllib"):
            try:
                for l in open(os.path.join(base, s[6:].strip())):
                    if l.strip().startswith("newmtl"):
                        mtl_names.append(l.strip()[6:].strip())
            except OSError:
                pass
    P = np.asarray(P, F).reshape(-1, 3)
    Nn = np.asarray(N, F).reshape(-1, 3)
    T = np.asarray(T, F).reshape(-1, 2)
    stem = os.path.splitext(os.path.basename(path))[0]
    meshes, lookup = [], {}
    for si, sh in enumerate(shapes):
        for (corners, mi) in sh["faces"]:
            mname = mtl_names[mi] if 0 <= mi < len(mtl_names) else ""
            key = (si, mi)
            if key not in lookup:
                sname = sh["name"] or f"{stem}_shape_{si}"
                lookup[key] = len(meshes)
                meshes.append([sname + ("::" + mname if mname else ""), mname, [], [], []])
            m = meshes[lookup[key]]
            v = np.stack([P[c[0]] for c in corners])
            has_n = all(c[2] >= 0 for c in corners)
            if has_n:
                n = _f32normalize(np.stack([Nn[c[2]] for c in corners]))
            else:
                fn = _f32normalize(_f32cross((v[1] - v[0])[None], (v[2] - v[0])[None]))[0]
                n = np.stack([fn, fn, fn])
            t = np.stack([T[c[1]] if c[1] >= 0 else np.zeros(2, F) for c in corners])
            m[2].append(v.reshape(9)); m[3].append(n.reshape(9)); m[4].append(t.reshape(6))
    return [(nm, mt, np.asarray(v, F), np.asarray(n, F), np.asarray(t, F)) for nm, mt, v, n, t in meshes]


def triangle_areas(v: np.ndarray) -> np.ndarray:
    t = v.reshape(-1, 3, 3)
    c = _f32cross((t[:, 1] - t[:, 0]).astype(F), (t[:, 2] - t[:, 0]).astype(F))
    return (F(0.5) * np.sqrt(_f32dot(c, c))).astype(F)


def read_png(path: str) -> np.ndarray:
    """(h, w, 4) uint8 RGBA of an 8-bit non-interlaced PNG (grey, RGB, RGBA,
    grey+alpha), rows top-down: the CPU check of the library's decoder."""
    import struct
    import zlib

    data = open(path, "rb").read()
    if data[:8] != b"\x89PNG\r\n\x1a\n":
        raise ValueError("not a PNG")
    pos, idat, hdr = 8, b"", None
    while pos < len(data):
        ln, typ = struct.unpack(">I4s", data[pos:pos + 8])
        body = data[pos + 8:pos + 8 + ln]
        if typ == b"IHDR":
            hdr = struct.unpack(">IIBBBBB", body)
        elif typ == b"IDAT":
            idat += body
        elif typ == b"IEND":
            break
        pos += 12 + ln
    w, h, depth, ctype, _, _, inter = hdr
    if depth != 8 or inter or ctype not in (0, 2, 4, 6):
        raise ValueError("unsupported PNG")
    ch = {0: 1, 2: 3, 4: 2, 6: 4}[ctype]
    raw = np.frombuffer(zlib.decompress(idat), np.uint8).reshape(h, 1 + w * ch)
    img = np.zeros((h, w * ch), np.int32)
    for y in range(h):
        f, row = raw[y, 0], raw[y, 1:].astype(np.int32)
        prev = img[y - 1] if y else np.zeros(w * ch, np.int32)
        out = np.zeros(w * ch, np.int32)
        for x in range(w * ch):
            a = out[x - ch] if x >= ch else 0
            b = prev[x]
            c = prev[x - ch] if x >= ch else 0
            if f == 0:
                pr = 0
            elif f == 1:
                pr = a
            elif f == 2:
                pr = b
            elif f == 3:
                pr = (a + b) >> 1
            else:
                pp = a + b - c
                pa, pb, pc = abs(pp - a), abs(pp - b), abs(pp - c)
                pr = a if (pa <= pb and pa <= pc) else (b if pb <= pc else c)
            out[x] = (row[x] + pr) & 255
        img[y] = out
    img = img.reshape(h, w, ch).astype(np.uint8)
    rgba = np.full((h, w, 4), 255, np.uint8)
    if ch in (1, 2):
        rgba[..., :3] = img[..., :1]
        if ch == 2:
            rgba[..., 3] = img[..., 1]
    else:
        rgba[..., :ch] = img
    return rgba


def load_scene(path: str) -> OracleScene:
    doc = json.load(open(path))
    s = OracleScene()
    cam = doc["camera"]
    if cam.get("type") != "pinhole":
        raise ValueError("unsupported camera")
    s.width, s.height = int(cam["resolution"][0]), int(cam["resolution"][1])
    s.fovy = float(F(cam.get("fov", 40)))
    s.max_bounces = int(cam.get("max_bounces", 5))
    s.rr = float(F(cam.get("rr", 0.8)))
    s.spp = int(cam.get("spp", 16))
    s.direction = tuple(float(F(x)) for x in cam.get("direction", [0, 0, -1]))
    s.denoise = bool(cam.get("denoise", False))
    tex_map = {}
    for tj in doc.get("textures", []):
        if "path" not in tj or "name" not in tj:
            continue
        try:
            img = read_png(tj["path"])
        except (OSError, ValueError):
            continue
        tex_map[tj["name"]] = len(s.textures)
        s.textures.append(img)
    mats = np.zeros((len(doc["materials"]), 16), F)
    mats[:, 0] = 1
    mats[:, 7] = 0.5
    mats[:, 9] = 1
    mats[:, 13] = 1
    mats[:, 14] = -1
    mat_map = {}
    for i, m in enumerate(doc["materials"]):
        if "name" not in m or "type" not in m or m["type"] not in TYPES:
            continue
        t = TYPES[m["type"]]
        row = mats[i]
        row[0] = t
        if t in (1, 2, 4) and "basecolor" in m:
            row[1:4] = m["basecolor"][:3]
        if t == 0 and "emission" in m:
            row[4:7] = m["emission"][:3]
        if t == 2:
            row[8] = m.get("metallic", 0.0)
            row[7] = m.get("roughness", 0.5)
        if t == 4:
            row[10:13] = m.get("scatter_distance", [1.0, 1.0, 1.0])[:3]
            if "ior" in m:
                row[13] = m["ior"]
            if "roughness" in m:
                row[7] = m["roughness"]
            row[8] = 0
        if t == 3:
            row[1:4] = m.get("basecolor", [1.0, 1.0, 1.0])[:3]
            row[13] = m.get("ior", 1.5)
            row[9] = m.get("transmission", 1.0)
            row[7] = m.get("roughness", 0.0)
            row[8] = 0
        if "diffuse_texture" in m and m["diffuse_texture"] in tex_map:
            row[14] = tex_map[m["diffuse_texture"]]
        mat_map[m["name"]] = i
    s.materials = mats
    verts, normals, uvs, pm, meshes, names = [], [], [], [], [], []
    mesh_map = {}
    for o in doc["objects"]:
        if "translate" in o or "rotate" in o or "scale" in o:
            identity = list(o.get("translate", [0, 0, 0])) == [0, 0, 0] and list(o.get("scale", [1, 1, 1])) == [1, 1, 1] \
                and all(list(r.values())[0] == 0 for r in o.get("rotate", []))
            if not identity:
                raise NotImplementedError("oracle loader handles identity object transforms only")
        loaded = load_obj(o["path"])
        expanded = len(loaded) > 1
        for (nm, mt, v, n, t) in loaded:
            if len(v) == 0:
                continue
            mname = o.get("material")
            if mname is None:
                ov = o.get("material_overrides", {})
                if mt and isinstance(ov, dict) and mt in ov:
                    mname = ov[mt]
                elif mt and mt in mat_map:
                    mname = mt
                else:
                    mname = o.get("default_material", "")
            if not mname or mname not in mat_map:
                continue
            mid = len(meshes)
            area = np.cumsum(triangle_areas(v), dtype=F)[-1]
            meshes.append([mat_map[mname], -1, len(pm), len(v), area, 0, 0, 0])
            pm.extend([mid] * len(v))
            verts.append(v); normals.append(n); uvs.append(t)
            name = o["name"] + "::" + nm if expanded else o["name"]
            mesh_map[name] = mid
            names.append(name)
    s.verts = np.concatenate(verts).astype(F)
    s.normals = np.concatenate(normals).astype(F)
    s.uvs = np.concatenate(uvs).astype(F)
    s.prim_mesh = np.asarray(pm, np.int32)
    s.mesh_names = names
    lights = []
    for l in doc["lights"]:
        if l.get("type") == "area":
            em = list(l.get("ke", [0, 0, 0]))
            if "material" in l and l["material"] in mat_map:
                em = list(mats[mat_map[l["material"]], 4:7])
            if l.get("lightMeshName") not in mesh_map:
                continue
            mid = mesh_map[l["lightMeshName"]]
            meshes[mid][1] = len(lights)
            lights.append([0, mid] + em[:3] + [0, 0, 0])
        elif l.get("type") == "env":
            s.env = load_hdr(l["path"])
            s.env_light = len(lights)
            lights.append([2, -1, 0, 0, 0, 0, 0, 0])
    s.meshes = np.asarray(meshes, F).reshape(-1, 8)
    s.lights = np.asarray(lights, F).reshape(-1, 8)
    return s


def orbit_camera(s: OracleScene):
    """InitCameraParam + ComputeCameraParam (scene.cpp:646-667,
    camera.h:58-84) in double precision: returns a dict of float64 arrays."""
    v = s.verts.reshape(-1, 3).astype(np.float64)
    lo, hi = v.min(0), v.max(0)
    target = (lo + hi) * 0.5
    diag = np.linalg.norm(hi - lo)
    fovy = s.fovy
    dist = diag * 0.5 / math.sin(math.radians(fovy) / 2) * 0.6
    d = np.asarray(s.direction, np.float64)
    d = d / np.linalg.norm(d)
    theta = math.acos(d[1])
    phi = math.atan2(d[0], d[2])
    pos = target + dist * np.array([math.sin(theta) * math.sin(phi), math.cos(theta), math.sin(theta) * math.cos(phi)])
    w = (pos - target) / np.linalg.norm(pos - target)
    u = np.cross([0, 1, 0], w)
    u /= np.linalg.norm(u)
    vv = np.cross(w, u)
    vv /= np.linalg.norm(vv)
    h = 2 * dist * math.tan(math.radians(fovy / 2))
    ww = h * s.width / s.height
    du = ww * u / s.width
    dv = h * vv / s.height
    ld = target - (s.width // 2) * du - (s.height // 2) * dv  # integer halves, as camera.h:83
    return {"position": pos, "target": target, "distance": dist, "u": u, "v": vv, "w": w, "du": du, "dv": dv,
            "left_down": ld, "theta": math.degrees(theta), "phi": math.degrees(phi)}
