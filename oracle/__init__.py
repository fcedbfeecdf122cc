"""Oracle (test infrastructure only): ctypes access to
  * liboracle.so          - the CPU restatement of the reference's render path
                            (crt_oracle.c), and
  * _ref/libcrtref.so     - the reference's own sources compiled as host C++
                            (present when built where the reference tree is).
Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference
legs use this package, as the checker; the product never imports it."""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libcrtref.so")
REF_CUDA_SO = os.path.join(HERE, "_ref", "libcrtref_cuda.so")
REF_RENDER_SO = os.path.join(HERE, "_ref", "libcrtref_render.so")
# the same builds with device link-time optimisation (oracle/Makefile)
REF_CUDA_LTO_SO = os.path.join(HERE, "_ref", "libcrtref_cuda_lto.so")
REF_RENDER_LTO_SO = os.path.join(HERE, "_ref", "libcrtref_render_lto.so")

_VP = C.c_void_p


# Where the reference source tree is read from when oracle/_ref is built
# (CRT_REFERENCE_DIR overrides it). Without the tree only liboracle.so builds.
DEFAULT_REFERENCE_DIR = "/root/reference"


def build() -> None:
    env = dict(os.environ)
    env.setdefault("CRT_REFERENCE_DIR", DEFAULT_REFERENCE_DIR)
    r = subprocess.run(["make", "-C", HERE, "-j", str(os.cpu_count() or 1)], capture_output=True, text=True,
                       env=env)
    if r.returncode != 0:
        raise RuntimeError("building the oracle failed:\n" + r.stdout[-3000:] + r.stderr[-3000:])


_oracle = None
_ref = None


class _OracleSceneC(C.Structure):
    _fields_ = [
        ("verts", _VP), ("normals", _VP), ("uvs", _VP), ("prim_mesh", _VP), ("ntris", C.c_long),
        ("meshes", _VP), ("materials", _VP), ("lights", _VP),
        ("nmeshes", C.c_int), ("nmaterials", C.c_int), ("nlights", C.c_int),
        ("env_light", C.c_int), ("env", _VP), ("env_w", C.c_int), ("env_h", C.c_int),
        ("cam_pos", C.c_float * 3), ("cam_ld", C.c_float * 3), ("cam_du", C.c_float * 3), ("cam_dv", C.c_float * 3),
        ("width", C.c_int), ("height", C.c_int), ("max_bounces", C.c_int), ("rr", C.c_float),
        ("rr_start", C.c_int), ("seed", C.c_ulonglong),
        ("ntex", C.c_int), ("tex", _VP), ("tex_w", _VP), ("tex_h", _VP),
    ]


def render(scene, camera, spp: int, first_sample: int = 0, seed: int = 1, max_bounces=None, rr=None,
           rr_start: int = 0, width=None, height=None, nthreads: int = 0):
    """Oracle path tracer over an oracle.scene.OracleScene with camera
    vectors {position, left_down, du, dv}; returns (direct, indirect, sumsq)
    float32 arrays of shape (H, W, 4), sums over samples, bottom-up rows."""
    keep = []

    def arr(a, dt):
        a = np.ascontiguousarray(a, dtype=dt)
        keep.append(a)
        return a.ctypes.data

    w = int(width or scene.width)
    h = int(height or scene.height)
    o = _OracleSceneC()
    o.verts = arr(scene.verts, np.float32)
    o.normals = arr(scene.normals, np.float32)
    o.uvs = arr(scene.uvs, np.float32)
    o.prim_mesh = arr(scene.prim_mesh, np.int32)
    o.ntris = len(scene.prim_mesh)
    o.meshes = arr(scene.meshes, np.float32)
    o.materials = arr(scene.materials, np.float32)
    o.lights = arr(scene.lights, np.float32)
    o.nmeshes, o.nmaterials, o.nlights = len(scene.meshes), len(scene.materials), len(scene.lights)
    o.env_light = scene.env_light
    if scene.env_light >= 0:
        o.env = arr(scene.env, np.float32)
        o.env_h, o.env_w = scene.env.shape[0], scene.env.shape[1]
    for k in range(3):
        o.cam_pos[k] = camera["position"][k]
        o.cam_ld[k] = camera["left_down"][k]
        o.cam_du[k] = camera["du"][k]
        o.cam_dv[k] = camera["dv"][k]
    o.width, o.height = w, h
    o.max_bounces = int(scene.max_bounces if max_bounces is None else max_bounces)
    o.rr = float(scene.rr if rr is None else rr)
    o.rr_start = rr_start
    o.seed = seed
    texs = [np.ascontiguousarray(t, dtype=np.uint8) for t in getattr(scene, "textures", [])]
    if texs:
        keep.extend(texs)
        ptrs = (C.c_void_p * len(texs))(*[t.ctypes.data for t in texs])
        tw = np.array([t.shape[1] for t in texs], np.int32)
        th = np.array([t.shape[0] for t in texs], np.int32)
        keep.extend([ptrs, tw, th])
        o.ntex = len(texs)
        o.tex = C.addressof(ptrs)
        o.tex_w, o.tex_h = tw.ctypes.data, th.ctypes.data
    d = np.zeros((h, w, 4), np.float32)
    i = np.zeros((h, w, 4), np.float32)
    q = np.zeros((h, w, 4), np.float32)
    oracle_lib().oracle_render(C.byref(o), first_sample, spp, d.ctypes.data, i.ctypes.data, q.ctypes.data, nthreads)
    return d, i, q


def env_tables(env):
    e = np.ascontiguousarray(env, dtype=np.float32)
    h, w = e.shape[:2]
    u = np.zeros(w * h, np.float32)
    v = np.zeros(h, np.float32)
    ra = np.zeros(2 * h, np.float32)
    ca = np.zeros(2 * w * h, np.float32)
    oracle_lib().oracle_env_tables(e.ctypes.data, w, h, u.ctypes.data, v.ctypes.data, ra.ctypes.data, ca.ctypes.data)
    return u, v, ra, ca


def oracle_lib() -> C.CDLL:
    global _oracle
    if _oracle is None:
        L = C.CDLL(ORACLE_SO)
        L.oracle_trace_brute.argtypes = [_VP, C.c_long, _VP, C.c_long, _VP, C.c_int]
        L.oracle_trace_fp64.argtypes = [_VP, C.c_long, _VP, C.c_long, _VP, _VP, C.c_int]
        L.oracle_visible.argtypes = [_VP, C.c_long, _VP, C.c_long, _VP, C.c_int]
        L.oracle_tri_isect.argtypes = [_VP, _VP, _VP, C.c_float, _VP, _VP, _VP]
        L.oracle_render.argtypes = [C.POINTER(_OracleSceneC), C.c_int, C.c_int, _VP, _VP, _VP, C.c_int]
        L.oracle_env_tables.argtypes = [_VP, C.c_int, C.c_int, _VP, _VP, _VP, _VP]
        _oracle = L
    return _oracle


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def ref_lib() -> C.CDLL:
    global _ref
    if _ref is None:
        L = C.CDLL(REF_SO)
        L.ref_scene_from_triangles.restype = _VP
        L.ref_scene_from_triangles.argtypes = [_VP, C.c_long]
        L.ref_scene_free.argtypes = [_VP]
        L.ref_bvh_stats.argtypes = [_VP, _VP, _VP]
        L.ref_trace_closest.argtypes = [_VP, _VP, C.c_long, _VP, C.c_int]
        L.ref_visible.argtypes = [_VP, _VP, C.c_long, _VP, C.c_int]
        _ref = L
    return _ref


def _f32(a, cols):
    return np.ascontiguousarray(a, dtype=np.float32).reshape(-1, cols)


def trace_brute(tris, rays, nthreads: int = 0) -> np.ndarray:
    t, r = _f32(tris, 9), _f32(rays, 8)
    out = np.empty((r.shape[0], 4), dtype=np.float32)
    oracle_lib().oracle_trace_brute(t.ctypes.data, t.shape[0], r.ctypes.data, r.shape[0], out.ctypes.data, nthreads)
    return out


def trace_fp64(tris, rays, nthreads: int = 0):
    t, r = _f32(tris, 9), _f32(rays, 8)
    out_t = np.empty(r.shape[0], dtype=np.float64)
    out_p = np.empty(r.shape[0], dtype=np.int32)
    oracle_lib().oracle_trace_fp64(t.ctypes.data, t.shape[0], r.ctypes.data, r.shape[0], out_t.ctypes.data,
                                   out_p.ctypes.data, nthreads)
    return out_t, out_p


def visible(tris, queries, nthreads: int = 0) -> np.ndarray:
    t, q = _f32(tris, 9), _f32(queries, 12)
    out = np.empty(q.shape[0], dtype=np.uint8)
    oracle_lib().oracle_visible(t.ctypes.data, t.shape[0], q.ctypes.data, q.shape[0], out.ctypes.data, nthreads)
    return out


def tri_isect(tri, o, d, closest=np.float32(1e8)):
    v = _f32(tri, 9)
    oo = np.ascontiguousarray(o, dtype=np.float32)
    dd = np.ascontiguousarray(d, dtype=np.float32)
    t, b1, b2 = C.c_float(), C.c_float(), C.c_float()
    ok = oracle_lib().oracle_tri_isect(v.ctypes.data, oo.ctypes.data, dd.ctypes.data, C.c_float(closest),
                                       C.byref(t), C.byref(b1), C.byref(b2))
    return bool(ok), t.value, b1.value, b2.value


class _quiet_stdout:
    """Silences file descriptor 1 while the reference's code prints progress
    (its BVH build and destructor write to stdout)."""

    def __enter__(self):
        import sys

        sys.stdout.flush()
        self._saved = os.dup(1)
        self._null = os.open(os.devnull, os.O_WRONLY)
        os.dup2(self._null, 1)

    def __exit__(self, *exc):
        C.CDLL(None).fflush(None)
        os.dup2(self._saved, 1)
        os.close(self._saved)
        os.close(self._null)


class RefScene:
    """The reference's own BVH (host-compiled) over a triangle soup."""

    def __init__(self, tris):
        self.tris = _f32(tris, 9)
        with _quiet_stdout():
            self._h = ref_lib().ref_scene_from_triangles(self.tris.ctypes.data, self.tris.shape[0])

    def stats(self):
        n, d = C.c_int(), C.c_int()
        ref_lib().ref_bvh_stats(self._h, C.byref(n), C.byref(d))
        return n.value, d.value

    def trace_closest(self, rays, nthreads: int = 0) -> np.ndarray:
        r = _f32(rays, 8)
        out = np.empty((r.shape[0], 4), dtype=np.float32)
        ref_lib().ref_trace_closest(self._h, r.ctypes.data, r.shape[0], out.ctypes.data, nthreads)
        return out

    def visible(self, queries, nthreads: int = 0) -> np.ndarray:
        q = _f32(queries, 12)
        out = np.empty(q.shape[0], dtype=np.uint8)
        ref_lib().ref_visible(self._h, q.ctypes.data, q.shape[0], out.ctypes.data, nthreads)
        return out

    def close(self):
        if self._h:
            with _quiet_stdout():
                ref_lib().ref_scene_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_refcuda = {}


def ref_cuda_available(lto: bool = False) -> bool:
    return os.path.exists(REF_CUDA_LTO_SO if lto else REF_CUDA_SO)


def ref_cuda_lib(lto: bool = False) -> C.CDLL:
    """The reference's traversal built for the GPU: -rdc, or (lto) with
    device link-time optimisation."""
    if lto not in _refcuda:
        L = C.CDLL(REF_CUDA_LTO_SO if lto else REF_CUDA_SO)
        L.refcuda_scene_from_triangles.restype = _VP
        L.refcuda_scene_from_triangles.argtypes = [_VP, C.c_long]
        L.refcuda_scene_free.argtypes = [_VP]
        L.refcuda_trace.argtypes = [_VP, _VP, C.c_long, _VP, _VP]
        L.refcuda_visible.argtypes = [_VP, _VP, C.c_long, _VP, _VP]
        _refcuda[lto] = L
    return _refcuda[lto]


class RefCudaScene:
    """The reference's own traversal compiled for the GPU (headless build):
    host BVH build + CreateBVH upload, one thread per ray calling
    BVH::IsIntersect / Light::Visible. Device pointers in, stream-ordered.
    lto selects the device-LTO build."""

    def __init__(self, tris, lto: bool = False):
        self.tris = _f32(tris, 9)
        self._lib = ref_cuda_lib(lto)
        with _quiet_stdout():
            self._h = self._lib.refcuda_scene_from_triangles(self.tris.ctypes.data, self.tris.shape[0])

    def trace(self, d_rays: int, n: int, d_out: int, stream: int = 0) -> None:
        rc = self._lib.refcuda_trace(self._h, d_rays, n, d_out, stream)
        if rc:
            raise RuntimeError(f"reference CUDA trace failed: cudaError {rc}")

    def visible(self, d_q: int, n: int, d_occ: int, stream: int = 0) -> None:
        rc = self._lib.refcuda_visible(self._h, d_q, n, d_occ, stream)
        if rc:
            raise RuntimeError(f"reference CUDA visible failed: cudaError {rc}")

    def close(self):
        if self._h:
            with _quiet_stdout():
                self._lib.refcuda_scene_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_refrender = {}


def ref_render_available(lto: bool = False) -> bool:
    return os.path.exists(REF_RENDER_LTO_SO if lto else REF_RENDER_SO)


def ref_render_lib(lto: bool = False) -> C.CDLL:
    """The reference's renderer and SVGF kernels built for the GPU: -rdc, or
    (lto) with device link-time optimisation."""
    if lto not in _refrender:
        L = C.CDLL(REF_RENDER_LTO_SO if lto else REF_RENDER_SO)
        L.refr_load.restype = _VP
        L.refr_load.argtypes = [C.c_char_p]
        L.refr_info.argtypes = [C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_float), _VP]
        L.refr_render.argtypes = [_VP, C.c_int, C.c_int, _VP, _VP, _VP, C.POINTER(C.c_float)]
        L.refr_svgf.argtypes = [C.c_int, C.c_int, C.c_int, _VP, _VP, _VP, _VP, _VP, _VP, C.c_int, C.c_float,
                                C.c_float, C.c_float, C.c_float, C.c_int, _VP, _VP, _VP]
        _refrender[lto] = L
    return _refrender[lto]


class RefRenderer:
    """The reference's own renderer, built headless for the GPU: its scene
    loader (Scene::Scene) and the non-denoised RenderLoop frame body, one
    sample per pixel per frame with its curand sampler (seed 1234). One
    scene per process (the reference keeps its scene in global state)."""

    def __init__(self, json_path: str, lto: bool = False):
        self._lib = ref_render_lib(lto)
        with _quiet_stdout():
            self._h = self._lib.refr_load(str(json_path).encode())
        if not self._h:
            raise RuntimeError(f"reference failed to load {json_path}")
        w, h, mb, rr = C.c_int(), C.c_int(), C.c_int(), C.c_float()
        cam = (C.c_float * 12)()
        self._lib.refr_info(C.byref(w), C.byref(h), C.byref(mb), C.byref(rr), cam)
        self.width, self.height, self.max_bounces, self.rr = w.value, h.value, mb.value, rr.value
        c = list(cam)
        self.camera = {"position": c[0:3], "left_down": c[3:6], "du": c[6:9], "dv": c[9:12]}

    def render(self, spp: int, with_sumsq: bool = True, max_bounces: int = 0):
        """Returns (direct, indirect, sumsq or None, ms): float32 (H, W, 4)
        sums over spp frames, rows bottom-up; ms = GPU time of the frames."""
        d = np.zeros((self.height, self.width, 4), np.float32)
        i = np.zeros_like(d)
        q = np.zeros_like(d) if with_sumsq else None
        ms = C.c_float()
        with _quiet_stdout():
            rc = self._lib.refr_render(self._h, spp, max_bounces, d.ctypes.data, i.ctypes.data,
                                              q.ctypes.data if q is not None else None, C.byref(ms))
        if rc:
            raise RuntimeError(f"reference render failed: cudaError {rc}")
        return d, i, q, ms.value


def ref_svgf(noisy_d, noisy_i, pos_tri, normal_mat, bary_mesh, motion_depth, max_history=24, sigma_light=8.0,
             sigma_normal=256.0, sigma_depth=1.0, reproj=0.1, atrous=5, timing=False, lto=False):
    """The reference's SVGF kernels (headless CUDA build) over a frame
    sequence: arrays of shape (F, H, W, 4) (normal_mat / bary_mesh uint16).
    Returns (out_direct, out_indirect), float32 (F, H, W, 4), and with
    timing=True also the GPU ms of each frame's denoise block. lto selects
    the device-LTO build."""
    nd = np.ascontiguousarray(noisy_d, np.float32)
    ni = np.ascontiguousarray(noisy_i, np.float32)
    gp = np.ascontiguousarray(pos_tri, np.float32)
    gn = np.ascontiguousarray(normal_mat, np.uint16)
    gb = np.ascontiguousarray(bary_mesh, np.uint16)
    gm = np.ascontiguousarray(motion_depth, np.float32)
    f, h, w, _ = nd.shape
    od = np.zeros_like(nd)
    oi = np.zeros_like(ni)
    ms = np.zeros(f, np.float32)
    rc = ref_render_lib(lto).refr_svgf(w, h, f, nd.ctypes.data, ni.ctypes.data, gp.ctypes.data, gn.ctypes.data,
                                    gb.ctypes.data, gm.ctypes.data, max_history, sigma_light, sigma_normal,
                                    sigma_depth, reproj, atrous, od.ctypes.data, oi.ctypes.data, ms.ctypes.data)
    if rc:
        raise RuntimeError(f"reference SVGF failed: cudaError {rc}")
    return (od, oi, ms) if timing else (od, oi)
