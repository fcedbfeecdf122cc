"""Host-side mirror of the reference's scene/query API over libcrt.so.

* Context            - device + stream (the reference's implicit device 0).
* Scene.from_triangles - geometry + device BVH (BVH::BVH/CreateBVH,
                       Src/Core/bvh.cu:9,308).
* Scene.trace_closest  - BVH::IsIntersect (Src/Core/bvh.cu:253).
* Scene.trace_shadow   - Light::Visible (Src/Core/light.cu:5).

Arguments may be numpy arrays (host path: the library copies in and out,
pipelined in chunks) or CUDA torch tensors (device path, no copies).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib


def _is_cuda_tensor(x) -> bool:
    return getattr(x, "is_cuda", False)


def _torch_stream(device, stream=None) -> int:
    """cudaStream_t of `stream` (or torch's current stream). Torch's default
    stream has handle 0, which the C ABI reads as "the context's own stream",
    so it is passed as cudaStreamLegacy (1) instead."""
    import torch

    s = stream if stream is not None else torch.cuda.current_stream(device).cuda_stream
    s = int(getattr(s, "cuda_stream", s))
    return s if s != 0 else 1


class Context:
    """A crt_ctx bound to one CUDA device."""

    def __init__(self, device: int = 0):
        self._h = C.c_void_p()
        _lib.call("crt_create", int(device), C.byref(self._h))
        self.device = device

    @property
    def handle(self):
        return self._h

    def close(self):
        if self._h:
            _lib.lib().crt_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Scene:
    """A scene resident on the device (geometry + BVH [+ materials/lights])."""

    def __init__(self, ctx: Context, handle: C.c_void_p):
        self.ctx = ctx
        self._h = handle

    @classmethod
    def from_triangles(cls, ctx: Context, tris: np.ndarray) -> "Scene":
        t = np.ascontiguousarray(tris, dtype=np.float32).reshape(-1, 9)
        h = C.c_void_p()
        _lib.call("crt_scene_from_triangles", ctx.handle, t.ctypes.data, int(t.shape[0]), C.byref(h))
        return cls(ctx, h)

    @property
    def handle(self):
        return self._h

    def info(self) -> dict:
        si = _lib.SceneInfo()
        _lib.call("crt_scene_info", self._h, C.byref(si))
        out = {}
        for name, _ in si._fields_:
            v = getattr(si, name)
            out[name] = list(v) if hasattr(v, "__len__") else v
        return out

    def close(self):
        if self._h:
            _lib.lib().crt_scene_free(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- queries -----------------------------------------------------------

    def trace_closest(self, rays, hits=None, stream=None):
        """Closest hits of rays (n, 8) float32 [o, tmin, d, tmax].
        Returns (n, 4) float32 [t, prim (int32 bits), b1, b2]."""
        if _is_cuda_tensor(rays):
            import torch

            n = rays.shape[0]
            if hits is None:
                hits = torch.empty((n, 4), dtype=torch.float32, device=rays.device)
            s = _torch_stream(rays.device, stream)
            _lib.call("crt_trace_closest_device", self._h, rays.data_ptr(), int(n), hits.data_ptr(), C.c_void_p(s))
            return hits
        r = np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 8)
        out = np.empty((r.shape[0], 4), dtype=np.float32) if hits is None else hits
        _lib.call("crt_trace_closest", self._h, r.ctypes.data, int(r.shape[0]), out.ctypes.data)
        return out

    def trace_shadow(self, queries, occluded=None, stream=None):
        """Light::Visible for queries (n, 12) float32 [p, n, light p, light n].
        Returns (n,) uint8, 1 = occluded."""
        if _is_cuda_tensor(queries):
            import torch

            n = queries.shape[0]
            if occluded is None:
                occluded = torch.empty((n,), dtype=torch.uint8, device=queries.device)
            s = _torch_stream(queries.device, stream)
            _lib.call("crt_trace_shadow_device", self._h, queries.data_ptr(), int(n), occluded.data_ptr(),
                      C.c_void_p(s))
            return occluded
        q = np.ascontiguousarray(queries, dtype=np.float32).reshape(-1, 12)
        out = np.empty((q.shape[0],), dtype=np.uint8) if occluded is None else occluded
        _lib.call("crt_trace_shadow", self._h, q.ctypes.data, int(q.shape[0]), out.ctypes.data)
        return out


def hit_prims(hits: np.ndarray) -> np.ndarray:
    """Primitive ids (int32) stored in column 1 of a hit array."""
    return np.ascontiguousarray(hits[:, 1]).view(np.int32)
