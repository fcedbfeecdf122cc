"""Host-side mirror of the reference's scene/query API over libcrt.so.

* Context            - device + stream (the reference's implicit device 0).
* Scene.from_triangles - geometry + device BVH (BVH::BVH/CreateBVH,
                       Src/Core/bvh.cu:9,308).
* Scene.trace_closest  - BVH::IsIntersect (Src/Core/bvh.cu:253).
* Scene.trace_shadow   - Light::Visible (Src/Core/light.cu:5).
* Scene.load           - Scene::Scene(jsonPath) (Src/Core/scene.cpp:50).
* Scene.from_spec      - the same scene built from generator arrays.
* Scene.render         - the non-denoised progressive frame loop of
                         Renderer::RenderLoop (Src/Core/renderer.cuh:1144-1193)
                         returning the float accumulators.

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
    """A crt_ctx bound to one CUDA device. Objects created on it (scenes,
    servers, SVGF states, denoiser networks) register here and are closed
    before the context, so none outlives the crt_ctx it points to."""

    def __init__(self, device: int = 0):
        import weakref

        self._h = C.c_void_p()
        _lib.call("crt_create", int(device), C.byref(self._h))
        self.device = device
        self._children = weakref.WeakSet()

    @property
    def handle(self):
        return self._h

    def _adopt(self, obj):
        if not self._h:
            raise RuntimeError("context is closed")
        self._children.add(obj)

    def check_device_errors(self) -> None:
        """Synchronises and raises CrtError if a kernel of this context
        recorded a device-side error since the last check (a BVH traversal
        that met an index outside its tree, or a tensor-core kernel that gave
        up a bounded wait)."""
        _lib.call("crt_check_device_errors", self._h)

    def close(self):
        if self._h:
            # servers first: they reference scenes
            kids = sorted(list(self._children), key=lambda o: 0 if type(o).__name__ == "Server" else 1)
            for obj in kids:
                try:
                    obj.close()
                except Exception:
                    pass
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
        ctx._adopt(self)

    @classmethod
    def from_triangles(cls, ctx: Context, tris: np.ndarray) -> "Scene":
        t = np.ascontiguousarray(tris, dtype=np.float32).reshape(-1, 9)
        h = C.c_void_p()
        _lib.call("crt_scene_from_triangles", ctx.handle, t.ctypes.data, int(t.shape[0]), C.byref(h))
        return cls(ctx, h)

    @classmethod
    def load(cls, ctx: Context, path: str) -> "Scene":
        """Loads a scene JSON (reference schema) with its OBJ / HDR assets."""
        h = C.c_void_p()
        _lib.call("crt_scene_load_json", ctx.handle, str(path).encode(), C.byref(h))
        return cls(ctx, h)

    @classmethod
    def from_spec(cls, ctx: Context, spec) -> "Scene":
        """Builds a generated scene (cudaraytracer_b200.scenes.SceneSpec)
        from memory through crt_scene_from_arrays: the scene that
        Scene.load(spec.write(...)) builds, without writing OBJ/HDR files.
        Material fields take the defaults of the JSON schema
        (Src/Core/scene.cpp:283-378), an area light takes its emission from
        its material's ke (or its own "ke"), and the environment image goes
        through the Radiance RGBE quantisation its .hdr file would apply."""
        from .scenes import decode_hdr_rgbe

        cam = spec.camera
        mats = _lib.MaterialDesc * len(spec.materials)
        md = mats()
        index = {}
        tex_names = list(getattr(spec, "textures", {}) or {})
        tex_imgs = [np.ascontiguousarray(spec.textures[n], dtype=np.uint8) for n in tex_names]
        for i, m in enumerate(spec.materials):
            d = md[i]
            t = {"light": 0, "diffuse": 1, "pbr": 2, "dielectric": 3, "glass": 3, "subsurface": 4}[m["type"]]
            d.type = t
            base = [0.0, 0.0, 0.0]
            ke = [0.0, 0.0, 0.0]
            scatter = [0.0, 0.0, 0.0]
            rough, metal, trans, ior = 0.5, 0.0, 1.0, 1.0
            if t in (1, 2, 4) and "basecolor" in m:
                base = m["basecolor"]
            if t == 0 and "emission" in m:
                ke = m["emission"]
            if t == 2:
                metal = m.get("metallic", 0.0)
                rough = m.get("roughness", 0.5)
            if t == 4:
                scatter = m.get("scatter_distance", [1.0, 1.0, 1.0])
                ior = m.get("ior", ior)
                rough = m.get("roughness", rough)
                metal = 0.0
            if t == 3:
                base = m.get("basecolor", [1.0, 1.0, 1.0])
                ior = m.get("ior", 1.5)
                trans = m.get("transmission", 1.0)
                rough = m.get("roughness", 0.0)
                metal = 0.0
            for k in range(3):
                d.basecolor[k], d.emission[k], d.scatter_distance[k] = base[k], ke[k], scatter[k]
            d.roughness, d.metallic, d.transmission, d.ior = rough, metal, trans, ior
            d.texture = tex_names.index(m["diffuse_texture"]) if m.get("diffuse_texture") in tex_names else -1
            index[m["name"]] = i
        tris = [np.ascontiguousarray(m.tris, dtype=np.float32).reshape(-1, 9) for m in spec.meshes]
        verts = np.ascontiguousarray(np.concatenate(tris))
        uvs = None
        if any(getattr(m, "uvs", None) is not None for m in spec.meshes):
            uvs = np.ascontiguousarray(np.concatenate([
                np.asarray(m.uvs, dtype=np.float32).reshape(-1, 6) if getattr(m, "uvs", None) is not None
                else np.zeros((t.shape[0], 6), np.float32) for m, t in zip(spec.meshes, tris)]))
        meshes = (_lib.MeshDesc * len(tris))()
        first = 0
        mesh_index = {}
        for i, (m, t) in enumerate(zip(spec.meshes, tris)):
            meshes[i].material = index[m.material]
            meshes[i].first = first
            meshes[i].count = t.shape[0]
            first += t.shape[0]
            mesh_index[m.name] = i
        lights = (_lib.LightDesc * max(1, len(spec.lights)))()
        env = None
        for i, l in enumerate(spec.lights):
            if l["type"] == "area":
                lights[i].type = 0
                lights[i].mesh = mesh_index[l["lightMeshName"]]
                ke = l.get("ke", [0.0, 0.0, 0.0])
                if "material" in l:
                    mm = md[index[l["material"]]]
                    ke = [mm.emission[k] for k in range(3)]
                for k in range(3):
                    lights[i].emission[k] = ke[k]
            elif l["type"] == "env":
                lights[i].type = 2
                rgb = decode_hdr_rgbe(spec.env)
                env = np.ascontiguousarray(np.concatenate([rgb, np.ones(rgb.shape[:2] + (1,), np.float32)], 2))
            else:
                raise ValueError(f"unsupported light type {l['type']}")
        d = _lib.SceneDesc()
        d.n_tris = verts.shape[0]
        d.verts = verts.ctypes.data
        if uvs is not None:
            d.uvs = uvs.ctypes.data
        if tex_imgs:
            tds = (_lib.TextureDesc * len(tex_imgs))()
            for k, img in enumerate(tex_imgs):
                tds[k].height, tds[k].width = img.shape[0], img.shape[1]
                tds[k].rgba = img.ctypes.data
            d.n_textures = len(tex_imgs)
            d.textures = C.addressof(tds)
        d.n_meshes, d.n_materials, d.n_lights = len(tris), len(spec.materials), len(spec.lights)
        d.meshes = C.addressof(meshes)
        d.materials = C.addressof(md)
        d.lights = C.addressof(lights)
        if env is not None:
            d.env_height, d.env_width = env.shape[0], env.shape[1]
            d.env_rgba = env.ctypes.data
        d.width, d.height = int(cam["resolution"][0]), int(cam["resolution"][1])
        d.spp = int(cam.get("spp", 16))
        d.max_bounces = int(cam.get("max_bounces", 5))
        d.rr = float(cam.get("rr", 0.8))
        d.fovy = float(cam.get("fov", 40))
        direction = cam.get("direction", [0.0, 0.0, -1.0])
        for k in range(3):
            d.direction[k] = direction[k]
        h = C.c_void_p()
        _lib.call("crt_scene_from_arrays", ctx.handle, C.byref(d), C.byref(h))
        return cls(ctx, h)

    @property
    def handle(self):
        return self._h

    # -- render path ---------------------------------------------------------

    def render_params(self) -> dict:
        p = _lib.RenderParams()
        _lib.call("crt_get_render_params", self._h, C.byref(p))
        return {k: getattr(p, k) for k, _ in p._fields_}

    def set_render_params(self, **kw) -> None:
        p = _lib.RenderParams()
        _lib.call("crt_get_render_params", self._h, C.byref(p))
        for k, v in kw.items():
            if not hasattr(p, k):
                raise KeyError(k)
            setattr(p, k, v)
        _lib.call("crt_set_render_params", self._h, C.byref(p))

    def camera(self) -> dict:
        c = _lib.Camera()
        _lib.call("crt_get_camera", self._h, C.byref(c))
        return {k: (list(getattr(c, k)) if hasattr(getattr(c, k), "__len__") else getattr(c, k)) for k, _ in c._fields_}

    def set_camera_orbit(self, target, distance, theta_deg, phi_deg, fovy_deg) -> None:
        c = _lib.Camera()
        for k in range(3):
            c.target[k] = target[k]
        c.distance, c.theta_deg, c.phi_deg, c.fovy_deg = distance, theta_deg, phi_deg, fovy_deg
        _lib.call("crt_set_camera_orbit", self._h, C.byref(c))

    def render(self, spp: int, with_sumsq: bool = False):
        """Renders spp samples per pixel from a cleared frame. Returns float32
        (H, W, 4) sums over samples (rows bottom-up): direct, indirect and,
        if requested, the per-pixel sum of squared sample values."""
        rp = self.render_params()
        h, w = rp["height"], rp["width"]
        d = np.empty((h, w, 4), np.float32)
        i = np.empty((h, w, 4), np.float32)
        q = np.empty((h, w, 4), np.float32) if with_sumsq else None
        _lib.call("crt_render", self._h, int(spp), d.ctypes.data, i.ctypes.data, q.ctypes.data if q is not None else None)
        return (d, i, q) if with_sumsq else (d, i)

    def render_device(self, direct, indirect, spp: int, first_sample: int = 0, sumsq=None, stream=None):
        """Adds samples [first_sample, first_sample + spp) into CUDA float32
        tensors of shape (H, W, 4) (asynchronous on the current stream)."""
        s = _torch_stream(direct.device, stream)
        _lib.call("crt_render_device", self._h, int(first_sample), int(spp), direct.data_ptr(), indirect.data_ptr(),
                  sumsq.data_ptr() if sumsq is not None else None, C.c_void_p(s))

    def ray_counts(self, stream=None) -> tuple:
        """(extend rays, shadow rays) traced by this scene's wavefront
        renders since it was created (path vertices and Light::Visible
        tests; subsurface probe rays are not counted)."""
        e, s = C.c_int64(0), C.c_int64(0)
        _lib.call("crt_scene_ray_counts", self._h, C.c_void_p(stream or 0), C.byref(e), C.byref(s))
        return e.value, s.value

    def render_device_noalloc(self, direct, indirect, spp: int, first_sample: int = 0, sumsq=None, stream=None):
        """render_device without device allocation: the library's fixed
        scratch holds the path queues (at most 65,536 pixels; calls must not
        overlap on the GPU). For hosts that forbid allocation during a frame."""
        s = _torch_stream(direct.device, stream)
        _lib.call("crt_render_device_noalloc", self._h, int(first_sample), int(spp), direct.data_ptr(),
                  indirect.data_ptr(), sumsq.data_ptr() if sumsq is not None else None, C.c_void_p(s))

    def gbuffer(self, prev_camera: dict | None = None, stream=None, out: dict | None = None):
        """Primary-hit G-buffer of the current camera (motion against
        prev_camera, a dict as returned by camera()). Returns a dict of CUDA
        tensors: pos_tri (H,W,4) f32, normal_mat (H,W,4) i16 bits of uint16,
        bary_mesh (H,W,4) same, motion_depth (H,W,4) f32. Every pixel is
        written; `out` (a dict of that shape) is filled instead of new
        tensors."""
        import torch

        if out is not None:
            g = out
        else:
            rp = self.render_params()
            h, w = rp["height"], rp["width"]
            dev = torch.device("cuda", self.ctx.device)
            g = {"pos_tri": torch.empty((h, w, 4), dtype=torch.float32, device=dev),
                 "normal_mat": torch.empty((h, w, 4), dtype=torch.int16, device=dev),
                 "bary_mesh": torch.empty((h, w, 4), dtype=torch.int16, device=dev),
                 "motion_depth": torch.empty((h, w, 4), dtype=torch.float32, device=dev)}
        dev = g["pos_tri"].device
        gb = _gbuffer_struct(g)
        cam = None
        if prev_camera is not None:
            cam = _lib.Camera()
            for k in range(3):
                cam.target[k] = prev_camera["target"][k]
            cam.distance = prev_camera["distance"]
            cam.theta_deg, cam.phi_deg, cam.fovy_deg = prev_camera["theta_deg"], prev_camera["phi_deg"], \
                prev_camera["fovy_deg"]
        s = _torch_stream(dev, stream)
        _lib.call("crt_gbuffer_from_primary", self._h, C.byref(cam) if cam is not None else None, C.byref(gb),
                  C.c_void_p(s))
        return g

    def gather(self, mode: int = 0, spp: int = 1, direct=None, indirect=None, gbuffer: dict | None = None,
               denoised: bool = False, stream=None):
        """GatherKernel: the display image (mode 0) or a debug view (1 depth,
        2 normal, 3 mesh id, 4 position) as a CUDA uint8 tensor (H, W, 4)
        in the reference's display-buffer layout."""
        import torch

        rp = self.render_params()
        dev = torch.device("cuda", self.ctx.device)
        out = torch.empty((rp["height"], rp["width"], 4), dtype=torch.uint8, device=dev)
        gb = _gbuffer_struct(gbuffer) if gbuffer is not None else None
        s = _torch_stream(dev, stream)
        _lib.call("crt_gather", self._h, int(mode), int(spp), 1 if denoised else 0,
                  direct.data_ptr() if direct is not None else None,
                  indirect.data_ptr() if indirect is not None else None, C.byref(gb) if gb is not None else None,
                  out.data_ptr(), C.c_void_p(s))
        return out

    def render_svgf_frame(self, svgf: "Svgf", frame_index: int, out_direct, out_indirect, params=None,
                          stream=None) -> None:
        """The reference's denoised frame: 1 spp + G-buffer + SVGF into CUDA
        float32 tensors (H, W, 4) (rgb, variance)."""
        s = _torch_stream(out_direct.device, stream)
        p = params if params is not None else default_denoise_params()
        _lib.call("crt_render_svgf_frame", self._h, svgf.handle, C.byref(p), int(frame_index), out_direct.data_ptr(),
                  out_indirect.data_ptr(), C.c_void_p(s))

    def render_views(self, cameras, direct, indirect, spp: int, first_sample: int = 0, sumsq=None,
                     use_graph: bool = True, stream=None) -> None:
        """Batched rendering of several orbit cameras (dicts with target,
        distance, theta_deg, phi_deg, fovy_deg) into view-major CUDA float32
        tensors of shape (n_views, H, W, 4)."""
        n = len(cameras)
        arr = (_lib.Camera * n)()
        for i, c in enumerate(cameras):
            for k in range(3):
                arr[i].target[k] = c["target"][k]
            arr[i].distance = c["distance"]
            arr[i].theta_deg, arr[i].phi_deg, arr[i].fovy_deg = c["theta_deg"], c["phi_deg"], c["fovy_deg"]
        s = _torch_stream(direct.device, stream)
        _lib.call("crt_render_views", self._h, n, arr, int(first_sample), int(spp), direct.data_ptr(),
                  indirect.data_ptr(), sumsq.data_ptr() if sumsq is not None else None, 1 if use_graph else 0,
                  C.c_void_p(s))

    def export_geometry(self):
        n = self.info()["num_triangles"]
        v = np.empty((n, 9), np.float32)
        nn = np.empty((n, 9), np.float32)
        uv = np.empty((n, 6), np.float32)
        pm = np.empty((n,), np.int32)
        _lib.call("crt_scene_export_geometry", self._h, v.ctypes.data, nn.ctypes.data, uv.ctypes.data, pm.ctypes.data)
        return v, nn, uv, pm

    def export_tables(self):
        inf = self.info()
        m = np.empty((inf["num_materials"], 16), np.float32)
        me = np.empty((inf["num_meshes"], 8), np.float32)
        li = np.empty((inf["num_lights"], 8), np.float32)
        _lib.call("crt_scene_export_tables", self._h, m.ctypes.data, me.ctypes.data, li.ctypes.data)
        return m, me, li

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


def bvh8_collapse(bin_nodes: np.ndarray):
    """Collapses a binary node array ((n, 16) float32 in this library's
    two-child layout, root at 0) into the 8-wide quantised layout on the
    host. Returns (wide_nodes (m, 16) float32, wide_links (m, 8) int32,
    depth)."""
    b = np.ascontiguousarray(bin_nodes, dtype=np.float32).reshape(-1, 16)
    cnt = C.c_int64(0)
    dep = C.c_int32(0)
    _lib.call("crt_bvh8_collapse", b.ctypes.data, b.shape[0], None, None, C.byref(cnt), C.byref(dep))
    nodes = np.zeros((cnt.value, 16), np.float32)
    links = np.zeros((cnt.value, 8), np.int32)
    _lib.call("crt_bvh8_collapse", b.ctypes.data, b.shape[0], nodes.ctypes.data, links.ctypes.data, C.byref(cnt),
              C.byref(dep))
    return nodes, links, dep.value


def hit_prims(hits: np.ndarray) -> np.ndarray:
    """Primitive ids (int32) stored in column 1 of a hit array."""
    return np.ascontiguousarray(hits[:, 1]).view(np.int32)


def _gbuffer_struct(g: dict):
    gb = _lib.GBuffer()
    gb.pos_tri = g["pos_tri"].data_ptr()
    gb.normal_mat = g["normal_mat"].data_ptr()
    gb.bary_mesh = g["bary_mesh"].data_ptr()
    gb.motion_depth = g["motion_depth"].data_ptr()
    return gb


def default_denoise_params() -> "_lib.DenoiseParams":
    """DenoiseParam defaults (Src/Utils/ui.h:14-25)."""
    p = _lib.DenoiseParams()
    _lib.call("crt_denoise_params_default", C.byref(p))
    return p


class Svgf:
    """SVGF state (temporal history, moments, history lengths) for one image
    size: TemporalDenoising + ComputeVarianceKernel + AtrousKernel of the
    reference, over device buffers."""

    def __init__(self, ctx: Context, width: int, height: int):
        self.ctx = ctx
        self.width, self.height = width, height
        self._h = C.c_void_p()
        _lib.call("crt_svgf_create", ctx.handle, int(width), int(height), C.byref(self._h))
        ctx._adopt(self)

    @property
    def handle(self):
        return self._h

    def reset(self) -> None:
        _lib.call("crt_svgf_reset", self._h)

    def frame(self, cur_gbuffer: dict, prev_gbuffer: dict, noisy_direct, noisy_indirect, out_direct, out_indirect,
              params=None, stream=None) -> None:
        """One SVGF frame over CUDA float32 (H, W, 4) tensors."""
        s = _torch_stream(noisy_direct.device, stream)
        p = params if params is not None else default_denoise_params()
        cur, prev = _gbuffer_struct(cur_gbuffer), _gbuffer_struct(prev_gbuffer)
        _lib.call("crt_svgf_frame", self._h, C.byref(p), C.byref(cur), C.byref(prev), noisy_direct.data_ptr(),
                  noisy_indirect.data_ptr(), out_direct.data_ptr(), out_indirect.data_ptr(), C.c_void_p(s))

    def close(self):
        if self._h:
            _lib.lib().crt_svgf_free(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
