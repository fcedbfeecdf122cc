"""ctypes binding of libcrt.so (the C ABI declared in include/crt.h).

The CUDA extension is the product path: there is no CPU fallback. Loading
fails loudly if libcrt.so is missing, and every call raises CrtError when the
library returns a non-zero crt_status.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import threading

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libcrt.so")

STATUS = {
    0: "CRT_OK",
    1: "CRT_ERR_INVALID",
    2: "CRT_ERR_IO",
    3: "CRT_ERR_PARSE",
    4: "CRT_ERR_CUDA",
    5: "CRT_ERR_OOM",
    6: "CRT_ERR_CAPACITY",
    7: "CRT_ERR_TIMEOUT",
}


class CrtError(RuntimeError):
    """A crt_* call returned a non-zero status."""

    def __init__(self, status: int, func: str, message: str):
        self.status = status
        self.code = STATUS.get(status, str(status))
        super().__init__(f"{func}: {self.code}: {message}")


class SceneInfo(C.Structure):
    _fields_ = [
        ("num_triangles", C.c_int64),
        ("num_bvh_nodes", C.c_int64),
        ("bvh_depth", C.c_int32),
        ("num_meshes", C.c_int32),
        ("num_materials", C.c_int32),
        ("num_lights", C.c_int32),
        ("bounds_min", C.c_float * 3),
        ("bounds_max", C.c_float * 3),
        ("build_ms", C.c_float),
        ("width", C.c_int32),
        ("height", C.c_int32),
        ("spp", C.c_int32),
        ("max_bounces", C.c_int32),
        ("rr", C.c_float),
        ("fovy", C.c_float),
        ("denoise", C.c_int32),
        ("has_env", C.c_int32),
        ("num_wide_nodes", C.c_int64),
        ("wide_depth", C.c_int32),
        ("wide_build_ms", C.c_float),
    ]


class RenderParams(C.Structure):
    _fields_ = [
        ("width", C.c_int32),
        ("height", C.c_int32),
        ("spp", C.c_int32),
        ("max_bounces", C.c_int32),
        ("rr", C.c_float),
        ("rr_start_bounce", C.c_int32),
        ("seed", C.c_uint64),
        ("spp_per_pass", C.c_int32),
        ("paths_per_pass", C.c_int32),
        ("stage_block", C.c_int32),
        ("stage_traversal", C.c_int32),
    ]


class Camera(C.Structure):
    _fields_ = [
        ("target", C.c_float * 3),
        ("distance", C.c_float),
        ("theta_deg", C.c_float),
        ("phi_deg", C.c_float),
        ("fovy_deg", C.c_float),
        ("position", C.c_float * 3),
        ("u", C.c_float * 3),
        ("v", C.c_float * 3),
        ("w", C.c_float * 3),
        ("du", C.c_float * 3),
        ("dv", C.c_float * 3),
        ("left_down", C.c_float * 3),
    ]


class GBuffer(C.Structure):
    _fields_ = [("pos_tri", C.c_void_p), ("normal_mat", C.c_void_p), ("bary_mesh", C.c_void_p),
                ("motion_depth", C.c_void_p)]


class DenoiseParams(C.Structure):
    _fields_ = [
        ("max_history_length", C.c_int32),
        ("sigma_light", C.c_float),
        ("sigma_normal", C.c_float),
        ("sigma_depth", C.c_float),
        ("reprojection_depth_factor", C.c_float),
        ("atrous_iterations", C.c_int32),
    ]


class MaterialDesc(C.Structure):
    _fields_ = [
        ("type", C.c_int32),
        ("basecolor", C.c_float * 3),
        ("emission", C.c_float * 3),
        ("roughness", C.c_float),
        ("metallic", C.c_float),
        ("transmission", C.c_float),
        ("scatter_distance", C.c_float * 3),
        ("ior", C.c_float),
        ("texture", C.c_int32),
    ]


class TextureDesc(C.Structure):
    _fields_ = [("width", C.c_int32), ("height", C.c_int32), ("rgba", C.c_void_p)]


class MeshDesc(C.Structure):
    _fields_ = [("material", C.c_int32), ("first", C.c_int32), ("count", C.c_int32)]


class LightDesc(C.Structure):
    _fields_ = [("type", C.c_int32), ("mesh", C.c_int32), ("emission", C.c_float * 3)]


class SceneDesc(C.Structure):
    _fields_ = [
        ("n_tris", C.c_int64),
        ("verts", C.c_void_p),
        ("normals", C.c_void_p),
        ("uvs", C.c_void_p),
        ("n_meshes", C.c_int32),
        ("n_materials", C.c_int32),
        ("n_lights", C.c_int32),
        ("meshes", C.c_void_p),
        ("materials", C.c_void_p),
        ("lights", C.c_void_p),
        ("env_width", C.c_int32),
        ("env_height", C.c_int32),
        ("env_rgba", C.c_void_p),
        ("n_textures", C.c_int32),
        ("textures", C.c_void_p),
        ("width", C.c_int32),
        ("height", C.c_int32),
        ("spp", C.c_int32),
        ("max_bounces", C.c_int32),
        ("rr", C.c_float),
        ("fovy", C.c_float),
        ("direction", C.c_float * 3),
    ]


class ServerConfig(C.Structure):
    _fields_ = [
        ("hbm_budget_bytes", C.c_int64),
        ("paths_per_pass", C.c_int32),
        ("max_requests", C.c_int32),
        ("passes_in_flight", C.c_int32),
        ("schedule", C.c_int32),
    ]


class Request(C.Structure):
    _fields_ = [
        ("scene", C.c_int32),
        ("width", C.c_int32),
        ("height", C.c_int32),
        ("spp", C.c_int32),
        ("max_bounces", C.c_int32),
        ("rr", C.c_float),
        ("rr_start_bounce", C.c_int32),
        ("seed", C.c_uint64),
        ("camera", Camera),
    ]


class ServerStats(C.Structure):
    _fields_ = [(k, C.c_int64) for k in ("queued", "running", "done", "passes", "paths", "bytes_budget",
                                         "bytes_scenes", "bytes_wavefront", "bytes_requests", "bytes_pool")] + [
        ("num_scenes", C.c_int32), ("passes_in_flight", C.c_int32)]


def build(force: bool = False) -> None:
    """Compiles libcrt.so in-tree with nvcc for sm_100a (make in csrc/)."""
    csrc = os.path.join(_HERE, "csrc")
    cmd = ["make", "-C", csrc, "-j", str(max(1, os.cpu_count() or 1))]
    if force:
        subprocess.run(["make", "-C", csrc, "clean"], check=True, capture_output=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("building libcrt.so failed:\n" + r.stdout[-4000:] + r.stderr[-4000:])


_lib = None
_lock = threading.Lock()

_VP = C.c_void_p
_SIGS = {
    "crt_create": (C.c_int, [C.c_int, C.POINTER(_VP)]),
    "crt_destroy": (None, [_VP]),
    "crt_last_error": (C.c_char_p, []),
    "crt_version": (C.c_char_p, []),
    "crt_scene_from_triangles": (C.c_int, [_VP, _VP, C.c_int64, C.POINTER(_VP)]),
    "crt_scene_free": (None, [_VP]),
    "crt_scene_info": (C.c_int, [_VP, C.POINTER(SceneInfo)]),
    "crt_scene_load_json": (C.c_int, [_VP, C.c_char_p, C.POINTER(_VP)]),
    "crt_scene_from_arrays": (C.c_int, [_VP, C.POINTER(SceneDesc), C.POINTER(_VP)]),
    "crt_image_decode": (C.c_int, [C.c_char_p, C.POINTER(C.c_int32), C.POINTER(C.c_int32), _VP]),
    "crt_scene_export_geometry": (C.c_int, [_VP, _VP, _VP, _VP, _VP]),
    "crt_scene_export_tables": (C.c_int, [_VP, _VP, _VP, _VP]),
    "crt_get_render_params": (C.c_int, [_VP, C.POINTER(RenderParams)]),
    "crt_set_render_params": (C.c_int, [_VP, C.POINTER(RenderParams)]),
    "crt_get_camera": (C.c_int, [_VP, C.POINTER(Camera)]),
    "crt_set_camera_orbit": (C.c_int, [_VP, C.POINTER(Camera)]),
    "crt_render": (C.c_int, [_VP, C.c_int32, _VP, _VP, _VP]),
    "crt_render_device": (C.c_int, [_VP, C.c_int32, C.c_int32, _VP, _VP, _VP, _VP]),
    "crt_render_device_noalloc": (C.c_int, [_VP, C.c_int32, C.c_int32, _VP, _VP, _VP, _VP]),
    "crt_render_views": (C.c_int, [_VP, C.c_int32, _VP, C.c_int32, C.c_int32, _VP, _VP, _VP, C.c_int32, _VP]),
    "crt_gather": (C.c_int, [_VP, C.c_int32, C.c_int32, C.c_int32, _VP, _VP, C.POINTER(GBuffer), _VP, _VP]),
    "crt_server_create": (C.c_int, [_VP, C.POINTER(ServerConfig), C.POINTER(_VP)]),
    "crt_server_free": (None, [_VP]),
    "crt_server_add_scene": (C.c_int, [_VP, _VP, C.POINTER(C.c_int32)]),
    "crt_server_submit": (C.c_int, [_VP, C.POINTER(Request), C.POINTER(C.c_int64)]),
    "crt_server_step": (C.c_int, [_VP, C.c_int32, C.POINTER(C.c_int32)]),
    "crt_server_poll": (C.c_int, [_VP, C.c_int64, C.POINTER(C.c_int32)]),
    "crt_server_result": (C.c_int, [_VP, C.c_int64, _VP, _VP]),
    "crt_server_result_device": (C.c_int, [_VP, C.c_int64, C.POINTER(_VP), C.POINTER(_VP)]),
    "crt_server_release": (C.c_int, [_VP, C.c_int64]),
    "crt_server_get_stats": (C.c_int, [_VP, C.POINTER(ServerStats)]),
    "crt_denoise_params_default": (C.c_int, [C.POINTER(DenoiseParams)]),
    "crt_gbuffer_from_primary": (C.c_int, [_VP, C.POINTER(Camera), C.POINTER(GBuffer), _VP]),
    "crt_svgf_create": (C.c_int, [_VP, C.c_int32, C.c_int32, C.POINTER(_VP)]),
    "crt_svgf_free": (None, [_VP]),
    "crt_svgf_reset": (C.c_int, [_VP]),
    "crt_svgf_frame": (C.c_int, [_VP, C.POINTER(DenoiseParams), C.POINTER(GBuffer), C.POINTER(GBuffer), _VP, _VP,
                                 _VP, _VP, _VP]),
    "crt_render_svgf_frame": (C.c_int, [_VP, _VP, C.POINTER(DenoiseParams), C.c_int32, _VP, _VP, _VP]),
    "crt_conv3x3_forward": (C.c_int, [_VP, _VP, C.c_int32, C.c_int32, C.c_int32, C.c_int32, _VP, _VP, C.c_int32,
                                      C.c_int32, _VP, _VP, _VP]),
    "crt_conv3x3_backward_data": (C.c_int, [_VP, _VP, C.c_int32, C.c_int32, C.c_int32, C.c_int32, _VP, C.c_int32,
                                            _VP, _VP, _VP]),
    "crt_conv3x3_backward_weights": (C.c_int, [_VP, _VP, _VP, C.c_int32, C.c_int32, C.c_int32, C.c_int32,
                                               C.c_int32, _VP, _VP]),
    "crt_check_device_errors": (C.c_int, [_VP]),
    "crt_kpcn_create": (C.c_int, [_VP, C.c_uint64, C.POINTER(_VP)]),
    "crt_kpcn_free": (None, [_VP]),
    "crt_kpcn_num_params": (C.c_int, [_VP, C.POINTER(C.c_int64)]),
    "crt_kpcn_get_params": (C.c_int, [_VP, _VP]),
    "crt_kpcn_set_params": (C.c_int, [_VP, _VP]),
    "crt_kpcn_get_grads": (C.c_int, [_VP, _VP]),
    "crt_kpcn_features": (C.c_int, [_VP, C.POINTER(GBuffer), _VP, _VP, C.c_int32, C.c_int64, C.c_float, _VP, _VP,
                                    _VP]),
    "crt_kpcn_forward": (C.c_int, [_VP, C.c_int32, C.c_int32, C.c_int32, _VP, _VP, _VP, _VP]),
    "crt_kpcn_train_step": (C.c_int, [_VP, C.c_int32, C.c_int32, C.c_int32, _VP, _VP, _VP, C.c_float,
                                      C.POINTER(C.c_float), _VP]),
    "crt_kpcn_debug_tensor": (C.c_int, [_VP, C.c_int32, _VP, C.c_int64]),
    "crt_trace_closest": (C.c_int, [_VP, _VP, C.c_int64, _VP]),
    "crt_trace_closest_device": (C.c_int, [_VP, _VP, C.c_int64, _VP, _VP]),
    "crt_trace_shadow": (C.c_int, [_VP, _VP, C.c_int64, _VP]),
    "crt_trace_shadow_device": (C.c_int, [_VP, _VP, C.c_int64, _VP, _VP]),
    "crt_scene_ray_counts": (C.c_int, [_VP, _VP, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
    "crt_bvh8_collapse": (C.c_int, [_VP, C.c_int64, _VP, _VP, C.POINTER(C.c_int64), C.POINTER(C.c_int32)]),
}


def lib() -> C.CDLL:
    """Loads libcrt.so (raises if it has not been built)."""
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise RuntimeError(
                    f"{LIB_PATH} is missing: run cudaraytracer_b200._lib.build() "
                    "(or __graft_entry__.build()); there is no CPU fallback"
                )
            L = C.CDLL(LIB_PATH)
            for name, (res, args) in _SIGS.items():
                f = getattr(L, name)
                f.restype = res
                f.argtypes = args
            _lib = L
        return _lib


def check(status: int, func: str) -> None:
    if status != 0:
        msg = lib().crt_last_error()
        raise CrtError(status, func, msg.decode() if msg else "")


def call(name: str, *args) -> None:
    check(getattr(lib(), name)(*args), name)
