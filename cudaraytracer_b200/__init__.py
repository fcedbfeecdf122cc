"""cudaraytracer_b200: a B200-native wavefront path tracer behind the scene /
render API of DarrenChen-CN/CudaRayTracer, exposed through the C ABI of
include/crt.h (libcrt.so, hand-written sm_100a CUDA)."""
from ._lib import CrtError, build  # noqa: F401
from .tracer import Context, Scene, Svgf, default_denoise_params, hit_prims  # noqa: F401
from . import scenes  # noqa: F401

__all__ = ["CrtError", "build", "Context", "Scene", "Svgf", "default_denoise_params", "hit_prims", "scenes"]
