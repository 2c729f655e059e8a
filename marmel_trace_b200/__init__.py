"""marmel_trace_b200 - B200 (sm_100a) renderer core for marmel-trace scenes.

The product is libmtgpu.so (C ABI in include/mtgpu.h). This package builds
it (``build``), loads it with ctypes (``_capi``), mirrors the reference's
render entry points on top of it (``api``) and generates the seeded synthetic
benchmark scenes (``scenes``).
"""
from . import _capi  # noqa: F401
from .api import (  # noqa: F401
    Camera,
    GpuScene,
    SceneDesc,
    camera_create,
    default_sky,
    normalize,
    pathtrace_radiance,
    pathtrace_render,
    render_image,
    render_image_ex,
)

__all__ = [
    "Camera",
    "GpuScene",
    "SceneDesc",
    "camera_create",
    "default_sky",
    "normalize",
    "pathtrace_radiance",
    "pathtrace_render",
    "render_image",
    "render_image_ex",
]
