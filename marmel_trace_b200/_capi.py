"""ctypes mirror of include/mtgpu.h and the loader of libmtgpu.so.

The shared library is built in-tree (marmel_trace_b200/libmtgpu.so) by
``marmel_trace_b200.build``. Loading fails loudly when it is missing: there is
no Python or CPU fallback for any entry point.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "libmtgpu.so"

# Status codes (mtgpu.h)
MT_OK = 0
MT_ERR_NULL = 1
MT_ERR_DIMS = 2
MT_ERR_COUNTS = 3
MT_ERR_NO_DEVICE = 10
MT_ERR_OOM = 11
MT_ERR_LAUNCH = 12
MT_ERR_WATCHDOG = 13
MT_ERR_UNSUPPORTED = 14
MT_ERR_INVALID = 15
MT_ERR_OVERFLOW = 16

PRIM_SPHERE, PRIM_PLANE, PRIM_BOX, PRIM_TRIANGLE, PRIM_CYLINDER = 0, 1, 2, 3, 4
PRECISION_FP32, PRECISION_FP64 = 0, 1
INTEGRATOR_MEGAKERNEL, INTEGRATOR_WAVEFRONT = 0, 1
MODE_PATHTRACE, MODE_WHITTED = 0, 1

TEXTURE_NONE, TEXTURE_CHECKER, TEXTURE_STRIPES, TEXTURE_PLANET_EARTH = 0, 1, 2, 3
TEXTURE_PLANET_MOON, TEXTURE_NOISE, TEXTURE_IMAGE, TEXTURE_UV_CHECKER = 4, 5, 6, 7

# mt_prim (208 bytes) and mt_material (288 bytes) as numpy structured dtypes,
# so large primitive arrays cross the C ABI without a copy.
PRIM_DTYPE = np.dtype(
    [("kind", "<i4"), ("material", "<i4"), ("smooth", "<i4"), ("has_uv", "<i4"), ("v", "<f8", 9), ("n", "<f8", 9),
     ("uv", "<f8", 6)]
)
MATERIAL_DTYPE = np.dtype(
    [
        ("albedo", "<f8", 3),
        ("specular", "<f8", 3),
        ("shininess", "<f8"),
        ("reflectivity", "<f8"),
        ("transparency", "<f8"),
        ("ior", "<f8"),
        ("absorption", "<f8", 3),
        ("deep_color", "<f8", 3),
        ("metallic", "<f8"),
        ("roughness", "<f8"),
        ("emissive", "<f8", 3),
        ("atmosphere_glow", "<f8", 3),
        ("bump_strength", "<f8"),
        ("is_water", "<i4"),
        ("beer_lambert", "<i4"),
        ("pbr", "<i4"),
        ("texture_kind", "<i4"),
        ("texture_scale", "<f8"),
        ("texture_color_a", "<f8", 3),
        ("texture_color_b", "<f8", 3),
        ("texture_rgb", "<u8"),     # const unsigned char * (address of the image bytes, or 0)
        ("texture_width", "<i4"),
        ("texture_height", "<i4"),
    ]
)
assert PRIM_DTYPE.itemsize == 208 and MATERIAL_DTYPE.itemsize == 288

D3 = C.c_double * 3


class MtSky(C.Structure):
    _fields_ = [
        ("sun_dir", D3),
        ("sun_color", D3),
        ("horizon_color", D3),
        ("zenith_color", D3),
        ("gradient_gamma", C.c_double),
        ("sun_glow_exponent", C.c_double),
        ("sun_glow_strength", C.c_double),
        ("cloud_height", C.c_double),
        ("cloud_scale", C.c_double),
        ("cloud_coverage", C.c_double),
        ("cloud_softness", C.c_double),
        ("cloud_sharpness", C.c_double),
        ("cloud_thickness", C.c_double),
        ("sun_radius", C.c_double),
        ("star_intensity", C.c_double),
        ("nebula_intensity", C.c_double),
        ("galaxy_intensity", C.c_double),
        ("cloud_octaves", C.c_int32),
        ("seed", C.c_uint32),
        ("cloud_density", C.c_double),
        ("cloud_steps", C.c_int32),
        ("reserved", C.c_int32),
    ]


class MtOcean(C.Structure):
    _fields_ = [
        ("enabled", C.c_int32),
        ("seed", C.c_uint32),
        ("center", D3),
        ("amplitude", C.c_double),
        ("wavelength", C.c_double),
        ("direction", D3),
        ("chop", C.c_double),
        ("chop_wavelength", C.c_double),
    ]


class MtSceneDesc(C.Structure):
    _fields_ = [
        ("prims", C.c_void_p),
        ("prim_count", C.c_int32),
        ("material_count", C.c_int32),
        ("materials", C.c_void_p),
        ("sky", MtSky),
        ("fog_density", C.c_double),
        ("water_level", C.c_double),
        ("water_material", C.c_int32),
        ("fog_shadow_steps", C.c_int32),
        ("ocean", MtOcean),
        ("fog_color", D3),
        ("fog_height", C.c_double),
        ("fog_height_falloff", C.c_double),
        ("fog_inscatter_strength", C.c_double),
        ("fog_sun_anisotropy", C.c_double),
        ("fog_noise_scale", C.c_double),
        ("fog_noise_amount", C.c_double),
    ]


class MtCamera(C.Structure):
    _fields_ = [
        ("position", D3),
        ("lower_left", D3),
        ("horizontal", D3),
        ("vertical", D3),
        ("aperture", C.c_double),
        ("focus_distance", C.c_double),
        ("dome_radius", C.c_double),
        ("anamorphic_squeeze", C.c_double),
    ]


class MtRenderParams(C.Structure):
    _fields_ = [
        ("samples_per_pixel", C.c_int32),
        ("max_depth", C.c_int32),
        ("adaptive", C.c_int32),
        ("adaptive_max_spp", C.c_int32),
        ("adaptive_tau", C.c_double),
    ]


class MtOptions(C.Structure):
    _fields_ = [
        ("precision", C.c_int32),
        ("integrator", C.c_int32),
        ("block_size", C.c_int32),
        ("queue_capacity", C.c_int32),
        ("bvh_width", C.c_int32),
        ("sort_threshold", C.c_int32),
        ("use_graph", C.c_int32),
        ("device", C.c_int32),
        ("traversal", C.c_int32),
        ("bvh_builder", C.c_int32),
        ("occluder_cache", C.c_int32),
    ]


class MtTuneEntry(C.Structure):
    _fields_ = [("options", MtOptions), ("ms", C.c_float), ("pad", C.c_float)]


class MtTuneReport(C.Structure):
    _fields_ = [("chosen", MtOptions), ("chosen_ms", C.c_float), ("default_ms", C.c_float),
                ("n_entries", C.c_int32), ("pad", C.c_int32), ("entries", MtTuneEntry * 32)]


class MtBatchItem(C.Structure):
    _fields_ = [
        ("scene", C.c_void_p),
        ("cam", C.c_void_p),
        ("width", C.c_int32),
        ("height", C.c_int32),
        ("s0", C.c_int32),
        ("spp", C.c_int32),
        ("depth", C.c_int32),
        ("pad", C.c_int32),
        ("out_dev", C.c_void_p),
    ]


class MtSceneInfo(C.Structure):
    _fields_ = [
        ("prim_count", C.c_int32),
        ("plane_count", C.c_int32),
        ("node_count", C.c_int32),
        ("depth", C.c_int32),
        ("light_count", C.c_int32),
        ("light_prims", C.c_int32 * 8),
        ("device_bytes", C.c_int64),
    ]


class MtStats(C.Structure):
    _fields_ = [
        ("kernel_ms", C.c_double),
        ("primary_rays", C.c_int64),
        ("extension_rays", C.c_int64),
        ("shadow_rays", C.c_int64),
        ("node_visits", C.c_int64),
        ("prim_tests", C.c_int64),
        ("tri_tests", C.c_int64),
        ("any_node_visits", C.c_int64),
        ("any_prim_tests", C.c_int64),
        ("any_tri_tests", C.c_int64),
        ("launches", C.c_int32),
        ("error_flags", C.c_int32),
        ("stage_ms", C.c_double * 4),
        ("stage_launches", C.c_int64 * 4),
    ]


P = C.c_void_p
I = C.c_int
D = C.c_double

# name -> (restype, argtypes); every symbol declared in include/mtgpu.h
SIGNATURES = {
    "mt_options_default": (None, [P]),
    "mt_scene_create": (I, [P, P, P]),
    "mt_scene_release": (None, [P]),
    "mt_scene_get_info": (I, [P, P]),
    "mt_scene_export_bvh": (I, [P, P, P, P, P, P]),
    "mt_bvh_build_host": (I, [P, I, P, P, P, P, P, P]),
    "mt_camera_create": (None, [P, P, P, D, D, P]),
    "mt_pathtrace_render": (I, [P, P, I, I, I, I, P]),
    "mt_render_image": (I, [P, P, I, I, I, I, P]),
    "mt_render_image_ex": (I, [P, P, I, I, P, P]),
    "mt_render_linear": (I, [P, P, I, I, I, I, I, P]),
    "mt_render_accumulate_device": (I, [P, P, I, I, I, I, I, I, P, I, P]),
    "mt_render_accumulate_device_noalloc": (I, [P, P, I, I, I, I, I, P, I, P]),
    "mt_autotune": (I, [P, P, I, I, I, I, P]),
    "mt_bvh_build_device": (I, [P, I, I, P, P, P, P, P, P, P]),
    "mt_batch_create": (I, [I, I, I, P]),
    "mt_batch_release": (None, [P]),
    "mt_batch_render": (I, [P, I, P, P, P, P]),
    "mt_get_stats": (I, [P, P]),
    "mt_set_counting": (I, [P, I]),
    "mt_pathtrace_radiance": (I, [P, I, P, P, I, P, P]),
    "mt_whitted_trace": (I, [P, I, P, P, I, P, P]),
    "mt_intersect": (I, [P, I, P, P, D, D, P, P, P, P, P]),
    "mt_occluded": (I, [P, I, P, P, D, D, P]),
    "mt_trace_log_enable": (I, [P, I]),
    "mt_trace_log_read": (I, [P, P, I, P]),
    "mt_primary_rays": (I, [P, P, I, I, I, I, P]),
    "mt_scene_param_count": (I, [P]),
    "mt_scene_get_material_params": (I, [P, P, I]),
    "mt_scene_set_material_params": (I, [P, P, I]),
    "mt_adjoint_backward": (I, [P, P, I, I, I, I, P, P, I]),
    "mt_adjoint_backward_device": (I, [P, P, I, I, I, I, I, P, P, I, P]),
    "mt_measure_l2_read_gbs": (I, [I, C.c_size_t, I, P]),
    "mt_version": (C.c_char_p, []),
    "mt_last_error": (C.c_char_p, []),
}

_lib = None


def load(path: str | os.PathLike | None = None) -> C.CDLL:
    """Load libmtgpu.so (once). Raises if the library has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise RuntimeError(
            f"{p} is missing: build the CUDA library first "
            "(python -m marmel_trace_b200.build); there is no CPU fallback"
        )
    lib = C.CDLL(str(p))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


class MtError(RuntimeError):
    def __init__(self, code: int, where: str):
        msg = load().mt_last_error().decode(errors="replace")
        super().__init__(f"{where} failed with code {code}: {msg}")
        self.code = code


def check(code: int, where: str) -> None:
    if code != 0:
        raise MtError(code, where)


def ptr(a: np.ndarray | None) -> int | None:
    """Raw data pointer of a contiguous numpy array (None for None)."""
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"], "arrays crossing the C ABI must be contiguous"
    return a.ctypes.data
