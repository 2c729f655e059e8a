"""Host-side mirror of the reference's render interface, over the C ABI.

The functions keep the reference's names, argument meaning and return codes:

    pathtrace_render(scene, cam, width, height, spp, depth, rgb_out) -> int
        src/pathtrace.h:78-80 (0 ok, 1 NULL, 2 bad dimensions, 3 bad spp/depth)
    render_image(scene, cam, width, height, spp, depth, rgb_out) -> int
        src/render.h:29
    render_image_ex(scene, cam, width, height, params, rgb_out) -> int
        src/render.h:65
    pathtrace_radiance(scene, origins, dirs, depth, seed_keys) -> radiance
        src/pathtrace.h:48, batched
    camera_create(eye, target, up, vfov_deg, aspect) -> Camera
        src/camera.c:24-66

`scene` is a `GpuScene`: the device copy of a scene descriptor (`SceneDesc`,
the flat form of the reference's `Scene`). Every call goes through
libmtgpu.so; nothing here computes an image on the CPU.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field

import numpy as np

from . import _capi as capi
from ._capi import MATERIAL_DTYPE, PRIM_DTYPE, check, ptr

# sky_default_params (src/material.c:59-96)
SKY_DEFAULTS = dict(
    sun_dir=None,  # filled with normalize(0.45, 0.75, -0.50)
    sun_color=(1.00, 0.95, 0.85),
    horizon_color=(0.75, 0.85, 1.00),
    zenith_color=(0.35, 0.55, 0.95),
    gradient_gamma=0.6,
    sun_glow_exponent=350.0,
    sun_glow_strength=0.8,
    cloud_height=120.0,
    cloud_scale=0.0025,
    cloud_coverage=0.5,
    cloud_softness=0.12,
    cloud_sharpness=1.5,
    cloud_octaves=5,
    cloud_thickness=0.0,
    cloud_density=0.08,
    cloud_steps=16,
    seed=1337,
    sun_radius=0.0,
)

# FogParams defaults (FOG_DEFAULT_*, src/material.h:185-193) besides density.
FOG_DEFAULTS = dict(
    color=(0.70, 0.75, 0.80),
    height=0.0,
    height_falloff=0.0,
    inscatter_strength=0.50,
    sun_anisotropy=0.70,
    noise_scale=0.0,
    noise_amount=0.0,
    shadow_steps=0,
)


def normalize(v) -> tuple[float, float, float]:
    """vec3_normalize in IEEE double (src/vec3.c:29-37)."""
    x, y, z = (float(c) for c in v)
    len_sq = x * x + y * y + z * z
    if len_sq <= 1e-12:
        return (0.0, 0.0, 0.0)
    inv = 1.0 / math.sqrt(len_sq)
    return (x * inv, y * inv, z * inv)


def default_sky(**overrides) -> dict:
    sky = dict(SKY_DEFAULTS)
    sky["sun_dir"] = normalize((0.45, 0.75, -0.50))
    sky.update(overrides)
    return sky


@dataclass
class SceneDesc:
    """Flat scene: primitives in file order (the reference prim_index order),
    materials, sky and water metadata; the C ABI's mt_scene_desc."""

    prims: np.ndarray
    materials: np.ndarray
    sky: dict = field(default_factory=default_sky)
    water_level: float = 0.0
    water_material: int = -1
    fog_density: float = 0.0
    camera: dict | None = None  # eye, target, up, vfov (the scene's camera block)
    material_names: list[str] | None = None
    fog: dict | None = None  # the other FogParams fields (FOG_DEFAULTS keys)
    images: dict | None = None  # material index -> (H, W, 3) uint8 sRGB image (MT_TEXTURE_IMAGE)

    def __post_init__(self):
        assert self.prims.dtype == PRIM_DTYPE and self.materials.dtype == MATERIAL_DTYPE
        self.prims = np.ascontiguousarray(self.prims)
        self.materials = np.ascontiguousarray(self.materials)

    def c_desc(self) -> capi.MtSceneDesc:
        d = capi.MtSceneDesc()
        d.prims = ptr(self.prims) if len(self.prims) else None
        d.prim_count = len(self.prims)
        d.materials = ptr(self.materials) if len(self.materials) else None
        d.material_count = len(self.materials)
        s = self.sky
        for k in ("sun_dir", "sun_color", "horizon_color", "zenith_color"):
            setattr(d.sky, k, capi.D3(*s[k]))
        for k in (
            "gradient_gamma",
            "sun_glow_exponent",
            "sun_glow_strength",
            "cloud_height",
            "cloud_scale",
            "cloud_coverage",
            "cloud_softness",
            "cloud_sharpness",
            "cloud_thickness",
            "sun_radius",
        ):
            setattr(d.sky, k, float(s[k]))
        d.sky.cloud_octaves = int(s["cloud_octaves"])
        d.sky.seed = int(s["seed"]) & 0xFFFFFFFF
        d.sky.cloud_density = float(s.get("cloud_density", SKY_DEFAULTS["cloud_density"]))
        d.sky.cloud_steps = int(s.get("cloud_steps", SKY_DEFAULTS["cloud_steps"]))
        d.fog_density = float(self.fog_density)
        d.water_level = float(self.water_level)
        d.water_material = int(self.water_material)
        f = dict(FOG_DEFAULTS, **(self.fog or {}))
        d.fog_color = capi.D3(*f["color"])
        for k in ("height", "height_falloff", "inscatter_strength", "sun_anisotropy", "noise_scale", "noise_amount"):
            setattr(d, "fog_" + k, float(f[k]))
        d.fog_shadow_steps = int(f["shadow_steps"])
        # image textures: the materials array carries the address of each image
        for i, img in (self.images or {}).items():
            img = np.ascontiguousarray(img, np.uint8)
            assert img.ndim == 3 and img.shape[2] == 3
            self.images[i] = img
            self.materials[i]["texture_rgb"] = img.ctypes.data
            self.materials[i]["texture_height"], self.materials[i]["texture_width"] = img.shape[:2]
        return d

    def make_camera(self, width: int, height: int) -> "Camera":
        c = self.camera or dict(eye=(-18.0, 6.0, 22.0), target=(0.0, 5.0, -20.0), up=(0.0, 1.0, 0.0), vfov=40.0)
        return camera_create(c["eye"], c["target"], c["up"], c["vfov"], width / height)


class Camera:
    """mt_camera (Camera, src/camera.h)."""

    def __init__(self, c: capi.MtCamera):
        self.c = c

    @property
    def ref(self):
        return C.byref(self.c)


def camera_create(eye, target, up, vfov_deg: float, aspect: float) -> Camera:
    """camera_create (src/camera.c:24-66), evaluated by the C ABI."""
    lib = capi.load()
    out = capi.MtCamera()
    e, t, u = (np.asarray(v, dtype=np.float64) for v in (eye, target, up))
    lib.mt_camera_create(ptr(e), ptr(t), ptr(u), float(vfov_deg), float(aspect), C.byref(out))
    return Camera(out)


def bvh_build_host(prims: np.ndarray):
    """The library's host BVH for `prims` (no device): bounds (n, 6),
    links (n, 4) = left, right, first, count, the permutation and the depth."""
    lib = capi.load()
    prims = np.ascontiguousarray(prims)
    n, m, dep = C.c_int32(), C.c_int32(), C.c_int32()
    check(lib.mt_bvh_build_host(ptr(prims), len(prims), None, None, None, C.byref(n), C.byref(m), C.byref(dep)),
          "mt_bvh_build_host")
    b = np.zeros((n.value, 6), np.float64)
    l = np.zeros((n.value, 4), np.int32)
    o = np.zeros(max(m.value, 1), np.int32)
    check(lib.mt_bvh_build_host(ptr(prims), len(prims), ptr(b), ptr(l), ptr(o), C.byref(n), C.byref(m),
                                C.byref(dep)), "mt_bvh_build_host")
    return b, l, o[: m.value], dep.value


def bvh_build_device(prims: np.ndarray, device: int = 0):
    """The same BVH built on a CUDA device (mt_bvh_build_device): bounds,
    links, permutation, depth and the device build time in ms."""
    lib = capi.load()
    prims = np.ascontiguousarray(prims)
    n, m, dep, ms = C.c_int32(), C.c_int32(), C.c_int32(), C.c_float()
    check(lib.mt_bvh_build_device(ptr(prims), len(prims), device, None, None, None, C.byref(n), C.byref(m),
                                  C.byref(dep), None), "mt_bvh_build_device")
    b = np.zeros((n.value, 6), np.float64)
    l = np.zeros((n.value, 4), np.int32)
    o = np.zeros(max(m.value, 1), np.int32)
    check(lib.mt_bvh_build_device(ptr(prims), len(prims), device, ptr(b), ptr(l), ptr(o), C.byref(n), C.byref(m),
                                  C.byref(dep), C.byref(ms)), "mt_bvh_build_device")
    return b, l, o[: m.value], dep.value, ms.value


def make_options(precision: str = "fp32", integrator: str = "megakernel", **kw) -> capi.MtOptions:
    lib = capi.load()
    o = capi.MtOptions()
    lib.mt_options_default(C.byref(o))
    o.precision = {"fp32": capi.PRECISION_FP32, "fp64": capi.PRECISION_FP64}[precision]
    o.integrator = {"megakernel": capi.INTEGRATOR_MEGAKERNEL, "wavefront": capi.INTEGRATOR_WAVEFRONT}[integrator]
    for k, v in kw.items():
        setattr(o, k, int(v))
    return o


class GpuScene:
    """Device-resident scene (mt_scene*). Release with .release() or `with`."""

    def __init__(self, desc: SceneDesc, precision: str = "fp32", integrator: str = "megakernel", **opts):
        self.lib = capi.load()
        self.desc = desc
        self.precision = precision
        self.opts = make_options(precision, integrator, **opts)
        self._c_desc = desc.c_desc()
        h = C.c_void_p()
        check(self.lib.mt_scene_create(C.byref(self._c_desc), C.byref(self.opts), C.byref(h)), "mt_scene_create")
        self.h = h

    # -- lifetime -----------------------------------------------------
    def release(self):
        if getattr(self, "h", None) and self.h.value:
            self.lib.mt_scene_release(self.h)
            self.h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.release()

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass

    # -- introspection ------------------------------------------------
    def info(self) -> capi.MtSceneInfo:
        out = capi.MtSceneInfo()
        check(self.lib.mt_scene_get_info(self.h, C.byref(out)), "mt_scene_get_info")
        return out

    def stats(self) -> capi.MtStats:
        out = capi.MtStats()
        check(self.lib.mt_get_stats(self.h, C.byref(out)), "mt_get_stats")
        return out

    def set_counting(self, on: bool):
        check(self.lib.mt_set_counting(self.h, 1 if on else 0), "mt_set_counting")

    def export_bvh(self):
        n, m = C.c_int32(), C.c_int32()
        check(self.lib.mt_scene_export_bvh(self.h, None, None, None, C.byref(n), C.byref(m)), "export_bvh")
        b = np.zeros((n.value, 6), np.float64)
        l = np.zeros((n.value, 4), np.int32)
        o = np.zeros(m.value, np.int32)
        check(self.lib.mt_scene_export_bvh(self.h, ptr(b), ptr(l), ptr(o), C.byref(n), C.byref(m)), "export_bvh")
        return b, l, o

    # -- renderers (raise on error) -------------------------------------
    def pathtrace(self, cam: Camera, w: int, h: int, spp: int, depth: int) -> np.ndarray:
        out = np.zeros((h, w, 3), np.uint8)
        check(self.lib.mt_pathtrace_render(self.h, cam.ref, w, h, spp, depth, ptr(out)), "mt_pathtrace_render")
        return out

    def whitted(self, cam: Camera, w: int, h: int, spp: int, depth: int) -> np.ndarray:
        out = np.zeros((h, w, 3), np.uint8)
        check(self.lib.mt_render_image(self.h, cam.ref, w, h, spp, depth, ptr(out)), "mt_render_image")
        return out

    def autotune(self, cam: Camera, w: int, h: int, probe_spp: int, depth: int) -> dict:
        """mt_autotune: time the wavefront configurations on a probe window
        and keep the fastest on this scene. Returns the chosen options, the
        probe times and every timed candidate."""
        rep = capi.MtTuneReport()
        check(self.lib.mt_autotune(self.h, cam.ref, w, h, probe_spp, depth, C.byref(rep)), "mt_autotune")

        def opts(o):
            return {"traversal": {0: "static", 1: "static", 2: "dynamic"}[o.traversal], "block": o.block_size,
                    "bvh_width": o.bvh_width, "sort_threshold": o.sort_threshold,
                    "queue_capacity": o.queue_capacity or 1 << 25, "occluder_cache": o.occluder_cache}

        return {"chosen": opts(rep.chosen), "chosen_ms": rep.chosen_ms, "default_ms": rep.default_ms,
                "candidates": [dict(opts(rep.entries[i].options), ms=round(rep.entries[i].ms, 3))
                               for i in range(rep.n_entries)]}

    def linear(self, cam: Camera, w: int, h: int, spp: int, depth: int, mode: str = "pathtrace") -> np.ndarray:
        out = np.zeros((h, w, 3), np.float32)
        m = capi.MODE_PATHTRACE if mode == "pathtrace" else capi.MODE_WHITTED
        check(self.lib.mt_render_linear(self.h, cam.ref, w, h, spp, depth, m, ptr(out)), "mt_render_linear")
        return out

    def radiance(self, origins, dirs, depth: int, seeds, mode: str = "pathtrace") -> np.ndarray:
        o = np.ascontiguousarray(origins, np.float64)
        d = np.ascontiguousarray(dirs, np.float64)
        s = np.ascontiguousarray(seeds, np.uint32)
        n = len(s)
        out = np.zeros((n, 3), np.float64)
        fn = self.lib.mt_pathtrace_radiance if mode == "pathtrace" else self.lib.mt_whitted_trace
        check(fn(self.h, n, ptr(o), ptr(d), depth, ptr(s), ptr(out)), fn.__name__)
        return out

    def intersect(self, origins, dirs, tmin: float = 1e-4, tmax: float = 1e30):
        o = np.ascontiguousarray(origins, np.float64)
        d = np.ascontiguousarray(dirs, np.float64)
        n = len(o)
        prim = np.zeros(n, np.int32)
        t = np.zeros(n, np.float64)
        nrm = np.zeros((n, 3), np.float64)
        front = np.zeros(n, np.int32)
        mat = np.zeros(n, np.int32)
        check(
            self.lib.mt_intersect(self.h, n, ptr(o), ptr(d), tmin, tmax, ptr(prim), ptr(t), ptr(nrm), ptr(front), ptr(mat)),
            "mt_intersect",
        )
        return prim, t, nrm, front, mat

    def occluded(self, origins, dirs, tmin: float, tmax: float) -> np.ndarray:
        o = np.ascontiguousarray(origins, np.float64)
        d = np.ascontiguousarray(dirs, np.float64)
        occ = np.zeros(len(o), np.int32)
        check(self.lib.mt_occluded(self.h, len(o), ptr(o), ptr(d), tmin, tmax, ptr(occ)), "mt_occluded")
        return occ

    def trace_log_enable(self, capacity: int):
        """Record the wavefront stages' traversal queries (mt_trace_log_enable)."""
        check(self.lib.mt_trace_log_enable(self.h, int(capacity)), "mt_trace_log_enable")

    def trace_log_read(self, capacity: int):
        """(records, seen): the logged queries as a structured array with
        fields o (3), d (3), t, result, kind, bounce, light, and the number of
        queries seen since the log was enabled."""
        raw = np.zeros((max(int(capacity), 1), 12), np.float32)
        seen = C.c_int64()
        check(self.lib.mt_trace_log_read(self.h, ptr(raw), int(capacity), C.byref(seen)), "mt_trace_log_read")
        n = min(seen.value, int(capacity))
        raw = raw[:n]
        ints = raw.view(np.int32)
        rec = np.zeros(n, dtype=[("o", np.float32, 3), ("d", np.float32, 3), ("t", np.float32), ("result", np.int32),
                                 ("kind", np.int32), ("bounce", np.int32), ("light", np.int32)])
        rec["o"] = raw[:, 0:3]
        rec["d"] = raw[:, 3:6]
        rec["t"] = raw[:, 6]
        rec["result"] = ints[:, 7]
        rec["kind"] = ints[:, 8]
        rec["bounce"] = ints[:, 9]
        rec["light"] = ints[:, 10]
        return rec, seen.value

    def primary_rays(self, cam: Camera, w: int, h: int, spp: int, mode: str = "pathtrace") -> np.ndarray:
        out = np.zeros((h * w * spp, 6), np.float64)
        m = capi.MODE_PATHTRACE if mode == "pathtrace" else capi.MODE_WHITTED
        check(self.lib.mt_primary_rays(self.h, cam.ref, w, h, spp, m, ptr(out)), "mt_primary_rays")
        return out


# ---------------------------------------------------------------------
# Reference-named entry points returning the reference's status codes.
# ---------------------------------------------------------------------
def pathtrace_render(scene: GpuScene | None, cam: Camera | None, width: int, height: int, spp: int, depth: int,
                     rgb_out: np.ndarray | None) -> int:
    lib = capi.load()
    return lib.mt_pathtrace_render(scene.h if scene else None, cam.ref if cam else None, width, height, spp, depth,
                                   ptr(rgb_out) if rgb_out is not None else None)


def render_image(scene, cam, width, height, spp, depth, rgb_out) -> int:
    lib = capi.load()
    return lib.mt_render_image(scene.h if scene else None, cam.ref if cam else None, width, height, spp, depth,
                               ptr(rgb_out) if rgb_out is not None else None)


def render_image_ex(scene, cam, width, height, params: dict | None, rgb_out) -> int:
    lib = capi.load()
    p = None
    if params is not None:
        p = capi.MtRenderParams(
            int(params.get("samples_per_pixel", 1)),
            int(params.get("max_depth", 0)),
            int(params.get("adaptive", 0)),
            int(params.get("adaptive_max_spp", 0)),
            float(params.get("adaptive_tau", 0.0)),
        )
    return lib.mt_render_image_ex(scene.h if scene else None, cam.ref if cam else None, width, height,
                                  C.byref(p) if p is not None else None, ptr(rgb_out) if rgb_out is not None else None)


def pathtrace_radiance(scene: GpuScene, origins, dirs, depth: int, seed_keys) -> np.ndarray:
    return scene.radiance(origins, dirs, depth, seed_keys, mode="pathtrace")
