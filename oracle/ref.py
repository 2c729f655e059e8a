"""ctypes access to the oracle: the reference renderer compiled from its own
sources into oracle/_ref/libmtref.so by oracle/Makefile.

TEST INFRASTRUCTURE ONLY. Imported by tests/, by __graft_entry__.smoke() as
the checker, and by the CPU-baseline leg of bench.py. The GPU product path
never imports this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_ref" / "libmtref.so"
CLI = HERE / "_ref" / "raytracer"

P, I, D, U = C.c_void_p, C.c_int, C.c_double, C.c_uint

_SIG = {
    "mtref_load_text": (P, [C.c_char_p, I, I, C.c_char_p, I]),
    "mtref_load_file": (P, [C.c_char_p, I, I, C.c_char_p, I]),
    "mtref_from_desc": (P, [P, P]),
    "mtref_free": (None, [P]),
    "mtref_prim_count": (I, [P]),
    "mtref_material_count": (I, [P]),
    "mtref_lights": (I, [P, P]),
    "mtref_export": (I, [P, P, P, P, P]),
    "mtref_set_camera": (None, [P, P]),
    "mtref_camera_create": (None, [P, P, P, D, D, P]),
    "mtref_intersect": (I, [P, I, P, P, D, D, P, P, P, P, P]),
    "mtref_intersect_linear": (I, [P, I, P, P, D, D, P, P]),
    "mtref_occluded": (I, [P, I, P, P, D, D, P]),
    "mtref_water_height": (D, [P, D, D]),
    "mtref_pt_hash3": (U, [U, U, U]),
    "mtref_pt_rand01": (D, [U, U, U]),
    "mtref_pt_to_byte": (C.c_ubyte, [D]),
    "mtref_pathtrace_render": (I, [P, I, I, I, I, P]),
    "mtref_pt_primary_rays": (I, [P, I, I, I, P]),
    "mtref_pathtrace_radiance": (I, [P, I, P, P, I, P, P]),
    "mtref_pathtrace_linear": (I, [P, I, I, I, I, I, P, I]),
    "mtref_render_hash3": (U, [U, U, U]),
    "mtref_to_byte": (C.c_ubyte, [D]),
    "mtref_render_image": (I, [P, I, I, I, I, P]),
    "mtref_render_image_ex": (I, [P, I, I, I, I, I, I, D, P]),
    "mtref_render_last_seconds": (D, []),
    "mtref_wh_primary_rays": (I, [P, I, I, I, P]),
    "mtref_whitted_trace": (I, [P, I, P, P, I, P, P]),
    "mtref_whitted_linear": (I, [P, I, I, I, I, P, I]),
    "mtref_bvh_export": (I, [P, P, P, P, P, P, P, P, P]),
    "mtref_bvh_count": (I, [P, I, P, P, D, D, P, P, P]),
    "mtref_queries": (I, [P, I, I, P, P, P, P, P, P, I]),
    "mtref_bvh_count_batch": (I, [P, I, I, P, P, P, P, P, I]),
    "mtdual_param_count": (I, [P]),
    "mtdual_pathtrace_grad": (I, [P, I, I, I, I, I, P, D, P, I, P, P]),
}

_lib = None


def sources_present() -> bool:
    """Whether oracle/Makefile finds the reference sources (its REF_DIR, or
    the MT_REF_DIR environment variable)."""
    return subprocess.run(["make", "-s", "-C", str(HERE), "have-ref"], capture_output=True).returncode == 0


def available() -> bool:
    return LIB.exists() or sources_present()


def build() -> None:
    """Compile the oracle (needs the reference sources; never run on the GPU box)."""
    if not sources_present():
        raise RuntimeError("reference sources not found (set MT_REF_DIR to the reference checkout)")
    subprocess.run(["make", "-s", "-C", str(HERE), "cpu", "-j8"], check=True)


def load() -> C.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not LIB.exists():
        build()
    lib = C.CDLL(str(LIB))
    for name, (res, args) in _SIG.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def _p(a):
    return None if a is None else a.ctypes.data


class RefScene:
    """A reference `Scene` + `Camera` held by the oracle library."""

    def __init__(self, handle):
        if not handle:
            raise RuntimeError("oracle scene construction failed")
        self.lib = load()
        self.h = C.c_void_p(handle)

    @classmethod
    def from_text(cls, text: str | None, width: int, height: int) -> "RefScene":
        lib = load()
        err = C.create_string_buffer(512)
        h = lib.mtref_load_text(text.encode() if text is not None else None, width, height, err, 512)
        if not h:
            raise RuntimeError(f"reference parser: {err.value.decode()}")
        return cls(h)

    @classmethod
    def from_file(cls, path: str, width: int, height: int) -> "RefScene":
        lib = load()
        err = C.create_string_buffer(512)
        h = lib.mtref_load_file(str(path).encode(), width, height, err, 512)
        if not h:
            raise RuntimeError(f"reference parser: {err.value.decode()}")
        return cls(h)

    @classmethod
    def from_desc(cls, desc, camera=None) -> "RefScene":
        lib = load()
        cd = desc.c_desc()
        h = lib.mtref_from_desc(C.byref(cd), C.byref(camera.c) if camera is not None else None)
        return cls(h)

    def free(self):
        if self.h and self.h.value:
            self.lib.mtref_free(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass

    def set_camera(self, cam):
        self.lib.mtref_set_camera(self.h, C.byref(cam.c))

    def export(self):
        """Scene -> (SceneDesc, Camera) through the reference-side binding."""
        from marmel_trace_b200 import _capi as capi
        from marmel_trace_b200.api import Camera, SceneDesc

        n = self.lib.mtref_prim_count(self.h)
        m = self.lib.mtref_material_count(self.h)
        prims = np.zeros(n, capi.PRIM_DTYPE)
        mats = np.zeros(m, capi.MATERIAL_DTYPE)
        d = capi.MtSceneDesc()
        cam = capi.MtCamera()
        rc = self.lib.mtref_export(self.h, _p(prims), _p(mats), C.byref(d), C.byref(cam))
        if rc != 0:
            raise RuntimeError(f"binding export failed with code {rc}")
        s = d.sky
        sky = dict(
            sun_dir=tuple(s.sun_dir), sun_color=tuple(s.sun_color), horizon_color=tuple(s.horizon_color),
            zenith_color=tuple(s.zenith_color), gradient_gamma=s.gradient_gamma,
            sun_glow_exponent=s.sun_glow_exponent, sun_glow_strength=s.sun_glow_strength,
            cloud_height=s.cloud_height, cloud_scale=s.cloud_scale, cloud_coverage=s.cloud_coverage,
            cloud_softness=s.cloud_softness, cloud_sharpness=s.cloud_sharpness, cloud_octaves=s.cloud_octaves,
            cloud_thickness=s.cloud_thickness, seed=s.seed, sun_radius=s.sun_radius,
            cloud_density=s.cloud_density, cloud_steps=s.cloud_steps,
        )
        fog = dict(color=tuple(d.fog_color), height=d.fog_height, height_falloff=d.fog_height_falloff,
                   inscatter_strength=d.fog_inscatter_strength, sun_anisotropy=d.fog_sun_anisotropy,
                   noise_scale=d.fog_noise_scale, noise_amount=d.fog_noise_amount, shadow_steps=d.fog_shadow_steps)
        # image textures: copy the bytes the reference scene owns
        images = {}
        for i in range(m):
            addr = int(mats[i]["texture_rgb"])
            if addr:
                h, w = int(mats[i]["texture_height"]), int(mats[i]["texture_width"])
                images[i] = np.ctypeslib.as_array((C.c_uint8 * (h * w * 3)).from_address(addr)).reshape(h, w, 3).copy()
                mats[i]["texture_rgb"] = 0
        desc = SceneDesc(prims=prims, materials=mats, sky=sky, water_level=d.water_level,
                         water_material=d.water_material, fog_density=d.fog_density, fog=fog,
                         images=images or None)
        return desc, Camera(cam)

    def lights(self):
        buf = np.zeros(8, np.int32)
        n = self.lib.mtref_lights(self.h, _p(buf))
        return buf[:n].copy()

    # -- queries ------------------------------------------------------
    def intersect(self, o, d, tmin=1e-4, tmax=1e30):
        o = np.ascontiguousarray(o, np.float64)
        d = np.ascontiguousarray(d, np.float64)
        n = len(o)
        prim = np.zeros(n, np.int32)
        t = np.zeros(n)
        nrm = np.zeros((n, 3))
        front = np.zeros(n, np.int32)
        mat = np.zeros(n, np.int32)
        self.lib.mtref_intersect(self.h, n, _p(o), _p(d), tmin, tmax, _p(prim), _p(t), _p(nrm), _p(front), _p(mat))
        return prim, t, nrm, front, mat

    def intersect_linear(self, o, d, tmin=1e-4, tmax=1e30):
        o = np.ascontiguousarray(o, np.float64)
        d = np.ascontiguousarray(d, np.float64)
        prim = np.zeros(len(o), np.int32)
        t = np.zeros(len(o))
        self.lib.mtref_intersect_linear(self.h, len(o), _p(o), _p(d), tmin, tmax, _p(prim), _p(t))
        return prim, t

    def occluded(self, o, d, tmin, tmax):
        o = np.ascontiguousarray(o, np.float64)
        d = np.ascontiguousarray(d, np.float64)
        occ = np.zeros(len(o), np.int32)
        self.lib.mtref_occluded(self.h, len(o), _p(o), _p(d), tmin, tmax, _p(occ))
        return occ

    def queries(self, kind, o, d, tmin, tmax, threads=None):
        """Per-query bounds, threaded. kind "nearest": scene_intersect ->
        (prim, t); kind "shadow": pt_occluded_segment -> (blocked, None)."""
        o = np.ascontiguousarray(o, np.float64)
        d = np.ascontiguousarray(d, np.float64)
        n = len(o)
        lo = np.ascontiguousarray(np.broadcast_to(np.asarray(tmin, np.float64), (n,)))
        hi = np.ascontiguousarray(np.broadcast_to(np.asarray(tmax, np.float64), (n,)))
        res = np.zeros(n, np.int32)
        t = np.zeros(n) if kind == "nearest" else None
        k = {"nearest": 0, "shadow": 1}[kind]
        nt = threads or os.cpu_count() or 1
        rc = self.lib.mtref_queries(self.h, k, n, _p(o), _p(d), _p(lo), _p(hi), _p(res), _p(t), nt)
        if rc != 0:
            raise RuntimeError(f"mtref_queries returned {rc}")
        return res, t

    # -- renderers ----------------------------------------------------
    def pathtrace_render(self, w, h, spp, depth):
        out = np.zeros((h, w, 3), np.uint8)
        rc = self.lib.mtref_pathtrace_render(self.h, w, h, spp, depth, _p(out))
        if rc != 0:
            raise RuntimeError(f"pathtrace_render returned {rc}")
        return out

    def pathtrace_linear(self, w, h, spp, depth, s0=0, threads=None):
        """Per-pixel mean linear radiance over samples [s0, s0+spp)."""
        out = np.zeros((h, w, 3), np.float64)
        nt = threads or os.cpu_count() or 1
        self.lib.mtref_pathtrace_linear(self.h, w, h, s0, spp, depth, _p(out), nt)
        return out / spp

    def dual_grad(self, w, h, s0, s1, depth, adj, idx=None, scale=None):
        """Forward-mode (dual-number) gradient of sum(adj * mean image) over
        samples [s0, s1) with respect to the adjoint's parameters `idx`
        (default: all). Returns (grad, value_sum, mismatches): value_sum is the
        per-pixel sum of sample values; mismatches counts samples whose value
        or BSDF weight differs from the reference's own (must be 0)."""
        n = self.lib.mtdual_param_count(self.h)
        idx = np.arange(n, dtype=np.int32) if idx is None else np.ascontiguousarray(idx, dtype=np.int32)
        a = np.ascontiguousarray(adj, dtype=np.float32).reshape(h, w, 3)
        g = np.zeros(len(idx), np.float64)
        vs = np.zeros((h, w, 3), np.float64)
        sc = 1.0 / (s1 - s0) if scale is None else scale
        rc = self.lib.mtdual_pathtrace_grad(self.h, w, h, s0, s1, depth, _p(a), sc, _p(idx), len(idx), _p(g), _p(vs))
        if rc < 0:
            raise RuntimeError("the dual-number oracle does not cover this scene")
        return g, vs, rc

    def render_image_ex(self, w, h, spp, depth, adaptive=1, max_spp=0, tau=0.0):
        """render_image_ex: fixed or adaptive Whitted (src/render.c:1627)."""
        out = np.zeros((h, w, 3), np.uint8)
        rc = self.lib.mtref_render_image_ex(self.h, w, h, spp, depth, adaptive, max_spp, tau, _p(out))
        if rc != 0:
            raise RuntimeError(f"render_image_ex returned {rc}")
        return out

    def whitted_render(self, w, h, spp, depth):
        out = np.zeros((h, w, 3), np.uint8)
        rc = self.lib.mtref_render_image(self.h, w, h, spp, depth, _p(out))
        if rc != 0:
            raise RuntimeError(f"render_image returned {rc}")
        return out

    def whitted_linear(self, w, h, spp, depth, threads=None):
        out = np.zeros((h, w, 3), np.float64)
        nt = threads or os.cpu_count() or 1
        self.lib.mtref_whitted_linear(self.h, w, h, spp, depth, _p(out), nt)
        return out

    def primary_rays(self, w, h, spp, mode="pathtrace"):
        out = np.zeros((h * w * spp, 6), np.float64)
        fn = self.lib.mtref_pt_primary_rays if mode == "pathtrace" else self.lib.mtref_wh_primary_rays
        fn(self.h, w, h, spp, _p(out))
        return out

    def radiance(self, o, d, depth, seeds, mode="pathtrace"):
        o = np.ascontiguousarray(o, np.float64)
        d = np.ascontiguousarray(d, np.float64)
        s = np.ascontiguousarray(seeds, np.uint32)
        out = np.zeros((len(s), 3))
        fn = self.lib.mtref_pathtrace_radiance if mode == "pathtrace" else self.lib.mtref_whitted_trace
        fn(self.h, len(s), _p(o), _p(d), depth, _p(s), _p(out))
        return out

    def bvh_export(self):
        n, m, pc, dep = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        self.lib.mtref_bvh_export(self.h, None, None, None, C.byref(n), C.byref(m), None, C.byref(pc), C.byref(dep))
        b = np.zeros((n.value, 6))
        l = np.zeros((n.value, 4), np.int32)
        o = np.zeros(m.value, np.int32)
        pl = np.zeros(max(pc.value, 1), np.int32)
        self.lib.mtref_bvh_export(self.h, _p(b), _p(l), _p(o), C.byref(n), C.byref(m), _p(pl), C.byref(pc),
                                  C.byref(dep))
        return b, l, o, pl[: pc.value], dep.value

    def bvh_count(self, o, d, tmin=1e-4, tmax=1e30):
        o = np.ascontiguousarray(o, np.float64)
        d = np.ascontiguousarray(d, np.float64)
        np_, pt, lv = C.c_longlong(), C.c_longlong(), C.c_longlong()
        self.lib.mtref_bvh_count(self.h, len(o), _p(o), _p(d), tmin, tmax, C.byref(np_), C.byref(pt), C.byref(lv))
        return np_.value, pt.value, lv.value

    def bvh_work(self, kind, o, d, tmin, tmax, threads=None):
        """Canonical traversal work of the reference's tree over queries with
        per-query bounds: (inner nodes with both child boxes tested, triangle
        tests, other primitive tests). kind "nearest" (bvh_intersect) or
        "any" (bvh_occluded without its last-occluder shortcut)."""
        o = np.ascontiguousarray(o, np.float64)
        d = np.ascontiguousarray(d, np.float64)
        n = len(o)
        lo = np.ascontiguousarray(np.broadcast_to(np.asarray(tmin, np.float64), (n,)))
        hi = np.ascontiguousarray(np.broadcast_to(np.asarray(tmax, np.float64), (n,)))
        out = np.zeros(3, np.int64)
        nt = threads or os.cpu_count() or 1
        rc = self.lib.mtref_bvh_count_batch(self.h, 1 if kind == "any" else 0, n, _p(o), _p(d), _p(lo), _p(hi),
                                            _p(out), nt)
        if rc != 0:
            raise RuntimeError(f"mtref_bvh_count_batch returned {rc}")
        return int(out[0]), int(out[1]), int(out[2])


def camera_create(eye, target, up, vfov_deg: float, aspect: float):
    """The reference's camera_create (src/camera.c:24-66), evaluated by the
    oracle library (so that CPU-only callers never load libmtgpu)."""
    from marmel_trace_b200 import _capi as capi
    from marmel_trace_b200.api import Camera

    lib = load()
    out = capi.MtCamera()
    e, t, u = (np.ascontiguousarray(v, dtype=np.float64) for v in (eye, target, up))
    lib.mtref_camera_create(_p(e), _p(t), _p(u), float(vfov_deg), float(aspect), C.byref(out))
    return Camera(out)


def scene_camera(desc, width: int, height: int):
    """The camera a scene descriptor's make_camera builds, from the oracle."""
    c = desc.camera or dict(eye=(-18.0, 6.0, 22.0), target=(0.0, 5.0, -20.0), up=(0.0, 1.0, 0.0), vfov=40.0)
    return camera_create(c["eye"], c["target"], c["up"], c["vfov"], width / height)


def pt_hash3(a, b, c) -> int:
    return load().mtref_pt_hash3(a, b, c)


def pt_rand01(a, b, c) -> float:
    return load().mtref_pt_rand01(a, b, c)


def to_byte(x) -> int:
    return load().mtref_to_byte(x)
