"""CPU restatement of the reference's primary-ray front end (numpy, FP64).

TEST INFRASTRUCTURE ONLY: the checker for the smallest pieces of the hot
path, independent of both the reference build and the GPU library. Each
function cites the reference function it restates. It is pinned by the
tests against (a) the reference's own known-answer vectors from
tests/test_math.c and (b) the reference compiled in oracle/_ref.

Covered: the hash PRNG (src/pathtrace.c:92-117), camera_create / camera_ray
(src/camera.c:24-81), the per-sample primary ray of pt_render_pixel
(src/pathtrace.c:1057-1082, pinhole camera), ray-sphere, ray-plane and
ray-triangle tests (src/geometry.c:338-393,482-538), the nearest-hit linear
scan with the lowest-prim-index tie-break (src/geometry.c:1488-1512) and the
gamma quantiser (src/pathtrace.c:464-480).
"""
from __future__ import annotations

import math

import numpy as np

M32 = 0xFFFFFFFF


def hash_u32(x: np.ndarray) -> np.ndarray:
    """pt_hash_u32 (src/pathtrace.c:92-100)."""
    x = np.asarray(x, dtype=np.uint64) & M32
    x ^= x >> 16
    x = (x * 0x7FEB352D) & M32
    x ^= x >> 15
    x = (x * 0x846CA68B) & M32
    x ^= x >> 16
    return x


def hash3(a, b, c) -> np.ndarray:
    """pt_hash3 (src/pathtrace.c:103-110)."""
    a = np.asarray(a, dtype=np.uint64)
    b = np.asarray(b, dtype=np.uint64)
    c = np.asarray(c, dtype=np.uint64)
    h = np.uint64(0x9E3779B9)
    h = h ^ hash_u32((a + 0x85EBCA6B) & M32)
    h = hash_u32((h + b) & M32)
    h = h ^ hash_u32((c + 0xC2B2AE35) & M32)
    return hash_u32(h)


def rand01(a, b, c) -> np.ndarray:
    """pt_rand01 (src/pathtrace.c:113-117): (h >> 8) / 2^24."""
    return (hash3(a, b, c) >> 8).astype(np.float64) * (1.0 / 16777216.0)


def _norm(v):
    l2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2]
    if l2 <= 1e-12:
        return (0.0, 0.0, 0.0)
    inv = 1.0 / math.sqrt(l2)
    return (v[0] * inv, v[1] * inv, v[2] * inv)


def _cross(a, b):
    return (a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0])


def camera_create(frm, at, up, vfov_deg, aspect) -> dict:
    """camera_create (src/camera.c:24-66), pinhole fields."""
    forward = _norm(tuple(at[k] - frm[k] for k in range(3)))
    if sum(f * f for f in forward) <= 1e-12:
        forward = (0.0, 0.0, -1.0)
    right = _cross(forward, up)
    if sum(r * r for r in right) <= 1e-12:
        right = _cross(forward, (0.0, 1.0, 0.0) if abs(forward[1]) < 0.99 else (1.0, 0.0, 0.0))
    right = _norm(right)
    true_up = _cross(right, forward)
    half_h = math.tan(vfov_deg * (3.14159265358979323846 / 180.0) * 0.5)
    half_w = aspect * half_h
    horizontal = tuple(r * (2.0 * half_w) for r in right)
    vertical = tuple(u * (2.0 * half_h) for u in true_up)
    lower_left = tuple((frm[k] + forward[k]) - (horizontal[k] * 0.5 + vertical[k] * 0.5) for k in range(3))
    return dict(position=tuple(frm), lower_left=lower_left, horizontal=horizontal, vertical=vertical)


def pt_primary_rays(cam: dict, w: int, h: int, spp: int) -> np.ndarray:
    """Primary rays of pt_render_pixel for a pinhole camera, ((y*w+x)*spp+s) order."""
    ys, xs, ss = np.meshgrid(np.arange(h), np.arange(w), np.arange(spp), indexing="ij")
    xs, ys, ss = xs.ravel(), ys.ravel(), ss.ravel()
    jx = rand01(xs, ys, 2 * ss)
    jy = rand01(xs, ys, 2 * ss + 1)
    uu = (xs + jx) / w
    vv = 1.0 - (ys + jy) / h
    ll, hz, vt, pos = (np.array(cam[k]) for k in ("lower_left", "horizontal", "vertical", "position"))
    point = ll[None, :] + (hz[None, :] * uu[:, None] + vt[None, :] * vv[:, None])
    d = point - pos[None, :]
    l2 = d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1] + d[:, 2] * d[:, 2]
    inv = 1.0 / np.sqrt(l2)
    d = d * inv[:, None]
    o = np.broadcast_to(pos, d.shape)
    return np.concatenate([o, d], axis=1)


def _dot(a, b):
    return a[..., 0] * b[..., 0] + a[..., 1] * b[..., 1] + a[..., 2] * b[..., 2]


def _crossv(a, b):
    return np.stack([a[..., 1] * b[..., 2] - a[..., 2] * b[..., 1], a[..., 2] * b[..., 0] - a[..., 0] * b[..., 2],
                     a[..., 0] * b[..., 1] - a[..., 1] * b[..., 0]], axis=-1)


def sphere_t(center, radius, o, d, tmin, tmax):
    """intersect_sphere (src/geometry.c:338-369): distance or nan."""
    if radius <= 0.0:
        return np.full(len(o), np.nan)
    l = o - np.asarray(center)[None, :]
    half_b = _dot(l, d)
    c = _dot(l, l) - radius * radius
    disc = half_b * half_b - c
    with np.errstate(invalid="ignore"):
        sq = np.sqrt(disc)
    t0 = -half_b - sq
    t1 = -half_b + sq
    t = np.where(t0 < tmin, t1, t0)
    ok = (disc >= 0.0) & (t >= tmin) & (t <= tmax)
    return np.where(ok, t, np.nan)


def plane_t(point, normal, o, d, tmin, tmax):
    """intersect_plane (src/geometry.c:372-393); `normal` is the primitive's
    stored axis, which the test normalises once more."""
    n = np.asarray(_norm(normal))
    denom = _dot(d, n[None, :])
    with np.errstate(divide="ignore", invalid="ignore"):
        t = _dot(np.asarray(point)[None, :] - o, n[None, :]) / denom
    ok = (np.abs(denom) >= 1e-12) & (t >= tmin) & (t <= tmax)
    return np.where(ok, t, np.nan)


def triangle_t(a, b, c, o, d, tmin, tmax):
    """intersect_triangle (src/geometry.c:482-538): two-sided Moller-Trumbore."""
    a, b, c = (np.asarray(v, np.float64) for v in (a, b, c))
    e1 = (b - a)[None, :]
    e2 = (c - a)[None, :]
    pvec = _crossv(d, np.broadcast_to(e2, d.shape))
    det = _dot(np.broadcast_to(e1, d.shape), pvec)
    with np.errstate(divide="ignore", invalid="ignore"):
        inv_det = 1.0 / det
        tvec = o - a[None, :]
        u = _dot(tvec, pvec) * inv_det
        qvec = _crossv(tvec, np.broadcast_to(e1, d.shape))
        v = _dot(d, qvec) * inv_det
        t = _dot(np.broadcast_to(e2, d.shape), qvec) * inv_det
    ok = (np.abs(det) >= 1e-9) & (u >= -1e-9) & (u <= 1.0 + 1e-9) & (v >= -1e-9) & (u + v <= 1.0 + 1e-9)
    ok &= (t >= tmin) & (t <= tmax)
    return np.where(ok, t, np.nan)


def nearest_linear(prims, o, d, tmin=1e-4, tmax=1e30):
    """geometry_intersect (src/geometry.c:1488-1512): nearest hit, strict `<`
    in index order (= lowest prim index wins an equal t). Spheres, planes and
    triangles of a PRIM_DTYPE array; returns (prim, t) with prim -1 on miss."""
    best_t = np.full(len(o), np.inf)
    best_p = np.full(len(o), -1, np.int64)
    closest = np.full(len(o), float(tmax))
    for i, p in enumerate(prims):
        k = int(p["kind"])
        v = p["v"]
        if k == 0:
            t = sphere_t(v[:3], v[3], o, d, tmin, closest)
        elif k == 1:
            t = plane_t(v[:3], v[3:6], o, d, tmin, closest)
        elif k == 3:
            t = triangle_t(v[:3], v[3:6], v[6:9], o, d, tmin, closest)
        else:
            raise ValueError("restatement covers spheres, planes and triangles")
        take = ~np.isnan(t) & ((best_p < 0) | (t < best_t))
        best_t = np.where(take, t, best_t)
        best_p = np.where(take, i, best_p)
        closest = np.where(take, t, closest)
    return best_p, np.where(best_p >= 0, best_t, 0.0)


def to_byte(linear: np.ndarray) -> np.ndarray:
    """pathtrace_to_byte (src/pathtrace.c:464-480)."""
    c = np.asarray(linear, np.float64)
    c = np.where(c >= 0.0, c, 0.0)
    c = np.minimum(c, 1.0)
    v = np.power(c, 1.0 / 2.2) * 255.0
    return np.clip((v + 0.5).astype(np.int64), 0, 255).astype(np.uint8)
