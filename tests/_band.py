"""The FP32 ambiguity band of a traversal query, decided by the oracle.

The device answers a query in FP32 (watertight triangle test, FP32 slab
tests); the oracle answers it in FP64 with Moller-Trumbore. Where the two
differ, the query is inside the FP32 ambiguity band when the oracle's own
answer is not stable under perturbations at FP32 resolution: the origin
moved by `delta` along each world axis, or a bound (tmin / tmax) moved by
`delta`, where `delta` is a few FP32 ulps of the coordinates the query
touches (the origin's and the hit point's magnitudes). A nearest-hit query
is also inside the band when the device's primitive is hit in FP64 at a
distance within 1e-5 relative of the oracle's hit (a tie between two
surfaces at the same place).

Differences outside the band are genuine errors of the FP32 path.
"""
from __future__ import annotations

import numpy as np

# a few FP32 ulps (2^-23 = 1.19e-7) of the coordinate magnitude
ULPS = 4.0 * 2.0 ** -23

_AXES = np.array([[1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1]], np.float64)


def _delta(o, t_ref):
    scale = np.abs(o).max(axis=1) + np.minimum(np.abs(t_ref), 1e3)
    return ULPS * np.maximum(scale, 1.0)


def unstable(rs, kind: str, o, d, tmin, tmax, answer, t_ref):
    """True for every query whose oracle answer (`answer`: prim ids for
    kind "nearest", blocked flags for kind "shadow") changes under the
    perturbations above. `tmin`, `tmax`, `t_ref` are per query."""
    o = np.asarray(o, np.float64)
    d = np.asarray(d, np.float64)
    m = len(o)
    if m == 0:
        return np.zeros(0, bool)
    tmin = np.broadcast_to(np.asarray(tmin, np.float64), (m,))
    tmax = np.broadcast_to(np.asarray(tmax, np.float64), (m,))
    dl = _delta(o, t_ref)
    vo, vd, vlo, vhi = [], [], [], []
    for ax in _AXES:
        vo.append(o + dl[:, None] * ax)
        vd.append(d)
        vlo.append(tmin)
        vhi.append(tmax)
    for s in (-1.0, 1.0):
        vo.append(o)
        vd.append(d)
        vlo.append(np.maximum(tmin + s * dl, 0.0))
        vhi.append(tmax)
        vo.append(o)
        vd.append(d)
        vlo.append(tmin)
        vhi.append(tmax + s * dl)
    res, _ = rs.queries(kind, np.concatenate(vo), np.concatenate(vd), np.concatenate(vlo), np.concatenate(vhi))
    res = res.reshape(len(vo), m)
    return np.any(res != np.asarray(answer)[None, :], axis=0)


def triangle_t(desc, prim, o, d):
    """FP64 two-sided Moller-Trumbore distance of triangle `prim` (NaN when
    missed or not a triangle), per query; vertices from the scene
    descriptor."""
    from marmel_trace_b200 import _capi

    out = np.full(len(prim), np.nan)
    p = desc.prims[np.maximum(prim, 0)]
    tri = (p["kind"] == _capi.PRIM_TRIANGLE) & (prim >= 0)
    if not tri.any():
        return out
    v = p["v"][tri].reshape(-1, 3, 3).astype(np.float64)
    oo = np.asarray(o, np.float64)[tri]
    dd = np.asarray(d, np.float64)[tri]
    dd = dd / np.linalg.norm(dd, axis=1, keepdims=True)
    e1 = v[:, 1] - v[:, 0]
    e2 = v[:, 2] - v[:, 0]
    pv = np.cross(dd, e2)
    det = np.einsum("ij,ij->i", e1, pv)
    ok = np.abs(det) > 1e-12
    inv = np.where(ok, 1.0 / np.where(ok, det, 1.0), 0.0)
    tv = oo - v[:, 0]
    u = np.einsum("ij,ij->i", tv, pv) * inv
    qv = np.cross(tv, e1)
    w = np.einsum("ij,ij->i", dd, qv) * inv
    t = np.einsum("ij,ij->i", e2, qv) * inv
    hit = ok & (u >= -1e-6) & (w >= -1e-6) & (u + w <= 1 + 1e-6)
    out[np.flatnonzero(tri)] = np.where(hit, t, np.nan)
    return out


def classify_nearest(rs, desc, o, d, tmin, tmax, got_prim, want_prim, want_t):
    """(differ, in_band) masks for nearest-hit queries."""
    differ = got_prim != want_prim
    in_band = np.zeros(len(o), bool)
    idx = np.flatnonzero(differ)
    if len(idx):
        t_ref = np.where(want_prim[idx] >= 0, want_t[idx], 1e3)
        band = unstable(rs, "nearest", o[idx], d[idx], np.broadcast_to(tmin, (len(o),))[idx],
                        np.broadcast_to(tmax, (len(o),))[idx], want_prim[idx], t_ref)
        tg = triangle_t(desc, got_prim[idx], o[idx], d[idx])
        tie = np.isfinite(tg) & (want_prim[idx] >= 0) & (np.abs(tg - want_t[idx]) <= 1e-5 * np.abs(want_t[idx]))
        in_band[idx] = band | tie
    return differ, in_band


def classify_shadow(rs, o, d, tmin, tmax, got, want):
    """(differ, in_band) masks for shadow (blocked) queries."""
    differ = got != want
    in_band = np.zeros(len(o), bool)
    idx = np.flatnonzero(differ)
    if len(idx):
        t_ref = np.minimum(np.asarray(tmax)[idx], 1e3)
        in_band[idx] = unstable(rs, "shadow", o[idx], d[idx], np.broadcast_to(tmin, (len(o),))[idx],
                                np.asarray(tmax)[idx], want[idx], t_ref)
    return differ, in_band
