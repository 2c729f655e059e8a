// mt_geom.cuh - ray / primitive tests and BVH traversal.
//
// FP64 instantiation: the reference's tests restated operation by operation
// (src/geometry.c:338-699,705-800,1373-1451) so hits, distances and normals
// agree bit for bit.
// FP32 instantiation: the same acceptance rules with two numerically robust
// tests in place of the textbook forms:
//   * triangles use the watertight test of Woop, Benthin and Wald, "Watertight
//     Ray/Triangle Intersection", JCGT 2(1), 2013 (shear to the ray's dominant
//     axis, 2D edge functions; no cracks along shared edges);
//   * spheres use the perpendicular-distance discriminant of Haines et al.,
//     "Precision Improvements for Ray/Sphere Intersection", Ray Tracing Gems
//     ch. 7, 2019, which avoids the |o-c|^2 - r^2 cancellation.
#pragma once

#include "mt_layout.h"
#include "mt_math.cuh"

namespace mt {

template <typename R> struct Hit {
    R t;
    R u, v;       // triangle barycentrics (weights of b and c)
    int prim;     // reference prim_index
    int code;     // kind << 28 | slot
};

// Per-ray precomputation shared by every node and primitive test.
template <typename R> struct RayPre {
    V3<R> o, d, inv;
    V3<R> oi;  // o * inv: an FP32 slab distance is one fma, box * inv - oi
    // watertight-triangle shear (FP32 path)
    int kx, ky, kz;
    float sx, sy, sz;
};

template <typename R> MT_D RayPre<R> ray_pre(V3<R> o, V3<R> d)
{
    RayPre<R> p;
    p.o = o;
    p.d = d;
    // 1/dir per component (src/bvh.c:571): IEEE infinities for zero components.
    p.inv = v3<R>(R(1) / d.x, R(1) / d.y, R(1) / d.z);
    if constexpr (sizeof(R) == 4) {
        // FP32 slab tests use the fma form, where an infinite inverse would give
        // inf - inf; a (near-)zero component gets a finite 1e30 of its sign
        // instead, which orders every slab of the scene the same way.
        p.inv.x = fabsf(d.x) < 1e-30f ? copysignf(1e30f, d.x) : p.inv.x;
        p.inv.y = fabsf(d.y) < 1e-30f ? copysignf(1e30f, d.y) : p.inv.y;
        p.inv.z = fabsf(d.z) < 1e-30f ? copysignf(1e30f, d.z) : p.inv.z;
    }
    p.oi = v3<R>(o.x * p.inv.x, o.y * p.inv.y, o.z * p.inv.z);
    float ax = fabsf((float)d.x), ay = fabsf((float)d.y), az = fabsf((float)d.z);
    int kz = (ax > ay) ? ((ax > az) ? 0 : 2) : ((ay > az) ? 1 : 2);
    int kx = kz + 1 == 3 ? 0 : kz + 1;
    int ky = kx + 1 == 3 ? 0 : kx + 1;
    float dz = kz == 0 ? (float)d.x : (kz == 1 ? (float)d.y : (float)d.z);
    if (dz < 0.0f) {
        int t = kx;
        kx = ky;
        ky = t;
    }
    float dx = kx == 0 ? (float)d.x : (kx == 1 ? (float)d.y : (float)d.z);
    float dy = ky == 0 ? (float)d.x : (ky == 1 ? (float)d.y : (float)d.z);
    p.kx = kx;
    p.ky = ky;
    p.kz = kz;
    p.sx = dx / dz;
    p.sy = dy / dz;
    p.sz = 1.0f / dz;
    return p;
}

template <typename R> MT_D R comp(V3<R> v, int k) { return k == 0 ? v.x : (k == 1 ? v.y : v.z); }
MT_D float comp4(float4 v, int k) { return k == 0 ? v.x : (k == 1 ? v.y : v.z); }

// ------------------------------------------------------------------
// Spheres (intersect_sphere src/geometry.c:338-369, occluded_sphere :1373-1381)
// ------------------------------------------------------------------
MT_D bool sphere_t(const double *s, const RayPre<double> &rp, double tmin, double tmax, double *t_out)
{
    double radius = s[3];
    if (radius <= 0.0) return false;
    V3<double> l = sub(rp.o, v3(s[0], s[1], s[2]));
    double half_b = dot(l, rp.d);
    double c = length_sq(l) - radius * radius;
    double disc = half_b * half_b - c;
    if (disc < 0.0) return false;
    double sq = sqrt(disc);
    double t = -half_b - sq;
    if (t < tmin) {
        t = -half_b + sq;
        if (t < tmin || t > tmax) return false;
    } else if (t > tmax) {
        return false;
    }
    *t_out = t;
    return true;
}

MT_D bool sphere_t(const float *s, const RayPre<float> &rp, float tmin, float tmax, float *t_out)
{
    float radius = s[3];
    if (radius <= 0.0f) return false;
    V3<float> f = sub(rp.o, v3(s[0], s[1], s[2]));
    float b = -dot(f, rp.d);
    V3<float> l = add(f, scale(rp.d, b));           // component of f perpendicular to d
    float r2 = radius * radius;
    float disc = r2 - dot(l, l);
    if (disc < 0.0f) return false;
    float q = b + copysignf(sqrtf(disc), b);
    float c = dot(f, f) - r2;
    float t0, t1;
    if (q == 0.0f) {
        t0 = t1 = 0.0f;
    } else {
        t0 = c / q;
        t1 = q;
    }
    if (t0 > t1) {
        float tt = t0;
        t0 = t1;
        t1 = tt;
    }
    float t = t0;
    if (t < tmin) {
        t = t1;
        if (t < tmin || t > tmax) return false;
    } else if (t > tmax) {
        return false;
    }
    *t_out = t;
    return true;
}

// ------------------------------------------------------------------
// Planes (intersect_plane src/geometry.c:372-393); the unit normal is
// precomputed on the host with vec3_normalize's exact arithmetic.
// ------------------------------------------------------------------
template <typename R>
MT_D bool plane_t(const R *p, V3<R> o, V3<R> d, R tmin, R tmax, R *t_out)
{
    V3<R> n = v3(p[3], p[4], p[5]);
    R denom = dot(d, n);
    if (mfabs(denom) < R(1e-12)) return false;
    R t = dot(sub(v3(p[0], p[1], p[2]), o), n) / denom;
    if (t < tmin || t > tmax) return false;
    *t_out = t;
    return true;
}

// ------------------------------------------------------------------
// Boxes: slab method with entry/exit face (intersect_box src/geometry.c:396-479)
// and the any-hit variant (occluded_box :1392-1411), which orders its slab
// distances with a swap instead of fmin/fmax.
// ------------------------------------------------------------------
template <typename R>
MT_D bool box_t(const R *b, V3<R> o, V3<R> d, R tmin, R tmax, R *t_out, int *axis_out, int *sign_out)
{
    R lo[3] = {b[0] - b[3], b[1] - b[4], b[2] - b[5]};
    R hi[3] = {b[0] + b[3], b[1] + b[4], b[2] + b[5]};
    R oo[3] = {o.x, o.y, o.z};
    R dd[3] = {d.x, d.y, d.z};
    R tn = -INFINITY, tf = INFINITY;
    int entry_axis = -1, entry_sign = 0, exit_axis = -1, exit_sign = 0;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        R inv = R(1) / dd[i];
        R t1 = (lo[i] - oo[i]) * inv;
        R t2 = (hi[i] - oo[i]) * inv;
        R t_near = mfmin(t1, t2);
        R t_far = mfmax(t1, t2);
        if (t_near > tn) {
            tn = t_near;
            entry_axis = i;
            entry_sign = (inv > R(0)) ? -1 : 1;
        }
        if (t_far < tf) {
            tf = t_far;
            exit_axis = i;
            exit_sign = (inv > R(0)) ? 1 : -1;
        }
        if (tf < tn) return false;
    }
    if (tn >= tmin && tn <= tmax) {
        *t_out = tn;
        *axis_out = entry_axis;
        *sign_out = entry_sign;
        return true;
    }
    if (tf >= tmin && tf <= tmax) {
        *t_out = tf;
        *axis_out = exit_axis;
        *sign_out = exit_sign;
        return true;
    }
    return false;
}

template <typename R> MT_D bool box_occluded(const R *b, V3<R> o, V3<R> d, R tmin, R tmax)
{
    R lo[3] = {b[0] - b[3], b[1] - b[4], b[2] - b[5]};
    R hi[3] = {b[0] + b[3], b[1] + b[4], b[2] + b[5]};
    R oo[3] = {o.x, o.y, o.z};
    R dd[3] = {d.x, d.y, d.z};
    R tn = -INFINITY, tf = INFINITY;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        R inv = R(1) / dd[i];
        R t1 = (lo[i] - oo[i]) * inv;
        R t2 = (hi[i] - oo[i]) * inv;
        if (t1 > t2) {
            R tmp = t1;
            t1 = t2;
            t2 = tmp;
        }
        if (t1 > tn) tn = t1;
        if (t2 < tf) tf = t2;
        if (tn > tf) return false;
    }
    return (tn >= tmin && tn <= tmax) || (tf >= tmin && tf <= tmax);
}

// ------------------------------------------------------------------
// Tapered capped cylinder (intersect_cylinder src/geometry.c:549-699).
// Returns t and the outward normal (before facing the ray).
// ------------------------------------------------------------------
// Which surface of a tapered cylinder was hit (for the hit's texture u, v).
template <typename R> struct CylPart {
    int is_cap;  // 1: a cap disc, 0: the side
    int cap;     // 0: base (s = 0), 1: top (s = 1)
    R s;         // side: axial coordinate in [0, 1]
};

template <typename R>
MT_D bool cylinder_hit(const R *c, V3<R> o, V3<R> d, R tmin, R tmax, R *t_out, V3<R> *n_out,
                       CylPart<R> *part = nullptr)
{
    V3<R> pa = v3(c[0], c[1], c[2]);
    V3<R> pb = v3(c[3], c[4], c[5]);
    V3<R> A = sub(pb, pa);
    R h = length(A);
    if (h < R(1e-12)) return false;
    V3<R> axis = scale(A, R(1) / h);
    R r0 = c[6], r1 = c[7];
    R k = (r1 - r0) / h;
    V3<R> d0 = sub(o, pa);
    R Od = dot(d, axis);
    R d0d = dot(d0, axis);
    V3<R> D_perp = sub(d, scale(axis, Od));
    V3<R> d0_perp = sub(d0, scale(axis, d0d));
    R ra = k * Od;
    R rb = r0 + k * d0d;
    R qa = length_sq(D_perp) - ra * ra;
    R qb = dot(D_perp, d0_perp) - rb * ra;
    R qc = length_sq(d0_perp) - rb * rb;

    bool found = false;
    R best_t = R(0), best_s = R(0);
    int best_is_cap = 0, best_cap = 0;
    V3<R> best_n = v3(R(0), R(0), R(0));

    if (mfabs(qa) > R(1e-15)) {
        R disc = qb * qb - qa * qc;
        if (disc >= R(0)) {
            R sq = msqrt(disc);
            R roots[2];
            roots[0] = (-qb - sq) / qa;
            roots[1] = (-qb + sq) / qa;
            if (roots[0] > roots[1]) {
                R tmp = roots[0];
                roots[0] = roots[1];
                roots[1] = tmp;
            }
            for (int i = 0; i < 2; ++i) {
                R t = roots[i];
                if (t < tmin || t > tmax) continue;
                R s = (d0d + t * Od) / h;
                if (s < R(0) || s > R(1)) continue;
                V3<R> point = at(o, d, t);
                V3<R> axis_pt = add(pa, scale(axis, s * h));
                V3<R> radial = sub(point, axis_pt);
                R rlen = length(radial);
                V3<R> radial_dir = (rlen > R(1e-15)) ? scale(radial, R(1) / rlen) : v3(R(0), R(0), R(0));
                V3<R> n = sub(scale(radial_dir, h), scale(axis, r1 - r0));
                n = normalize(n);
                if (length_sq(n) < R(0.5)) n = radial_dir;
                if (!found || t < best_t) {
                    found = true;
                    best_t = t;
                    best_n = n;
                    best_s = s;
                }
            }
        }
    } else if (mfabs(qb) > R(1e-15)) {
        R t = -qc / (R(2) * qb);
        if (t >= tmin && t <= tmax) {
            R s = (d0d + t * Od) / h;
            if (s >= R(0) && s <= R(1)) {
                V3<R> point = at(o, d, t);
                V3<R> axis_pt = add(pa, scale(axis, s * h));
                V3<R> radial = sub(point, axis_pt);
                V3<R> radial_dir = normalize(radial);
                V3<R> n = sub(scale(radial_dir, h), scale(axis, r1 - r0));
                n = normalize(n);
                if (length_sq(n) < R(0.5)) n = radial_dir;
                found = true;
                best_t = t;
                best_n = n;
                best_s = s;
            }
        }
    }
    if (mfabs(Od) > R(1e-15)) {
        for (int cap = 0; cap < 2; ++cap) {
            R s_cap = (cap == 0) ? R(0) : R(1);
            R r_cap = (cap == 0) ? r0 : r1;
            if (r_cap <= R(0)) continue;
            V3<R> cap_center = (cap == 0) ? pa : pb;
            R t = ((s_cap * h) - d0d) / Od;
            if (t < tmin || t > tmax) continue;
            V3<R> point = at(o, d, t);
            V3<R> radial = sub(point, cap_center);
            if (length_sq(radial) > r_cap * r_cap) continue;
            V3<R> n = (cap == 0) ? neg(axis) : axis;
            if (!found || t < best_t) {
                found = true;
                best_t = t;
                best_n = n;
                best_is_cap = 1;
                best_cap = cap;
            }
        }
    }
    if (!found) return false;
    *t_out = best_t;
    *n_out = best_n;
    if (part) {
        part->is_cap = best_is_cap;
        part->cap = best_cap;
        part->s = best_s;
    }
    return true;
}

// ------------------------------------------------------------------
// Triangles
// ------------------------------------------------------------------
// FP64: Moller-Trumbore, two-sided, det guard 1e-9, barycentric slack 1e-9
// (intersect_triangle src/geometry.c:482-538 / occluded_triangle :1414-1433).
MT_D bool tri_t(const DevScene<double> &S, int slot, const RayPre<double> &rp, double tmin, double tmax,
                double *t_out, double *u_out, double *v_out)
{
    const double *T = S.tris + 9 * (size_t)slot;
    V3<double> a = v3(T[0], T[1], T[2]);
    V3<double> e1 = v3(T[3], T[4], T[5]);
    V3<double> e2 = v3(T[6], T[7], T[8]);
    V3<double> pvec = cross(rp.d, e2);
    double det = dot(e1, pvec);
    if (fabs(det) < 1e-9) return false;
    double inv_det = 1.0 / det;
    V3<double> tvec = sub(rp.o, a);
    double u = dot(tvec, pvec) * inv_det;
    if (u < -1e-9 || u > 1.0 + 1e-9) return false;
    V3<double> qvec = cross(tvec, e1);
    double v = dot(rp.d, qvec) * inv_det;
    if (v < -1e-9 || u + v > 1.0 + 1e-9) return false;
    double t = dot(e2, qvec) * inv_det;
    if (t < tmin || t > tmax) return false;
    *t_out = t;
    *u_out = u;
    *v_out = v;
    return true;
}

// FP32: watertight test (Woop, Benthin, Wald 2013). Vertices are stored
// relative to nothing (v0, v1, v2) so the shear is applied to exact
// differences from the ray origin. tri_edges evaluates the edge functions
// U, V, W (one sign for a hit), det = U + V + W and the scaled distance T, so
// that t = T / det; false when the ray misses the triangle's edges.
struct TriEdges {
    float U, V, W, det, T;
};
MT_D bool tri_edges(const DevScene<float> &S, int slot, const RayPre<float> &rp, TriEdges *e)
{
    const float4 *T = S.tri4 + 3 * (size_t)slot;
    float4 q0 = __ldg(T), q1 = __ldg(T + 1), q2 = __ldg(T + 2);
    float Akx = comp4(q0, rp.kx) - comp(rp.o, rp.kx), Aky = comp4(q0, rp.ky) - comp(rp.o, rp.ky),
          Akz = comp4(q0, rp.kz) - comp(rp.o, rp.kz);
    float Bkx = comp4(q1, rp.kx) - comp(rp.o, rp.kx), Bky = comp4(q1, rp.ky) - comp(rp.o, rp.ky),
          Bkz = comp4(q1, rp.kz) - comp(rp.o, rp.kz);
    float Ckx = comp4(q2, rp.kx) - comp(rp.o, rp.kx), Cky = comp4(q2, rp.ky) - comp(rp.o, rp.ky),
          Ckz = comp4(q2, rp.kz) - comp(rp.o, rp.kz);
    float Ax = Akx - rp.sx * Akz, Ay = Aky - rp.sy * Akz;
    float Bx = Bkx - rp.sx * Bkz, By = Bky - rp.sy * Bkz;
    float Cx = Ckx - rp.sx * Ckz, Cy = Cky - rp.sy * Ckz;
    float U = Cx * By - Cy * Bx;
    float V = Ax * Cy - Ay * Cx;
    float W = Bx * Ay - By * Ax;
    if (U == 0.0f || V == 0.0f || W == 0.0f) {
        // Edge case of the paper: re-evaluate the edge functions in double.
        U = (float)((double)Cx * (double)By - (double)Cy * (double)Bx);
        V = (float)((double)Ax * (double)Cy - (double)Ay * (double)Cx);
        W = (float)((double)Bx * (double)Ay - (double)By * (double)Ax);
    }
    if ((U < 0.0f || V < 0.0f || W < 0.0f) && (U > 0.0f || V > 0.0f || W > 0.0f)) return false;
    float det = U + V + W;
    if (det == 0.0f) return false;
    float Az = rp.sz * Akz, Bz = rp.sz * Bkz, Cz = rp.sz * Ckz;
    e->U = U;
    e->V = V;
    e->W = W;
    e->det = det;
    e->T = U * Az + V * Bz + W * Cz;
    return true;
}

MT_D bool tri_t(const DevScene<float> &S, int slot, const RayPre<float> &rp, float tmin, float tmax,
                float *t_out, float *u_out, float *v_out)
{
    TriEdges e;
    if (!tri_edges(S, slot, rp, &e)) return false;
    float rcp = 1.0f / e.det;
    float t = e.T * rcp;
    if (!(t >= tmin && t <= tmax)) return false;
    *t_out = t;
    *u_out = e.V * rcp;
    *v_out = e.W * rcp;
    return true;
}

// Any-hit form: t = T / det in [tmin, tmax] is decided as T against
// tmin * det and tmax * det, with det made positive (no division).
MT_D bool tri_occ(const DevScene<float> &S, int slot, const RayPre<float> &rp, float tmin, float tmax)
{
    TriEdges e;
    if (!tri_edges(S, slot, rp, &e)) return false;
    const float T = e.det < 0.0f ? -e.T : e.T;
    const float det = fabsf(e.det);
    return T >= tmin * det && T <= tmax * det;
}

// FP64: the any-hit test is the nearest-hit test's boolean.
MT_D bool tri_occ(const DevScene<double> &S, int slot, const RayPre<double> &rp, double tmin, double tmax)
{
    double t, u, v;
    return tri_t(S, slot, rp, tmin, tmax, &t, &u, &v);
}

// ------------------------------------------------------------------
// Generic primitive tests by code (kind << 28 | slot)
// ------------------------------------------------------------------
template <typename R>
MT_D bool prim_hit_t(const DevScene<R> &S, int code, const RayPre<R> &rp, R tmin, R tmax, R *t, R *u, R *v)
{
    int kind = code >> 28;
    int slot = code & 0x0FFFFFFF;
    *u = R(0);
    *v = R(0);
    switch (kind) {
    case KIND_TRIANGLE:
        return tri_t(S, slot, rp, tmin, tmax, t, u, v);
    case KIND_SPHERE:
        return sphere_t(S.spheres + 4 * (size_t)slot, rp, tmin, tmax, t);
    case KIND_BOX: {
        int ax, sg;
        return box_t(S.boxes + 6 * (size_t)slot, rp.o, rp.d, tmin, tmax, t, &ax, &sg);
    }
    case KIND_CYLINDER: {
        V3<R> n;
        return cylinder_hit(S.cyls + 8 * (size_t)slot, rp.o, rp.d, tmin, tmax, t, &n);
    }
    default:
        return false;
    }
}

template <typename R>
MT_D bool prim_occluded(const DevScene<R> &S, int code, const RayPre<R> &rp, R tmin, R tmax)
{
    int kind = code >> 28;
    int slot = code & 0x0FFFFFFF;
    R t, u, v;
    switch (kind) {
    case KIND_TRIANGLE:
        return tri_occ(S, slot, rp, tmin, tmax);
    case KIND_SPHERE:
        return sphere_t(S.spheres + 4 * (size_t)slot, rp, tmin, tmax, &t);
    case KIND_BOX:
        return box_occluded(S.boxes + 6 * (size_t)slot, rp.o, rp.d, tmin, tmax);
    case KIND_CYLINDER: {
        V3<R> n;
        return cylinder_hit(S.cyls + 8 * (size_t)slot, rp.o, rp.d, tmin, tmax, &t, &n);
    }
    default:
        return false;
    }
}

// ------------------------------------------------------------------
// Two-child slab test on one 64-byte node (bvh_slab_2way, src/bvh.c:495-533).
// ------------------------------------------------------------------
//
// FP32: one fma per slab plane (box * inv - o * inv). FP64: the reference's
// (box - o) * inv.
template <typename R>
MT_D void node_test(const float4 q0, const float4 q1, const float4 q2, const RayPre<R> &rp, R tmin, R tmax,
                    bool *hl, bool *hr, R *tl, R *tr);
template <>
MT_D void node_test<float>(const float4 q0, const float4 q1, const float4 q2, const RayPre<float> &rp, float tmin,
                           float tmax, bool *hl, bool *hr, float *tl, float *tr)
{
    float lx0 = fmaf(q0.x, rp.inv.x, -rp.oi.x), lx1 = fmaf(q0.y, rp.inv.x, -rp.oi.x);
    float ly0 = fmaf(q0.z, rp.inv.y, -rp.oi.y), ly1 = fmaf(q0.w, rp.inv.y, -rp.oi.y);
    float lz0 = fmaf(q2.x, rp.inv.z, -rp.oi.z), lz1 = fmaf(q2.y, rp.inv.z, -rp.oi.z);
    float rx0 = fmaf(q1.x, rp.inv.x, -rp.oi.x), rx1 = fmaf(q1.y, rp.inv.x, -rp.oi.x);
    float ry0 = fmaf(q1.z, rp.inv.y, -rp.oi.y), ry1 = fmaf(q1.w, rp.inv.y, -rp.oi.y);
    float rz0 = fmaf(q2.z, rp.inv.z, -rp.oi.z), rz1 = fmaf(q2.w, rp.inv.z, -rp.oi.z);
    // Entry clamped to tmin, exit to tmax: a child is hit when its clamped
    // entry is not past its clamped exit. For every ray whose entry and exit
    // are not NaN (a nonzero direction leaves at least one axis NaN-free) this
    // is the test lexit >= lenter && lexit >= tmin && lenter <= tmax, with the
    // entry distance max(lenter, tmin), in fewer instructions.
    const float lenter = fmax3f(fminf(lx0, lx1), fminf(ly0, ly1), fmaxf(fminf(lz0, lz1), tmin));
    const float lexit = fmin3f(fmaxf(lx0, lx1), fmaxf(ly0, ly1), fminf(fmaxf(lz0, lz1), tmax));
    const float renter = fmax3f(fminf(rx0, rx1), fminf(ry0, ry1), fmaxf(fminf(rz0, rz1), tmin));
    const float rexit = fmin3f(fmaxf(rx0, rx1), fmaxf(ry0, ry1), fminf(fmaxf(rz0, rz1), tmax));
    *hl = lenter <= lexit;
    *hr = renter <= rexit;
    *tl = lenter;
    *tr = renter;
}
template <>
MT_D void node_test<double>(const float4 q0, const float4 q1, const float4 q2, const RayPre<double> &rp, double tmin,
                            double tmax, bool *hl, bool *hr, double *tl, double *tr)
{
    using R = double;
    R lx0 = (R(q0.x) - rp.o.x) * rp.inv.x, lx1 = (R(q0.y) - rp.o.x) * rp.inv.x;
    R ly0 = (R(q0.z) - rp.o.y) * rp.inv.y, ly1 = (R(q0.w) - rp.o.y) * rp.inv.y;
    R lz0 = (R(q2.x) - rp.o.z) * rp.inv.z, lz1 = (R(q2.y) - rp.o.z) * rp.inv.z;
    R rx0 = (R(q1.x) - rp.o.x) * rp.inv.x, rx1 = (R(q1.y) - rp.o.x) * rp.inv.x;
    R ry0 = (R(q1.z) - rp.o.y) * rp.inv.y, ry1 = (R(q1.w) - rp.o.y) * rp.inv.y;
    R rz0 = (R(q2.z) - rp.o.z) * rp.inv.z, rz1 = (R(q2.w) - rp.o.z) * rp.inv.z;
    R lenter = mfmax(mfmax(mfmin(lx0, lx1), mfmin(ly0, ly1)), mfmin(lz0, lz1));
    R lexit = mfmin(mfmin(mfmax(lx0, lx1), mfmax(ly0, ly1)), mfmax(lz0, lz1));
    R renter = mfmax(mfmax(mfmin(rx0, rx1), mfmin(ry0, ry1)), mfmin(rz0, rz1));
    R rexit = mfmin(mfmin(mfmax(rx0, rx1), mfmax(ry0, ry1)), mfmax(rz0, rz1));
    *hl = (lexit >= lenter && lexit >= tmin && lenter <= tmax);
    *hr = (rexit >= renter && rexit >= tmin && renter <= tmax);
    *tl = lenter < tmin ? tmin : lenter;
    *tr = renter < tmin ? tmin : renter;
}

// ------------------------------------------------------------------
// BVH traversal.
//
// Each thread keeps its traversal stack in dynamic shared memory: entry k of
// thread t lives at mt_stack_smem[k * blockDim.x + t], so the 32 lanes of a
// warp touch 32 different banks. Every kernel that traverses launches with
// S.stack_depth * blockDim.x * 4 bytes of dynamic shared memory; the stack
// depth is the flattened tree's depth + 1, which bounds the stack by
// construction (a push only happens on the way down).
//
// Loop shape ("while-while", Aila and Laine, "Understanding the Efficiency of
// Ray Traversal on GPUs", HPG 2009): descend through inner nodes keeping the
// nearer child in a register and pushing the farther one, until the walk
// reaches a leaf; then test the leaf's primitives; then pop.
// ------------------------------------------------------------------
extern __shared__ int mt_stack_smem[];

static constexpr int kEmpty = (int)0x80000000;  // INT_MIN: no node

// Child code of a leaf: ~((first << 4) | (tri_only << 3) | count), count <= 7.
// For a triangle-only leaf `first` is the first triangle slot (the slots of
// one leaf are consecutive); otherwise it indexes the primitive references.
MT_HD int leaf_code(int first, int tri_only, int count) { return ~((first << 4) | (tri_only << 3) | count); }

template <typename R> MT_D int tri_prim_index(const DevScene<R> &S, int slot);
template <> MT_D int tri_prim_index<float>(const DevScene<float> &S, int slot)
{
    return __float_as_int(__ldg(&S.tri4[3 * (size_t)slot].w));
}
template <> MT_D int tri_prim_index<double>(const DevScene<double> &S, int slot) { return __ldg(S.tri_prim + slot); }

MT_D void count_add(unsigned long long *p, unsigned long long v)
{
    if (v) atomicAdd(p, v);
}

// Traversal work counters of one thread (flushed once per ray batch).
struct TravCount {
    unsigned long long nvis = 0, ntest = 0, ntri = 0;
};

template <typename R, bool ANY> MT_D void trav_count_flush(const DevScene<R> &S, TravCount &c)
{
    if (!S.counters) return;
    if (ANY) {
        count_add(&S.counters->any_node_visits, c.nvis);
        count_add(&S.counters->any_prim_tests, c.ntest);
        count_add(&S.counters->any_tri_tests, c.ntri);
    } else {
        count_add(&S.counters->node_visits, c.nvis);
        count_add(&S.counters->prim_tests, c.ntest);
        count_add(&S.counters->tri_tests, c.ntri);
    }
    c = TravCount();
}

// Resumable traversal of one ray: the walk advances one leaf at a time
// (trav_step), so a kernel can interleave rays on a lane.
template <typename R> struct Trav {
    RayPre<R> rp;
    R tmin, closest;
    int node;   // next node to visit, kEmpty when the walk is over
    int sp;     // stack entries in use
    bool found;
    int any_code;  // any hit: the tree primitive that blocked (kind << 28 | slot), -1 for a plane
    int any_leaf;  // any hit: the leaf (leaf_code) holding that primitive, -1 for a plane
};

// Nearest hit (ANY = false) or any hit (ANY = true) in [tmin, tmax].
// Nearest hit keeps the reference's semantics exactly: planes first
// (src/bvh.c:579-591), then the tree; each primitive is tested against
// [tmin, closest] and an equal t goes to the LOWEST prim_index
// (src/bvh.c:641-646). Node order and culling only change the amount of
// work, never the result. Any hit is bvh_occluded's boolean
// (src/bvh.c:714-813); the last-occluder cache there only reorders tests.
//
// trav_init tests the planes and sets the walk at the root.
template <typename R, bool ANY>
MT_D void trav_init(const DevScene<R> &S, Trav<R> &tv, const RayPre<R> &rp, R tmin, R tmax, Hit<R> *best,
                    TravCount &c)
{
    tv.rp = rp;
    tv.tmin = tmin;
    tv.closest = tmax;
    tv.found = false;
    tv.sp = 0;
    tv.any_code = -1;
    tv.any_leaf = -1;
    for (int i = 0; i < S.plane_count; ++i) {
        R t;
        ++c.ntest;
        if (plane_t(S.planes + 6 * (size_t)i, rp.o, rp.d, tmin, tv.closest, &t)) {
            int pi = S.plane_prims[i];
            if (ANY) {
                tv.found = true;
                break;
            }
            if (!tv.found || t < best->t || (t == best->t && pi < best->prim)) {
                best->t = t;
                best->u = R(0);
                best->v = R(0);
                best->prim = pi;
                best->code = (KIND_PLANE << 28) | i;
                tv.closest = t;
                tv.found = true;
            }
        }
    }
    tv.node = (S.node_count > 0 && !(ANY && tv.found)) ? 0 : kEmpty;
}

// Primitive tests of one leaf (code < 0, see leaf_code). REC (nearest hit):
// tv.any_leaf records the leaf of the current best hit.
template <typename R, bool ANY, bool REC = false>
MT_D void trav_leaf(const DevScene<R> &S, Trav<R> &tv, int node, Hit<R> *best, TravCount &c)
{
    const RayPre<R> &rp = tv.rp;
    const R tmin = tv.tmin;
    int leaf = ~node;
    int first = leaf >> 4, count = leaf & 7;
    if ((leaf >> 3) & 1) {
        for (int i = 0; i < count; ++i) {
            R t, u, v;
            ++c.ntest;
            ++c.ntri;
            const bool hit = ANY ? tri_occ(S, first + i, rp, tmin, tv.closest)
                                 : tri_t(S, first + i, rp, tmin, tv.closest, &t, &u, &v);
            if (hit) {
                if (ANY) {
                    tv.found = true;
                    tv.any_code = (KIND_TRIANGLE << 28) | (first + i);
                    tv.any_leaf = node;
                    break;
                }
                int pi = tri_prim_index(S, first + i);
                if (!tv.found || t < best->t || (t == best->t && pi < best->prim)) {
                    best->t = t;
                    best->u = u;
                    best->v = v;
                    best->prim = pi;
                    best->code = (KIND_TRIANGLE << 28) | (first + i);
                    tv.closest = t;
                    tv.found = true;
                    if (REC) tv.any_leaf = node;
                }
            }
        }
    } else {
        for (int i = 0; i < count; ++i) {
            int2 ref = __ldg(S.refs + first + i);
            R t, u, v;
            ++c.ntest;
            c.ntri += (ref.y >> 28) == KIND_TRIANGLE;
            bool hit = ANY ? prim_occluded(S, ref.y, rp, tmin, tv.closest)
                           : prim_hit_t(S, ref.y, rp, tmin, tv.closest, &t, &u, &v);
            if (hit) {
                if (ANY) {
                    tv.found = true;
                    tv.any_code = ref.y;
                    tv.any_leaf = node;
                    break;
                }
                if (!tv.found || t < best->t || (t == best->t && ref.x < best->prim)) {
                    best->t = t;
                    best->u = u;
                    best->v = v;
                    best->prim = ref.x;
                    best->code = ref.y;
                    tv.closest = t;
                    tv.found = true;
                    if (REC) tv.any_leaf = node;
                }
            }
        }
    }
}

// Descend the binary tree from `node` (nearer child in a register, farther
// child pushed) to the next leaf; kEmpty when the walk is over or the stack
// would overflow (error word set).
template <typename R>
MT_D int descend2(const DevScene<R> &S, const Trav<R> &tv, int node, int &sp, int *stk, int stride, TravCount &c)
{
    const int cap = S.stack_depth;
    while (node >= 0) {
        const float4 *Nd = S.nodes + 4 * (size_t)node;
        float4 q0 = __ldg(Nd), q1 = __ldg(Nd + 1), q2 = __ldg(Nd + 2);
        int4 q3 = __ldg(reinterpret_cast<const int4 *>(Nd + 3));
        bool hl, hr;
        R tl, tr;
        ++c.nvis;
        node_test(q0, q1, q2, tv.rp, tv.tmin, tv.closest, &hl, &hr, &tl, &tr);
        if (hl && hr) {
            bool lnear = tl <= tr;
            int nearc = lnear ? q3.x : q3.y;
            int farc = lnear ? q3.y : q3.x;
            if (sp >= cap) {
                atomicOr(S.err, ERR_STACK);
                return kEmpty;
            }
            stk[sp * stride] = farc;
            ++sp;
            node = nearc;
        } else if (hl) {
            node = q3.x;
        } else if (hr) {
            node = q3.y;
        } else {
            node = sp > 0 ? stk[--sp * stride] : kEmpty;
        }
    }
    return node;
}

// Slab test of one child box (the arithmetic of node_test).
template <typename R>
MT_D bool box_hit(float lx, float hx, float ly, float hy, float lz, float hz, const RayPre<R> &rp, R tmin, R tmax,
                  R *enter)
{
    static_assert(sizeof(R) == 4, "wide trees are an FP32 path");
    R x0 = fmaf(lx, rp.inv.x, -rp.oi.x), x1 = fmaf(hx, rp.inv.x, -rp.oi.x);
    R y0 = fmaf(ly, rp.inv.y, -rp.oi.y), y1 = fmaf(hy, rp.inv.y, -rp.oi.y);
    R z0 = fmaf(lz, rp.inv.z, -rp.oi.z), z1 = fmaf(hz, rp.inv.z, -rp.oi.z);
    R en = mfmax(mfmax(mfmin(x0, x1), mfmin(y0, y1)), mfmin(z0, z1));
    R ex = mfmin(mfmin(mfmax(x0, x1), mfmax(y0, y1)), mfmax(z0, z1));
    *enter = en < tmin ? tmin : en;
    return ex >= en && ex >= tmin && en <= tmax;
}

// Descend the wide tree (W = 4 or 8 children per node): test every child box,
// continue with the nearest hit child and push the other hit children
// farthest first, so they pop nearest first.
template <typename R, int W>
MT_D int descend_wide(const DevScene<R> &S, const Trav<R> &tv, int node, int &sp, int *stk, int stride,
                      TravCount &c)
{
    constexpr int G = W / 4;  // float4 words per coordinate row
    const int cap = S.wide_stack_depth;
    while (node >= 0) {
        const float4 *Nd = S.wnodes + (size_t)(8 * G) * node;
        ++c.nvis;
        R d[W];
        int ch[W];
        unsigned mask = 0;
#pragma unroll
        for (int g = 0; g < G; ++g) {
            const float4 lx = __ldg(Nd + 0 * G + g), hx = __ldg(Nd + 1 * G + g);
            const float4 ly = __ldg(Nd + 2 * G + g), hy = __ldg(Nd + 3 * G + g);
            const float4 lz = __ldg(Nd + 4 * G + g), hz = __ldg(Nd + 5 * G + g);
            const int4 cc = __ldg(reinterpret_cast<const int4 *>(Nd + 6 * G + g));
            const int b = 4 * g;
            ch[b] = cc.x;
            ch[b + 1] = cc.y;
            ch[b + 2] = cc.z;
            ch[b + 3] = cc.w;
            if (cc.x != kEmpty && box_hit(lx.x, hx.x, ly.x, hy.x, lz.x, hz.x, tv.rp, tv.tmin, tv.closest, &d[b]))
                mask |= 1u << b;
            if (cc.y != kEmpty && box_hit(lx.y, hx.y, ly.y, hy.y, lz.y, hz.y, tv.rp, tv.tmin, tv.closest, &d[b + 1]))
                mask |= 2u << b;
            if (cc.z != kEmpty && box_hit(lx.z, hx.z, ly.z, hy.z, lz.z, hz.z, tv.rp, tv.tmin, tv.closest, &d[b + 2]))
                mask |= 4u << b;
            if (cc.w != kEmpty && box_hit(lx.w, hx.w, ly.w, hy.w, lz.w, hz.w, tv.rp, tv.tmin, tv.closest, &d[b + 3]))
                mask |= 8u << b;
        }
        if (!mask) {
            node = sp > 0 ? stk[--sp * stride] : kEmpty;
            continue;
        }
        // nearest hit child
        R bd = R(3.0e38);
        int bi = 0, next = kEmpty;
#pragma unroll
        for (int i = 0; i < W; ++i)
            if (((mask >> i) & 1u) && d[i] < bd) {
                bd = d[i];
                bi = i;
                next = ch[i];
            }
        mask &= ~(1u << bi);
        if (sp + __popc(mask) > cap) {
            atomicOr(S.err, ERR_STACK);
            return kEmpty;
        }
        // the others, farthest first
        while (mask) {
            R fd = R(-1.0);
            int fi = 0, fc = kEmpty;
#pragma unroll
            for (int i = 0; i < W; ++i)
                if (((mask >> i) & 1u) && d[i] >= fd) {
                    fd = d[i];
                    fi = i;
                    fc = ch[i];
                }
            stk[sp * stride] = fc;
            ++sp;
            mask &= ~(1u << fi);
        }
        node = next;
    }
    return node;
}

// One while-while step: descend to a leaf, test it, pop the next node.
// Returns false once the walk is over. `stk` is this thread's stack (entry k
// at stk[k * stride]). W is the tree: 2 (binary `nodes`), 4 or 8 (`wnodes`).
template <typename R, bool ANY, int W = 2, bool REC = false>
MT_D bool trav_step(const DevScene<R> &S, Trav<R> &tv, int *stk, int stride, Hit<R> *best, TravCount &c)
{
    int sp = tv.sp;
    int node;
    if constexpr (W == 2)
        node = descend2(S, tv, tv.node, sp, stk, stride, c);
    else
        node = descend_wide<R, W>(S, tv, tv.node, sp, stk, stride, c);
    if (node == kEmpty) {
        tv.node = kEmpty;
        return false;
    }
    trav_leaf<R, ANY, REC>(S, tv, node, best, c);
    if (ANY && tv.found) {
        tv.node = kEmpty;
        return false;
    }
    node = sp > 0 ? stk[--sp * stride] : kEmpty;
    tv.node = node;
    tv.sp = sp;
    return node != kEmpty;
}

// The whole walk of one ray.
template <typename R, bool ANY, int W = 2>
MT_D bool traverse(const DevScene<R> &S, const RayPre<R> &rp, R tmin, R tmax, Hit<R> *best)
{
    TravCount c;
    Trav<R> tv;
    trav_init<R, ANY>(S, tv, rp, tmin, tmax, best, c);
    if (tv.node != kEmpty) {
        int *stk = mt_stack_smem + threadIdx.x;
        while (trav_step<R, ANY, W>(S, tv, stk, blockDim.x, best, c)) {
        }
    }
    trav_count_flush<R, ANY>(S, c);
    return tv.found;
}

template <typename R, int W = 2>
MT_D bool scene_nearest(const DevScene<R> &S, const RayPre<R> &rp, R tmin, R tmax, Hit<R> *best)
{
    return traverse<R, false, W>(S, rp, tmin, tmax, best);
}

template <typename R, int W = 2> MT_D bool scene_any(const DevScene<R> &S, const RayPre<R> &rp, R tmin, R tmax)
{
    Hit<R> dummy;
    return traverse<R, true, W>(S, rp, tmin, tmax, &dummy);
}

// Any hit among the primitives of one leaf (leaf_code; -1: none). Every
// primitive is tested against the same [tmin, tmax] as in the walk, so a hit
// here is a hit of the whole any-hit query.
template <typename R> MT_D bool leaf_occluded(const DevScene<R> &S, int node, const RayPre<R> &rp, R tmin, R tmax)
{
    const int leaf = ~node, first = leaf >> 4, count = leaf & 7;
    if ((leaf >> 3) & 1) {
        for (int i = 0; i < count; ++i)
            if (tri_occ(S, first + i, rp, tmin, tmax)) return true;
    } else {
        for (int i = 0; i < count; ++i)
            if (prim_occluded(S, __ldg(S.refs + first + i).y, rp, tmin, tmax)) return true;
    }
    return false;
}

// Any hit among the leaves of an occluder-cache entry: WAYS leaf codes, newest
// first, -1 for an empty way (entries fill from the front, and nothing but
// leaf codes and -1 is ever stored).
// Returns the way whose leaf blocks the ray, or -1. MOVE: a hit past the
// first way moves that leaf to the front (the entry is only an ordered set of
// candidates, so reordering it changes no answer).
template <typename R, int WAYS, bool MOVE = false>
MT_D int occ_ways_hit(const DevScene<R> &S, int *cache, const RayPre<R> &rp, R tmin, R tmax)
{
    int c[WAYS];
    if constexpr (WAYS == 4) {
        const int4 e = *reinterpret_cast<const int4 *>(cache);
        c[0] = e.x;
        c[1] = e.y;
        c[2] = e.z;
        c[3] = e.w;
    } else {
#pragma unroll
        for (int k = 0; k < WAYS; ++k) c[k] = cache[k];
    }
#pragma unroll
    for (int k = 0; k < WAYS; ++k) {
        if (c[k] == -1) return -1;
        if (leaf_occluded(S, c[k], rp, tmin, tmax)) {
            if constexpr (MOVE && WAYS == 4) {
                if (k > 0) {
                    int4 m;
                    m.x = c[k];
                    m.y = c[0];
                    m.z = k > 1 ? c[1] : c[2];
                    m.w = k > 2 ? c[2] : c[3];
                    *reinterpret_cast<int4 *>(cache) = m;
                }
            }
            return k;
        }
    }
    return -1;
}

template <typename R, int WAYS>
MT_D bool occ_ways_occluded(const DevScene<R> &S, const int *cache, const RayPre<R> &rp, R tmin, R tmax)
{
    int c[WAYS];
    if constexpr (WAYS == 4) {
        // a four-way entry is 16 bytes at a 16-byte boundary: one load
        const int4 e = *reinterpret_cast<const int4 *>(cache);
        c[0] = e.x;
        c[1] = e.y;
        c[2] = e.z;
        c[3] = e.w;
    } else {
#pragma unroll
        for (int k = 0; k < WAYS; ++k) c[k] = cache[k];
    }
#pragma unroll
    for (int k = 0; k < WAYS; ++k) {
        if (c[k] == -1) return false;  // entries fill from the front
        if (leaf_occluded(S, c[k], rp, tmin, tmax)) return true;
    }
    return false;
}

// Any hit that first tries the leaves in the entry `cache` (occ_ways_occluded)
// -- a hit there is a hit of the query, so the answer is the same -- and
// otherwise walks the tree and pushes the blocking leaf to the front of the
// entry. Caching leaves rather than single primitives catches the
// neighbouring primitives of a blocker, which nearby connections often meet
// instead. test_cached = false: the caller has already tested the entry.
template <typename R, int W = 2, int WAYS = 1>
MT_D bool scene_any_cached(const DevScene<R> &S, const RayPre<R> &rp, R tmin, R tmax, int *cache,
                           bool test_cached = true)
{
    const int c = cache[0];
    if (test_cached && occ_ways_occluded<R, WAYS>(S, cache, rp, tmin, tmax)) {
        if (S.counters) count_add(&S.counters->any_prim_tests, 1ull);
        return true;
    }
    TravCount cnt;
    Trav<R> tv;
    Hit<R> dummy;
    trav_init<R, true>(S, tv, rp, tmin, tmax, &dummy, cnt);
    if (tv.node != kEmpty) {
        int *stk = mt_stack_smem + threadIdx.x;
        while (trav_step<R, true, W>(S, tv, stk, blockDim.x, &dummy, cnt)) {
        }
    }
    trav_count_flush<R, true>(S, cnt);
    if (tv.found && tv.any_leaf != -1 && tv.any_leaf != c) {
        if constexpr (WAYS == 4) {
            const int4 e = *reinterpret_cast<const int4 *>(cache);
            *reinterpret_cast<int4 *>(cache) = make_int4(tv.any_leaf, e.x, e.y, e.z);
        } else {
#pragma unroll
            for (int k = WAYS - 1; k > 0; --k) cache[k] = cache[k - 1];
            cache[0] = tv.any_leaf;
        }
    }
    return tv.found;
}

// ------------------------------------------------------------------
// Pass-through shadow segments with an occluder cache (scenes with water or
// transparency > 0.8). The chain of pt_occluded_segment starts with the
// nearest hit over every primitive; when that hit is opaque the answer is
// "occluded". A cached opaque blocker P hit at t_P makes that certain as soon
// as no pass-through primitive is hit in [tmin, t_P]: the nearest hit is then
// at t <= t_P and opaque. The pass tree (DevScene::pass_root) answers that
// question over the pass-through primitives alone.
// ------------------------------------------------------------------

// Whether primitive `pi` lets a shadow ray through (src/pathtrace.c:514-516;
// a material index out of range stops the segment there).
template <typename R> MT_D bool prim_passes(const DevScene<R> &S, int pi)
{
    const int m = __ldg(S.prim_info + pi).y;
    if (m < 0 || m >= S.material_count) return false;
    const DevMaterial<R> &M = S.materials[m];
    return M.is_water || M.transparency > R(0.8);
}

// The nearest t in [tmin, tmax] among the opaque primitives of the cached
// leaves of a four-way entry (leaf codes of the main tree, newest first, -1
// empty); -1 when none is hit. Hits use the nearest-hit tests, so each t is
// the one the chain's first link would see.
template <typename R>
MT_D R occ_opaque_nearest(const DevScene<R> &S, const int *entry, const RayPre<R> &rp, R tmin, R tmax)
{
    const int4 e = *reinterpret_cast<const int4 *>(entry);
    const int c[4] = {e.x, e.y, e.z, e.w};
    R best = R(-1);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        if (c[k] == -1) break;
        const int leaf = ~c[k], first = leaf >> 4, count = leaf & 7;
        const bool tri_only = (leaf >> 3) & 1;
        for (int i = 0; i < count; ++i) {
            R t, u, v;
            int pi;
            bool hit;
            if (tri_only) {
                hit = tri_t(S, first + i, rp, tmin, tmax, &t, &u, &v);
                pi = hit ? tri_prim_index(S, first + i) : 0;
            } else {
                const int2 ref = __ldg(S.refs + first + i);
                hit = prim_hit_t(S, ref.y, rp, tmin, tmax, &t, &u, &v);
                pi = ref.x;
            }
            if (hit && (best < R(0) || t < best) && !prim_passes(S, pi)) best = t;
        }
    }
    return best;
}

// Whether some pass-through primitive is hit in [tmin, tmax] (nearest-hit
// tests over the pass tree; the walk stops at the first hit).
template <typename R> MT_D bool pass_hit(const DevScene<R> &S, const RayPre<R> &rp, R tmin, R tmax)
{
    if (S.pass_root < 0) return false;  // kEmptyPassTree (callers check kNoPassTree)
    TravCount cnt;
    Trav<R> tv;
    Hit<R> best;
    tv.rp = rp;
    tv.tmin = tmin;
    tv.closest = tmax;
    tv.found = false;
    tv.sp = 0;
    tv.any_code = -1;
    tv.any_leaf = -1;
    tv.node = S.pass_root;
    int *stk = mt_stack_smem + threadIdx.x;
    while (trav_step<R, false, 2>(S, tv, stk, blockDim.x, &best, cnt))
        if (tv.found) break;
    trav_count_flush<R, false>(S, cnt);
    return tv.found;
}

// scene_nearest (binary tree) that also returns the leaf of the nearest hit
// (-1 for a plane or no hit).
template <typename R>
MT_D bool scene_nearest_leaf(const DevScene<R> &S, const RayPre<R> &rp, R tmin, R tmax, Hit<R> *best, int *leaf)
{
    TravCount cnt;
    Trav<R> tv;
    trav_init<R, false>(S, tv, rp, tmin, tmax, best, cnt);
    if (tv.node != kEmpty) {
        int *stk = mt_stack_smem + threadIdx.x;
        while (trav_step<R, false, 2, true>(S, tv, stk, blockDim.x, best, cnt)) {
        }
    }
    trav_count_flush<R, false>(S, cnt);
    *leaf = tv.found ? tv.any_leaf : -1;
    return tv.found;
}

// scene_intersect / scene_occluded entry semantics: a direction that is not
// unit length (|d|^2 off by more than 1e-12) is normalised first
// (src/bvh.c:563-566, :720-723).
template <typename R> MT_D V3<R> unit_dir(V3<R> d)
{
    R len_sq = length_sq(d);
    if (len_sq > R(0) && mfabs(len_sq - R(1)) > R(1e-12)) d = normalize(d);
    return d;
}

// Full hit record of the reference (Hit, src/geometry.h:74-83).
template <typename R> struct SurfaceHit {
    R t;
    V3<R> point;
    V3<R> normal;   // unit, facing the incoming ray
    int prim;
    int material;
    int front_face;
    int code;       // kind << 28 | slot (hit_uv)
    R bu, bv;       // triangle barycentrics of the traversal hit (hit_uv)
};

// geo_store_hit (src/geometry.c:78-91): orient the unit normal against the ray.
template <typename R>
MT_D void store_hit(SurfaceHit<R> *out, R t, V3<R> point, V3<R> n, V3<R> d)
{
    bool front = dot(d, n) < R(0);
    out->t = t;
    out->point = point;
    out->normal = front ? n : neg(n);
    out->front_face = front ? 1 : 0;
}

// Recover point / normal / front face / material for a traversal hit.
template <typename R>
MT_D void finish_hit(const DevScene<R> &S, V3<R> o, V3<R> d, const Hit<R> &h, SurfaceHit<R> *out)
{
    int kind = h.code >> 28;
    int slot = h.code & 0x0FFFFFFF;
    out->prim = h.prim;
    out->material = __ldg(S.prim_info + h.prim).y;
    out->code = h.code;
    out->bu = h.u;
    out->bv = h.v;
    V3<R> point = at(o, d, h.t);
    switch (kind) {
    case KIND_SPHERE: {
        const R *s = S.spheres + 4 * (size_t)slot;
        V3<R> n = scale(sub(point, v3(s[0], s[1], s[2])), R(1) / s[3]);
        store_hit(out, h.t, point, n, d);
        break;
    }
    case KIND_PLANE: {
        const R *p = S.planes + 6 * (size_t)slot;
        store_hit(out, h.t, point, v3(p[3], p[4], p[5]), d);
        break;
    }
    case KIND_BOX: {
        R t;
        int axis = -1, sign = 0;
        box_t(S.boxes + 6 * (size_t)slot, o, d, h.t, h.t, &t, &axis, &sign);
        V3<R> n;
        if (axis < 0) {
            n = neg(d);
        } else {
            n = v3(R(0), R(0), R(0));
            if (axis == 0) n.x = R(sign);
            else if (axis == 1) n.y = R(sign);
            else n.z = R(sign);
        }
        store_hit(out, h.t, point, n, d);
        break;
    }
    case KIND_CYLINDER: {
        R t;
        V3<R> n;
        cylinder_hit(S.cyls + 8 * (size_t)slot, o, d, h.t, h.t, &t, &n);
        store_hit(out, h.t, point, n, d);
        break;
    }
    case KIND_TRIANGLE:
    default: {
        V3<R> e1, e2;
        bool smooth;
        if constexpr (sizeof(R) == 8) {
            const R *T = S.tris + 9 * (size_t)slot;
            e1 = v3(T[3], T[4], T[5]);
            e2 = v3(T[6], T[7], T[8]);
            smooth = S.tri_smooth[slot] != 0;
        } else {
            const float4 *T = S.tri4 + 3 * (size_t)slot;
            float4 a = __ldg(T), b = __ldg(T + 1), c = __ldg(T + 2);
            e1 = v3<R>(b.x - a.x, b.y - a.y, b.z - a.z);
            e2 = v3<R>(c.x - a.x, c.y - a.y, c.z - a.z);
            smooth = __float_as_int(b.w) != 0;
        }
        V3<R> n;
        bool have = false;
        if (smooth) {
            const R *N = S.tri_normals + 9 * (size_t)slot;
            R w = R(1) - h.u - h.v;
            n = add(scale(v3(N[0], N[1], N[2]), w), add(scale(v3(N[3], N[4], N[5]), h.u), scale(v3(N[6], N[7], N[8]), h.v)));
            R nlen = length(n);
            if (nlen > R(1e-12)) {
                n = scale(n, R(1) / nlen);
                have = true;
            }
        }
        if (!have) {
            n = cross(e1, e2);
            R nlen = length(n);
            n = (nlen > R(0)) ? scale(n, R(1) / nlen) : v3(R(0), R(1), R(0));
        }
        store_hit(out, h.t, point, n, d);
        break;
    }
    }
}

// scene_intersect (src/scene.c:767-775) with the full hit record.
// The reference's hit (u, v) for UV-mapped textures: sphere longitude /
// latitude (src/geometry.c:359-366), plane tangent coordinates (:383-390),
// box face coordinates (:463-476), cylinder cap disc or side angle / height
// (:665-696), triangle barycentrics or interpolated vertex UVs (:526-534).
// o, d: the ray of the hit (d unit); h: the traversal hit.
template <typename R> MT_D V3<R> uv_tangent(V3<R> n, V3<R> *b)
{
    V3<R> up = (mfabs(n.y) > R(0.9)) ? v3(R(0), R(0), R(1)) : v3(R(0), R(1), R(0));
    V3<R> t = normalize(cross(up, n));
    *b = cross(n, t);
    return t;
}

template <typename R>
MT_NOINLINE void hit_uv(const DevScene<R> &S, V3<R> o, V3<R> d, const Hit<R> &h, R *u_out, R *v_out)
{
    const int kind = h.code >> 28;
    const int slot = h.code & 0x0FFFFFFF;
    const V3<R> point = at(o, d, h.t);
    const R two_pi = R(2) * R(3.14159265358979323846);
    R u = R(0), v = R(0);
    switch (kind) {
    case KIND_SPHERE: {
        const R *s = S.spheres + 4 * (size_t)slot;
        V3<R> n = scale(sub(point, v3(s[0], s[1], s[2])), R(1) / s[3]);
        R phi = matan2(n.z, n.x);
        R theta = masin(mfmax(R(-1), mfmin(R(1), n.y)));
        u = R(0.5) + phi / two_pi;
        v = R(0.5) + theta / R(3.14159265358979323846);
        u = u - mfloor(u);
        v = mfmax(R(0), mfmin(R(1), v));
        break;
    }
    case KIND_PLANE: {
        const R *p = S.planes + 6 * (size_t)slot;
        V3<R> n = v3(p[3], p[4], p[5]), B;
        V3<R> T = uv_tangent(n, &B);
        V3<R> diff = sub(point, v3(p[0], p[1], p[2]));
        u = dot(diff, T);
        v = dot(diff, B);
        u = u - mfloor(u);
        v = v - mfloor(v);
        break;
    }
    case KIND_BOX: {
        const R *b = S.boxes + 6 * (size_t)slot;
        R t;
        int axis = -1, sign = 0;
        box_t(b, o, d, h.t, h.t, &t, &axis, &sign);
        const R lo[3] = {b[0] - b[3], b[1] - b[4], b[2] - b[5]};
        const R hi[3] = {b[0] + b[3], b[1] + b[4], b[2] + b[5]};
        const R dx = hi[0] - lo[0], dy = hi[1] - lo[1], dz = hi[2] - lo[2];
        if (axis == 0) {
            u = (dz > R(1e-12)) ? (point.z - lo[2]) / dz : R(0);
            v = (dy > R(1e-12)) ? (point.y - lo[1]) / dy : R(0);
        } else if (axis == 1) {
            u = (dx > R(1e-12)) ? (point.x - lo[0]) / dx : R(0);
            v = (dz > R(1e-12)) ? (point.z - lo[2]) / dz : R(0);
        } else {
            u = (dx > R(1e-12)) ? (point.x - lo[0]) / dx : R(0);
            v = (dy > R(1e-12)) ? (point.y - lo[1]) / dy : R(0);
        }
        u = mfmax(R(0), mfmin(R(1), u));
        v = mfmax(R(0), mfmin(R(1), v));
        break;
    }
    case KIND_CYLINDER: {
        const R *c = S.cyls + 8 * (size_t)slot;
        R t;
        V3<R> n;
        CylPart<R> part;
        part.is_cap = 0;
        part.cap = 0;
        part.s = R(0);
        cylinder_hit(c, o, d, h.t, h.t, &t, &n, &part);
        const V3<R> pa = v3(c[0], c[1], c[2]), pb = v3(c[3], c[4], c[5]);
        const V3<R> A = sub(pb, pa);
        const R hgt = length(A);
        const V3<R> axis = scale(A, R(1) / hgt);
        V3<R> B;
        V3<R> T = uv_tangent(axis, &B);
        if (part.is_cap) {
            const V3<R> cap_center = part.cap == 0 ? pa : pb;
            const R r_cap = part.cap == 0 ? c[6] : c[7];
            V3<R> radial = sub(point, cap_center);
            R rx = (r_cap > R(1e-12)) ? dot(radial, T) / (R(2) * r_cap) : R(0);
            R ry = (r_cap > R(1e-12)) ? dot(radial, B) / (R(2) * r_cap) : R(0);
            u = mfmax(R(0), mfmin(R(1), R(0.5) + rx));
            v = mfmax(R(0), mfmin(R(1), R(0.5) + ry));
        } else {
            V3<R> axis_pt = add(pa, scale(axis, part.s * hgt));
            V3<R> radial = sub(point, axis_pt);
            R phi = matan2(dot(radial, B), dot(radial, T));
            u = R(0.5) + phi / two_pi;
            u = u - mfloor(u);
            v = mfmax(R(0), mfmin(R(1), part.s));
        }
        break;
    }
    case KIND_TRIANGLE:
    default: {
        u = h.u;
        v = h.v;
        if (S.tri_uv) {
            const R *q = S.tri_uv + 6 * (size_t)slot;
            if (q[0] == q[0]) {  // not NaN: the triangle has vertex UVs
                R w = R(1) - h.u - h.v;
                u = w * q[0] + h.u * q[2] + h.v * q[4];
                v = w * q[1] + h.u * q[3] + h.v * q[5];
            }
        }
        break;
    }
    }
    *u_out = u;
    *v_out = v;
}

template <typename R>
MT_D bool scene_intersect(const DevScene<R> &S, V3<R> o, V3<R> d, R tmin, R tmax, SurfaceHit<R> *out)
{
    d = unit_dir(d);
    RayPre<R> rp = ray_pre(o, d);
    Hit<R> h;
    if (S.counters) atomicAdd(&S.counters->extension_rays, 1ull);
    if (!scene_nearest(S, rp, tmin, tmax, &h)) return false;
    finish_hit(S, o, d, h, out);
    return true;
}

// What a link of a pass-through shadow chain reads of scene_intersect's hit
// record: t, the hit point and the material, with finish_hit's values for
// them (the normal and texture terms are not computed). `leaf` (optional):
// the leaf of the hit, as scene_nearest_leaf.
template <typename R> struct LinkHit {
    R t;
    V3<R> point;
    int material;
};
template <typename R>
MT_D bool scene_link(const DevScene<R> &S, V3<R> o, V3<R> d, R tmin, R tmax, LinkHit<R> *out, int *leaf = nullptr)
{
    d = unit_dir(d);
    const RayPre<R> rp = ray_pre(o, d);
    Hit<R> h;
    int lf;
    if (S.counters) atomicAdd(&S.counters->extension_rays, 1ull);
    // one walk for every link (the leaf is recorded either way)
    const bool found = scene_nearest_leaf(S, rp, tmin, tmax, &h, &lf);
    if (leaf) *leaf = lf;
    if (!found) return false;
    out->t = h.t;
    out->point = at(o, d, h.t);
    out->material = __ldg(S.prim_info + h.prim).y;
    return true;
}

// scene_occluded (src/scene.c:804-811).
template <typename R> MT_D bool scene_occluded(const DevScene<R> &S, V3<R> o, V3<R> d, R tmin, R tmax)
{
    d = unit_dir(d);
    RayPre<R> rp = ray_pre(o, d);
    if (S.counters) atomicAdd(&S.counters->shadow_rays, 1ull);
    return scene_any(S, rp, tmin, tmax);
}

// primitive_intersect on one emissive-light sphere by prim_index
// (src/pathtrace.c:594, src/render.c:536): only the distance is needed.
template <typename R>
MT_D bool light_sphere_t(const DevScene<R> &S, int prim, V3<R> o, V3<R> d, R tmin, R tmax, R *t)
{
    d = unit_dir(d);
    int2 info = __ldg(S.prim_info + prim);
    int slot = info.x & 0x0FFFFFFF;
    RayPre<R> rp;
    rp.o = o;
    rp.d = d;
    return sphere_t(S.spheres + 4 * (size_t)slot, rp, tmin, tmax, t);
}

}  // namespace mt
