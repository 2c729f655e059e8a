// mt_math.cuh - scalar / vector math and the hash PRNG of the device path.
//
// Everything is templated on the arithmetic type R (float for the production
// path, double for the exact-parity path). The double instantiation follows
// the reference's expression order operation by operation (src/vec3.h,
// src/vec3.c), and is compiled with --fmad=false, so add / mul / div / sqrt
// round exactly as the reference's x86-64 build does.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#define MT_HD __host__ __device__ __forceinline__
#define MT_D __device__ __forceinline__
// Rare, large paths (textures, fog, volumetric media) stay out of line, so the
// common path of the kernels that can reach them keeps its registers.
#define MT_NOINLINE __device__ __noinline__

namespace mt {

// ------------------------------------------------------------------
// Scalar helpers with explicit float / double overloads, so no float
// expression is ever silently promoted to double.
// ------------------------------------------------------------------
MT_D float msqrt(float x) { return sqrtf(x); }
MT_D double msqrt(double x) { return sqrt(x); }
MT_D float mfabs(float x) { return fabsf(x); }
MT_D double mfabs(double x) { return fabs(x); }
MT_D float mfmin(float a, float b) { return fminf(a, b); }
MT_D double mfmin(double a, double b) { return fmin(a, b); }
MT_D float mfmax(float a, float b) { return fmaxf(a, b); }
MT_D double mfmax(double a, double b) { return fmax(a, b); }
// Three-input min / max (one instruction on sm_100): the same value as two
// fminf / fmaxf, NaN inputs ignored as there.
MT_D float fmin3f(float a, float b, float c)
{
    float r;
    asm("min.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}
MT_D float fmax3f(float a, float b, float c)
{
    float r;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}
MT_D float mfloor(float x) { return floorf(x); }
MT_D double mfloor(double x) { return floor(x); }
MT_D float mpow(float a, float b) { return powf(a, b); }
MT_D double mpow(double a, double b) { return pow(a, b); }
MT_D float mexp(float x) { return expf(x); }
MT_D double mexp(double x) { return exp(x); }
MT_D float mcos(float x) { return cosf(x); }
MT_D double mcos(double x) { return cos(x); }
MT_D float msin(float x) { return sinf(x); }
MT_D double msin(double x) { return sin(x); }
MT_D float mtan(float x) { return tanf(x); }
MT_D double mtan(double x) { return tan(x); }
MT_D float matan2(float y, float x) { return atan2f(y, x); }
MT_D double matan2(double y, double x) { return atan2(y, x); }
MT_D float masin(float x) { return asinf(x); }
MT_D double masin(double x) { return asin(x); }
MT_D bool misfinite(float x) { return isfinite(x); }
MT_D bool misfinite(double x) { return isfinite(x); }
MT_D void msincos(float x, float *s, float *c) { sincosf(x, s, c); }
MT_D void msincos(double x, double *s, double *c)
{
    // Two separate calls, as the reference evaluates cos() and sin().
    *c = cos(x);
    *s = sin(x);
}

template <typename R> struct Const {
    static constexpr R pi = R(3.14159265358979323846);
};

// ------------------------------------------------------------------
// 3-vector (reference Vec3, src/vec3.h:17-19)
// ------------------------------------------------------------------
template <typename R> struct V3 {
    R x, y, z;
};

template <typename R> MT_HD V3<R> v3(R x, R y, R z) { return V3<R>{x, y, z}; }
template <typename R> MT_HD V3<R> add(V3<R> a, V3<R> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <typename R> MT_HD V3<R> sub(V3<R> a, V3<R> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <typename R> MT_HD V3<R> neg(V3<R> a) { return {-a.x, -a.y, -a.z}; }
template <typename R> MT_HD V3<R> scale(V3<R> a, R s) { return {a.x * s, a.y * s, a.z * s}; }
template <typename R> MT_HD V3<R> mul(V3<R> a, V3<R> b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
template <typename R> MT_HD R dot(V3<R> a, V3<R> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <typename R> MT_HD V3<R> cross(V3<R> a, V3<R> b)
{
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
template <typename R> MT_HD R length_sq(V3<R> a) { return dot(a, a); }
// vec3_lerp: a + (b - a) * t (src/vec3.h:95-100)
template <typename R> MT_HD V3<R> lerp(V3<R> a, V3<R> b, R t)
{
    return {a.x + (b.x - a.x) * t, a.y + (b.y - a.y) * t, a.z + (b.z - a.z) * t};
}
// vec3_reflect: i - 2 (i.n) n (src/vec3.h:105-111)
template <typename R> MT_HD V3<R> reflect(V3<R> i, V3<R> n)
{
    R d = dot(i, n);
    return {i.x - R(2) * d * n.x, i.y - R(2) * d * n.y, i.z - R(2) * d * n.z};
}
// vec3_at: o + t d (src/vec3.h:114-119)
template <typename R> MT_HD V3<R> at(V3<R> o, V3<R> d, R t)
{
    return {o.x + t * d.x, o.y + t * d.y, o.z + t * d.z};
}
template <typename R> MT_D R length(V3<R> a) { return msqrt(length_sq(a)); }
// vec3_normalize: zero when |a|^2 <= 1e-12, else a * (1/sqrt(|a|^2)) (src/vec3.c:29-37)
template <typename R> MT_D V3<R> normalize(V3<R> a)
{
    R len_sq = length_sq(a);
    if (len_sq <= R(1e-12)) return {R(0), R(0), R(0)};
    return scale(a, R(1) / msqrt(len_sq));
}
template <typename R> MT_D bool finite3(V3<R> v) { return misfinite(v.x) && misfinite(v.y) && misfinite(v.z); }

template <typename R> MT_D V3<R> load3(const R *p) { return {p[0], p[1], p[2]}; }

// ------------------------------------------------------------------
// Hash PRNG (pt_hash_u32 / pt_hash3 / pt_rand01, src/pathtrace.c:92-117,
// identical to render_hash_u32 / render_hash3 / render_rand01,
// src/render.c:371-396). Every uniform is (h >> 8) / 2^24, a 24-bit dyadic
// rational, so it is exact in both float and double: both device paths draw
// the reference's random stream bit for bit.
// ------------------------------------------------------------------
MT_HD uint32_t hash_u32(uint32_t x)
{
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}

MT_HD uint32_t hash3(uint32_t a, uint32_t b, uint32_t c)
{
    uint32_t h = 0x9e3779b9u;
    h ^= hash_u32(a + 0x85ebca6bu);
    h = hash_u32(h + b);
    h ^= hash_u32(c + 0xc2b2ae35u);
    return hash_u32(h);
}

template <typename R> MT_HD R rand01(uint32_t a, uint32_t b, uint32_t c)
{
    return R(hash3(a, b, c) >> 8) * R(1.0 / 16777216.0);
}

// Clamp helpers of the reference (pt_clamp01 / pt_clamp, src/pathtrace.c:141-154;
// clamp01 in src/material.c:25-30 differs: it does NOT map NaN to 0).
template <typename R> MT_D R pt_clamp01(R v)
{
    if (!(v > R(0))) return R(0);
    if (v > R(1)) return R(1);
    return v;
}
template <typename R> MT_D R pt_clamp(R v, R lo, R hi)
{
    if (!(v > lo)) return lo;
    if (v > hi) return hi;
    return v;
}
template <typename R> MT_D R mat_clamp01(R v)
{
    if (v < R(0)) return R(0);
    if (v > R(1)) return R(1);
    return v;
}

}  // namespace mt
