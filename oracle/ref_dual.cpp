/*
 * ref_dual.cpp - forward-mode (dual-number) differentiation of the reference
 * path tracer, the oracle for the path-replay adjoint.
 *
 * TEST INFRASTRUCTURE ONLY (see ref_harness.h). The reference's own
 * src/pathtrace.c is compiled into this unit (inside namespace refpt), so the
 * ray generation, random streams, BVH queries, shadow segments and BSDF
 * direction sampling are the reference's code. What depends on the
 * differentiated parameters -- per-material albedo, roughness, metallic and
 * emissive, absorption, and the sun radiance -- is restated below on a dual number
 * (value, tangent), following the reference line by line:
 *   pathtrace_radiance          src/pathtrace.c:800-1028
 *   pt_nee_sun / pt_nee_emissive src/pathtrace.c:534-606
 *   pt_sample_pbr / _legacy weights src/pathtrace.c:251-421
 *   material_shade_local / _pbr src/material.c:157-188, 234-290
 *   sky_sample (2D clouds)      src/material.c:473-590
 *
 * The estimator is the one the adjoint differentiates (detached sampling):
 * directions, lobe choices, lobe and direction pdfs and roulette
 * probabilities are the primal values; BSDF weights, shading, emission and
 * the sky carry tangents. Clamps pass a tangent only strictly inside their
 * range (a parameter sitting on a bound, e.g. metallic = 1, has zero
 * derivative), as the adjoint does.
 *
 * mtdual_pathtrace_grad seeds one parameter at a time and returns
 *   grad[j] = sum_pixels sum_samples adj(pixel) . scale . dL_sample / dtheta_j
 * which is what mt_adjoint_backward computes with scale = 1 / spp. The value
 * part of every sample is checked against the reference pathtrace_radiance and the
 * count of samples whose value differs is returned: it must be zero.
 */
#include <math.h>
#include <stddef.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#include <unistd.h>

extern "C" {
#include "camera.h"
#include "geometry.h"
#include "material.h"
#include "noise.h"
#include "render.h"
#include "sampling.h"
#include "scene.h"
#include "texture.h"
#include "vec3.h"

#include "ref_harness.h"
}

// pathtrace.h declares its three entry points with C linkage; they are
// renamed for this second copy so they do not collide with the C harness's.
#define pathtrace_radiance refpt_pathtrace_radiance
#define pathtrace_to_byte refpt_pathtrace_to_byte
#define pathtrace_render refpt_pathtrace_render
namespace refpt {
#include "pathtrace.c"
}
#undef pathtrace_radiance
#undef pathtrace_to_byte
#undef pathtrace_render

namespace {

// ---------------------------------------------------------------- dual numbers
struct D {
    double v, d;
};
inline D dc(double v) { return {v, 0.0}; }
inline D operator+(D a, D b) { return {a.v + b.v, a.d + b.d}; }
inline D operator-(D a, D b) { return {a.v - b.v, a.d - b.d}; }
inline D operator*(D a, D b) { return {a.v * b.v, a.d * b.v + a.v * b.d}; }
inline D operator/(D a, D b)
{
    double q = a.v / b.v;
    return {q, (a.d - q * b.d) / b.v};
}
inline D operator+(D a, double b) { return {a.v + b, a.d}; }
inline D operator+(double a, D b) { return {a + b.v, b.d}; }
inline D operator-(D a, double b) { return {a.v - b, a.d}; }
inline D operator-(double a, D b) { return {a - b.v, -b.d}; }
inline D operator*(D a, double b) { return {a.v * b, a.d * b}; }
inline D operator*(double a, D b) { return {a * b.v, a * b.d}; }
inline D operator/(D a, double b) { return {a.v / b, a.d / b}; }
inline D operator/(double a, D b)
{
    double q = a / b.v;
    return {q, -q * b.d / b.v};
}

struct DV3 {
    D x, y, z;
};
inline DV3 dv(Vec3 a) { return {dc(a.x), dc(a.y), dc(a.z)}; }
inline Vec3 val(const DV3 &a) { return vec3(a.x.v, a.y.v, a.z.v); }
inline DV3 add(const DV3 &a, const DV3 &b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline DV3 sub(const DV3 &a, const DV3 &b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline DV3 mul(const DV3 &a, const DV3 &b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
inline DV3 mul(const DV3 &a, Vec3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
inline DV3 mul(Vec3 a, const DV3 &b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
inline DV3 scale(const DV3 &a, D s) { return {a.x * s, a.y * s, a.z * s}; }
inline DV3 scale(const DV3 &a, double s) { return {a.x * s, a.y * s, a.z * s}; }
inline DV3 scale(Vec3 a, D s) { return {a.x * s, a.y * s, a.z * s}; }
// vec3_lerp (src/vec3.h:93-98): a + (b - a) * t
inline DV3 lerp(const DV3 &a, const DV3 &b, D t)
{
    return {a.x + (b.x - a.x) * t, a.y + (b.y - a.y) * t, a.z + (b.z - a.z) * t};
}
inline DV3 lerp(const DV3 &a, const DV3 &b, double t)
{
    return {a.x + (b.x - a.x) * t, a.y + (b.y - a.y) * t, a.z + (b.z - a.z) * t};
}

// clamp to [0, 1] with the reference's value; the tangent passes strictly inside
inline D clamp01_d(D v)
{
    if (!(v.v > 0.0)) return dc(v.v < 0.0 || v.v != v.v ? 0.0 : v.v);
    if (v.v > 1.0) return dc(1.0);
    if (v.v < 1.0) return v;
    return dc(v.v);
}

constexpr double kMaterialPi = 3.14159265358979323846;  // MATERIAL_PI, src/material.c:16

// material.c file statics (src/material.c:25-48)
inline double clamp01(double v) { return v < 0.0 ? 0.0 : (v > 1.0 ? 1.0 : v); }
inline double smoothstep(double e0, double e1, double x)
{
    double denom = e1 - e0;
    if (denom == 0.0) return x < e0 ? 0.0 : 1.0;
    double t = clamp01((x - e0) / denom);
    return t * t * (3.0 - 2.0 * t);
}
inline double pow_nonneg(double b, double e) { return b <= 0.0 ? 0.0 : pow(b, e); }

// ---------------------------------------------------------------- parameters
struct DMat {
    DV3 albedo, emissive, absorption;
    D roughness, metallic;
};

inline D dexp(D a)
{
    double e = exp(a.v);
    return {e, e * a.d};
}

// water_transmittance (src/material.c:1223-1236) with a tangent. The
// reference returns 1 for a zero coefficient; exp(-0 * d) is that same 1, and
// the derivative there is the limit -d (what finite differences see).
inline D water_transmittance_d(D a, double depth)
{
    D t = dexp(-1.0 * a * depth);
    if (!(t.v > 0.0)) return dc(0.0);
    if (t.v > 1.0) return dc(1.0);
    return t;
}

struct Params {
    const Scene *scene;
    DMat *mats;
    DV3 sun_color;
};

// material_roughness_to_alpha (src/material.c:227-232)
inline D roughness_to_alpha_d(D r)
{
    D c = clamp01_d(r);
    D a = c * c;
    return a.v < 1e-4 ? dc(1e-4) : a;
}

// material_shade_local (src/material.c:157-188)
DV3 shade_local_d(const Material *m, const DMat &p, Vec3 N, Vec3 L, Vec3 V, const DV3 &light)
{
    DV3 zero = dv(vec3(0.0, 0.0, 0.0));
    double ndl = vec3_dot(N, L);
    if (ndl <= 0.0) return zero;
    DV3 diffuse = scale(mul(p.albedo, light), ndl);
    Vec3 h = vec3_add(L, V);
    DV3 spec = zero;
    if (vec3_length_sq(h) > 1e-12) {
        Vec3 H = vec3_normalize(h);
        double ndh = vec3_dot(N, H);
        if (ndh > 0.0) {
            double spec_term = pow_nonneg(ndh, m->shininess);
            spec = scale(mul(m->specular, light), spec_term);
        }
    }
    return add(diffuse, spec);
}

// material_shade_pbr (src/material.c:234-290)
DV3 shade_pbr_d(const DMat &p, Vec3 N, Vec3 L, Vec3 V, const DV3 &light)
{
    DV3 zero = dv(vec3(0.0, 0.0, 0.0));
    double ndl = vec3_dot(N, L);
    if (ndl <= 0.0) return zero;
    double ndv = vec3_dot(N, V);
    if (ndv <= 0.0) return zero;
    D metallic = clamp01_d(p.metallic);
    D alpha = roughness_to_alpha_d(p.roughness);
    Vec3 h = vec3_add(L, V);
    double ndh = 0.0;
    if (vec3_length_sq(h) > 1e-12) {
        ndh = vec3_dot(N, vec3_normalize(h));
        if (ndh < 0.0) ndh = 0.0;
    }
    DV3 f0 = lerp(dv(vec3(0.04, 0.04, 0.04)), p.albedo, metallic);
    // fresnel_schlick_rgb (src/material.c:142-152): f0 + (1 - f0) * k
    double c = clamp01(ndv);
    double mm = 1.0 - c;
    double m2 = mm * mm;
    double k = m2 * m2 * mm;
    DV3 F = {f0.x + (1.0 - f0.x) * k, f0.y + (1.0 - f0.y) * k, f0.z + (1.0 - f0.z) * k};
    // d_ggx (src/material.c:203-208)
    D a2 = alpha * alpha;
    D dd = ndh * ndh * (a2 - 1.0) + 1.0;
    D Dg = a2 / (kMaterialPi * dd * dd);
    // g_smith_schlick (src/material.c:213-221) on clamp01(roughness)
    D r = clamp01_d(p.roughness);
    D kk = (r + 1.0) * (r + 1.0) / 8.0;
    if (kk.v < 0.0) kk = dc(0.0);
    else if (kk.v > 1.0) kk = dc(1.0);
    D gl = ndl / (ndl * (1.0 - kk) + kk);
    D gv = ndv / (ndv * (1.0 - kk) + kk);
    D G = gl * gv;
    double denom = 4.0 * ndl * ndv;
    D spec_scale = denom > 0.0 ? Dg * G / denom : dc(0.0);
    DV3 spec = scale(F, spec_scale);
    DV3 kd = scale(sub(dv(vec3(1.0, 1.0, 1.0)), F), 1.0 - metallic);
    DV3 f_diff = scale(mul(kd, p.albedo), 1.0 / kMaterialPi);
    DV3 f = add(f_diff, spec);
    return scale(mul(light, f), ndl);
}

inline DV3 shade_d(const Material *m, const DMat &p, Vec3 N, Vec3 L, Vec3 V, const DV3 &light)
{
    return m->pbr ? shade_pbr_d(p, N, L, V, light) : shade_local_d(m, p, N, L, V, light);
}

// sky_sample (src/material.c:473-590), planar clouds; sun_color carries tangents
DV3 sky_sample_d(Vec3 dir, const SkyParams *sky, const DV3 &sun_color)
{
    double hh = clamp01(dir.y);
    double t = pow_nonneg(hh, sky->gradient_gamma);
    DV3 base = dv(vec3_lerp(sky->horizon_color, sky->zenith_color, t));
    double cos_sun = vec3_dot(dir, sky->sun_dir);
    if (cos_sun > 0.0) {
        double glow = pow_nonneg(cos_sun, sky->sun_glow_exponent) * sky->sun_glow_strength;
        base = add(base, scale(sun_color, glow));
    }
    const double cloud_eps = 0.03;
    if (dir.y > cloud_eps) {
        double tt = sky->cloud_height / dir.y;
        double px = dir.x * tt;
        double pz = dir.z * tt;
        int octaves = sky->cloud_octaves;
        if (octaves < 1) octaves = 1;
        double raw = noise_fbm2(px * sky->cloud_scale, pz * sky->cloud_scale, octaves, 2.0, 0.5, sky->seed);
        double density = clamp01(0.5 * (raw + 1.0));
        double a = sky->cloud_coverage - sky->cloud_softness;
        double b = sky->cloud_coverage + sky->cloud_softness;
        double alpha = smoothstep(a, b, density);
        alpha = pow_nonneg(alpha, sky->cloud_sharpness);
        alpha *= smoothstep(0.0, 0.15, dir.y);
        if (alpha > 0.0) {
            double shadow = 0.6 + 0.4 * alpha;
            Vec3 cloud_color = vec3_scale(vec3(0.95, 0.95, 0.98), shadow);
            double lit = cos_sun > 0.0 ? cos_sun : 0.0;
            DV3 lit_cloud = add(dv(cloud_color), scale(mul(cloud_color, sun_color), 0.35 * lit));
            base = lerp(base, lit_cloud, alpha);
        }
    }
    return base;
}

// pt_occluded_segment (src/pathtrace.c:504-532) with the transmittance of
// water / beer_lambert surfaces carrying the absorption tangents
bool occluded_segment_d(const Params &pr, Ray r, double tmin, double tmax, DV3 *attenuation)
{
    const Scene *scene = pr.scene;
    *attenuation = dv(vec3(1.0, 1.0, 1.0));
    Ray cur = r;
    double remaining = tmax;
    for (int step = 0; step < 6; ++step) {
        Hit h;
        if (!scene_intersect(scene, cur, tmin, remaining, &h)) return false;
        const Material *m = scene_material(scene, h.material_index);
        if (m == NULL) return true;
        if (m->is_water || m->transparency > 0.8) {
            if (m->beer_lambert || m->is_water) {
                const DMat &p = pr.mats[h.material_index];
                DV3 seg = {dexp(-1.0 * p.absorption.x * h.t), dexp(-1.0 * p.absorption.y * h.t),
                           dexp(-1.0 * p.absorption.z * h.t)};
                *attenuation = mul(*attenuation, seg);
            }
            cur.origin = vec3_add(h.point, vec3_scale(cur.dir, 1e-3));
            remaining -= h.t;
            if (remaining <= 1e-3) return false;
            tmin = 1e-3;
            continue;
        }
        return true;
    }
    return true;
}

// pt_nee_sun (src/pathtrace.c:534-556)
DV3 nee_sun_d(const Params &pr, const Material *mm, const DMat &p, Vec3 P, Vec3 N, Vec3 V, const DV3 &throughput,
              unsigned seed_key, int bounce)
{
    const Scene *scene = pr.scene;
    DV3 zero = dv(vec3(0.0, 0.0, 0.0));
    Vec3 sun = scene->sky.sun_dir;
    double r1 = refpt::pt_rand01(seed_key, (unsigned)bounce, PT_CH_NEE_SUN_A);
    double r2 = refpt::pt_rand01(seed_key, (unsigned)bounce, PT_CH_NEE_SUN_B);
    Vec3 L = sky_sun_disk_dir(sun, scene->sky.sun_radius, r1, r2);
    if (!refpt::pt_is_finite(L) || vec3_dot(N, L) <= 0.0) return zero;
    Ray sr;
    sr.origin = vec3_add(P, vec3_scale(N, 1e-3));
    sr.dir = L;
    DV3 atten;
    if (occluded_segment_d(pr, sr, 1e-3, 1e30, &atten)) return zero;
    Vec3 cloud_trans = sky_cloud_transmittance(&scene->sky, sr.origin, sr.dir);
    atten = mul(atten, cloud_trans);
    if (atten.x.v < 1e-4 && atten.y.v < 1e-4 && atten.z.v < 1e-4) return zero;
    double rad = scene->sky.sun_radius * 3.14159265358979323846 / 180.0;
    double Omega = (scene->sky.sun_radius > 0.0) ? 2.0 * 3.14159265358979323846 * (1.0 - cos(rad)) : 1.0;
    DV3 sun_col = mul(pr.sun_color, atten);
    DV3 lit = shade_d(mm, p, N, L, V, sun_col);
    return mul(throughput, scale(lit, Omega));
}

// pt_nee_emissive (src/pathtrace.c:576-606); a light's radiance is its
// sphere's material emissive (scene.c collects it from there)
DV3 nee_emissive_d(const Params &pr, const Material *mm, const DMat &p, Vec3 P, Vec3 N, Vec3 V,
                   const DV3 &throughput, int self_prim, unsigned seed_key, int bounce)
{
    const Scene *scene = pr.scene;
    DV3 sum = dv(vec3(0.0, 0.0, 0.0));
    for (int li = 0; li < scene->emissive_light_count; ++li) {
        const EmissiveLight *lt = &scene->emissive_lights[li];
        if (lt->prim_index == self_prim) continue;
        Vec3 to_c = vec3_sub(lt->center, P);
        double dc2 = vec3_length_sq(to_c);
        double dcen = sqrt(dc2);
        if (dcen <= lt->radius) continue;
        double cos_mx = sqrt(1.0 - (lt->radius * lt->radius) / dc2);
        double Omega = 2.0 * 3.14159265358979323846 * (1.0 - cos_mx);
        if (!(Omega > 0.0)) continue;
        Vec3 w = vec3_scale(to_c, 1.0 / dcen);
        double u1 = refpt::pt_rand01(seed_key ^ (unsigned)li, (unsigned)bounce, PT_CH_NEE_EMIT_A);
        double u2 = refpt::pt_rand01(seed_key ^ (unsigned)li, (unsigned)bounce, PT_CH_NEE_EMIT_B);
        Vec3 wi = light_sphere_sample_dir(w, cos_mx, u1, u2);
        if (!refpt::pt_is_finite(wi) || vec3_dot(N, wi) <= 0.0) continue;
        Ray sr;
        sr.origin = vec3_add(P, vec3_scale(N, 1e-3));
        sr.dir = wi;
        Hit lh;
        if (!primitive_intersect(&scene->geo.prims[lt->prim_index], sr, 1e-3, 1e30, &lh)) continue;
        DV3 atten;
        if (occluded_segment_d(pr, sr, 1e-3, lh.t - 1e-3, &atten)) continue;
        int lmat = scene->geo.prims[lt->prim_index].material_index;
        DV3 le = (lmat >= 0 && lmat < scene->material_count) ? pr.mats[lmat].emissive : dv(lt->emissive);
        DV3 emit_col = mul(le, atten);
        DV3 lit = shade_d(mm, p, N, wi, V, emit_col);
        sum = add(sum, mul(throughput, scale(lit, Omega)));
    }
    return sum;
}

// The sampled lobe's weight with tangents (pt_sample_pbr / pt_sample_legacy,
// src/pathtrace.c:251-421); the direction, lobe and pdfs are the primal ones.
DV3 sample_weight_d(const Material *m, const DMat &p, Vec3 N, Vec3 d, Vec3 V, double u1, double u2, Vec3 wi,
                    Vec3 w, int specular)
{
    if (m->pbr) {
        D metallic = clamp01_d(p.metallic);
        D roughness = clamp01_d(p.roughness);
        D alpha = roughness_to_alpha_d(roughness);
        DV3 f0 = lerp(dv(vec3(0.04, 0.04, 0.04)), p.albedo, metallic);
        double p_spec = sampling_specular_probability(metallic.v, roughness.v, refpt::pt_luminance(val(f0)));
        double ndv = vec3_dot(N, V);
        // sampling_fresnel_schlick_rgb (src/sampling.c:141-156): f0 clamped
        auto fres = [](double cos_theta, const DV3 &f) {
            double c = clamp01(cos_theta);
            double mm = 1.0 - c;
            double m2 = mm * mm;
            double k = m2 * m2 * mm;
            D fx = clamp01_d(f.x), fy = clamp01_d(f.y), fz = clamp01_d(f.z);
            return DV3{fx + (1.0 - fx) * k, fy + (1.0 - fy) * k, fz + (1.0 - fz) * k};
        };
        if (specular) {
            Vec3 H = sampling_ggx_half_vector(N, alpha.v, u1, u2);
            double ndl = vec3_dot(N, wi);
            double ndh = vec3_dot(N, H);
            double vdh = vec3_dot(V, H);
            // pt_d_ggx / pt_g_smith_schlick (src/pathtrace.c:184-200)
            D a2 = alpha * alpha;
            D dd = ndh * ndh * (a2 - 1.0) + 1.0;
            D Dg = a2 / (SAMPLING_PI * dd * dd);
            D kk = (roughness + 1.0) * (roughness + 1.0) / 8.0;
            kk = clamp01_d(kk);
            D gl = ndl / (ndl * (1.0 - kk) + kk);
            D gv = ndv / (ndv * (1.0 - kk) + kk);
            D G = gl * gv;
            DV3 F = fres(vdh, f0);
            double pdf = sampling_ggx_pdf(ndh, vdh, alpha.v);
            D sc = Dg * G / (4.0 * ndv * pdf * p_spec);
            return scale(F, sc);
        }
        double denom = 1.0 - p_spec;
        DV3 F = fres(ndv, f0);
        DV3 kd = scale(sub(dv(vec3(1.0, 1.0, 1.0)), F), 1.0 - metallic);
        return scale(mul(kd, p.albedo), 1.0 / denom);
    }
    if (specular) return dv(w);  // mirror / dielectric: no differentiated parameter
    double r_mir = refpt::pt_clamp01(m->reflectivity);
    double r_die = refpt::pt_clamp01(m->transparency);
    double r_dif = 1.0 - r_mir - r_die;
    if (r_dif < 0.0) r_dif = 0.0;
    double p_dif = 1.0 - r_mir - r_die;
    double lobe = r_dif / p_dif;
    return scale(p.albedo, dc(lobe));
}

inline bool finite_d(const DV3 &a) { return isfinite(a.x.v) && isfinite(a.y.v) && isfinite(a.z.v); }

// water_attenuate (src/material.c:1238-1267) with the medium's dual absorption
DV3 water_attenuate_d(const Material *m, const DMat &p, Vec3 inner, double depth)
{
    double d = depth > 0.0 ? depth : 0.0;
    DV3 tr = {water_transmittance_d(p.absorption.x, d), water_transmittance_d(p.absorption.y, d),
              water_transmittance_d(p.absorption.z, d)};
    DV3 out = {inner.x * tr.x + m->deep_color.x * (1.0 - tr.x), inner.y * tr.y + m->deep_color.y * (1.0 - tr.y),
               inner.z * tr.z + m->deep_color.z * (1.0 - tr.z)};
    if (!(out.x.v >= 0.0)) out.x = dc(0.0);
    if (!(out.y.v >= 0.0)) out.y = dc(0.0);
    if (!(out.z.v >= 0.0)) out.z = dc(0.0);
    return out;
}

// pt_apply_medium (src/pathtrace.c:220-233)
void apply_medium_d(const Params &pr, const Material *m, double dist, DV3 *beta, DV3 *radiance)
{
    const DMat &p = pr.mats[m - pr.scene->materials];
    DV3 white = water_attenuate_d(m, p, vec3(1.0, 1.0, 1.0), dist);
    DV3 deep = water_attenuate_d(m, p, vec3(0.0, 0.0, 0.0), dist);
    DV3 transmittance = sub(white, deep);
    *radiance = add(*radiance, mul(*beta, deep));
    *beta = mul(*beta, transmittance);
}

// pathtrace_radiance (src/pathtrace.c:800-1028) with dual throughput/radiance
DV3 radiance_d(const Params &pr, Ray primary, int max_depth, unsigned seed_key, int *weight_mismatch)
{
    const Scene *scene = pr.scene;
    DV3 radiance = dv(vec3(0.0, 0.0, 0.0));
    if (max_depth < 0) max_depth = 0;
    Ray r;
    r.origin = primary.origin;
    r.dir = vec3_normalize(primary.dir);
    if (vec3_length_sq(r.dir) <= 0.0) return radiance;
    DV3 throughput = dv(vec3(1.0, 1.0, 1.0));
    const Material *medium = NULL;
    if (scene->water_material >= 0) {
        double w_h = scene_water_height(scene, primary.origin.x, primary.origin.z);
        if (primary.origin.y < w_h) medium = scene_material(scene, scene->water_material);
    }
    int last_bounce_specular = 1;
    for (int b = 0; b <= max_depth; b++) {
        Hit h;
        if (!scene_intersect(scene, r, PT_RAY_EPS, PT_RAY_MAX, &h)) {
            if (medium != NULL) {
                apply_medium_d(pr, medium, PT_MEDIUM_FALLBACK_DEPTH, &throughput, &radiance);
                medium = NULL;
            }
            radiance = add(radiance, mul(throughput, sky_sample_d(r.dir, &scene->sky, pr.sun_color)));
            break;
        }
        if (medium != NULL) apply_medium_d(pr, medium, h.t, &throughput, &radiance);
        const Material *m = scene_material(scene, h.material_index);
        if (m == NULL) {
            radiance = add(radiance, mul(throughput, sky_sample_d(r.dir, &scene->sky, pr.sun_color)));
            break;
        }
        const DMat &p = pr.mats[h.material_index];
        Vec3 P = h.point;
        Vec3 d = r.dir;
        Vec3 N = h.normal;
        if (m->is_water) {
            if (fabs(h.normal.y) > 0.999 && fabs(h.normal.x) < 1e-4 && fabs(h.normal.z) < 1e-4)
                N = water_normal(P.x, P.z, 0.0);
        }
        if (vec3_dot(N, d) > 0.0) N = vec3_neg(N);
        N = vec3_normalize(N);
        if (vec3_length_sq(N) <= 0.0) break;
        Vec3 V = vec3_neg(d);
        if (b == 0 || last_bounce_specular) radiance = add(radiance, mul(throughput, p.emissive));
        if (b == 0 && vec3_length_sq(m->atmosphere_glow) > 1e-6) {
            double cos_v = fmax(0.0, vec3_dot(N, V));
            double limb = pow(1.0 - cos_v, 3.5);
            double sun_dot = vec3_dot(N, scene->sky.sun_dir);
            double day_fac = 0.0;
            if (sun_dot > -0.15) {
                day_fac = (sun_dot + 0.15) / 0.35;
                if (day_fac > 1.0) day_fac = 1.0;
            }
            Vec3 glow_col = m->atmosphere_glow;
            if (sun_dot > -0.10 && sun_dot < 0.25) {
                double sunset_t = 1.0 - fabs(sun_dot - 0.05) / 0.20;
                if (sunset_t > 0.0) glow_col = vec3_lerp(glow_col, vec3(1.0, 0.45, 0.15), sunset_t * 0.6);
            }
            Vec3 atmo_term = vec3_scale(glow_col, limb * day_fac * 2.5);
            radiance = add(radiance, mul(throughput, atmo_term));
        }
        radiance = add(radiance, nee_emissive_d(pr, m, p, P, N, V, throughput, h.prim_index, seed_key, b));
        if (b == 0 || (b == 1 && medium != NULL && last_bounce_specular))
            radiance = add(radiance, nee_sun_d(pr, m, p, P, N, V, throughput, seed_key, b));
        unsigned kb = refpt::pt_hash3(seed_key ^ PT_KEY, (unsigned)b, 0u);
        double u1 = refpt::pt_rand01(kb, (unsigned)b, PT_CH_BSDF_A);
        double u2 = refpt::pt_rand01(kb, (unsigned)b, PT_CH_BSDF_B);
        double u_lobe = refpt::pt_rand01(kb, (unsigned)b, PT_CH_LOBE);
        double u_glass = refpt::pt_rand01(kb, (unsigned)b, PT_CH_GLASS);
        Vec3 wi, w;
        int ok;
        int refracted = 0;
        int sampled_specular = 0;
        if (m->pbr)
            ok = refpt::pt_sample_pbr(m, N, d, V, u1, u2, u_lobe, &wi, &w, &sampled_specular);
        else
            ok = refpt::pt_sample_legacy(m, N, d, V, h.front_face, u1, u2, u_lobe, u_glass, &wi, &w, &refracted,
                                         &sampled_specular);
        if (!ok) break;
        last_bounce_specular = sampled_specular;
        DV3 wd = sample_weight_d(m, p, N, d, V, u1, u2, wi, w, sampled_specular);
        if (wd.x.v != w.x || wd.y.v != w.y || wd.z.v != w.z) ++*weight_mismatch;
        throughput = mul(throughput, wd);
        if (!finite_d(throughput) || !(refpt::pt_max_component(val(throughput)) > 0.0)) break;
        if (refracted && (m->is_water || m->beer_lambert)) medium = h.front_face ? m : NULL;
        if (b >= PT_RR_START_BOUNCE) {
            double q = refpt::pt_clamp01(refpt::pt_max_component(val(throughput)));
            if (!(q > 0.0)) break;
            double u_rr = refpt::pt_rand01(kb, (unsigned)b, PT_CH_RR);
            if (u_rr >= q) break;
            throughput = scale(throughput, 1.0 / q);
        }
        Vec3 offset;
        if (refracted) offset = vec3_scale(wi, PT_RAY_EPS);
        else offset = vec3_scale(N, vec3_dot(wi, N) >= 0.0 ? PT_RAY_EPS : -PT_RAY_EPS);
        r.origin = vec3_add(P, offset);
        r.dir = wi;
    }
    if (!finite_d(radiance)) return dv(vec3(0.0, 0.0, 0.0));
    if (radiance.x.v < 0.0) radiance.x = dc(0.0);
    if (radiance.y.v < 0.0) radiance.y = dc(0.0);
    if (radiance.z.v < 0.0) radiance.z = dc(0.0);
    return radiance;
}

// primary ray of sample s at pixel (x, y) (pt_render_pixel, src/pathtrace.c:1057-1082)
Ray primary_ray(const MtRefHandle *H, int w, int h, int x, int y, int s)
{
    const Scene *scene = &H->scene;
    const Camera *cam = &H->cam;
    double jx = refpt::pt_rand01((unsigned)x, (unsigned)y, (unsigned)(s * 2 + 0));
    double jy = refpt::pt_rand01((unsigned)x, (unsigned)y, (unsigned)(s * 2 + 1));
    double lr1 = refpt::pt_rand01((unsigned)x, (unsigned)y, (unsigned)(s * 2 + 100));
    double lr2 = refpt::pt_rand01((unsigned)x, (unsigned)y, (unsigned)(s * 2 + 101));
    double uu = ((double)x + jx) / (double)w;
    double vv = 1.0 - ((double)y + jy) / (double)h;
    Ray ray = camera_ray_dof(cam, uu, vv, lr1, lr2);
    if (cam->dome_radius > 1e-4 && scene->water_material >= 0) {
        Vec3 p_dome = vec3_add(ray.origin, vec3_scale(ray.dir, cam->dome_radius));
        double wh = scene_water_height(scene, p_dome.x, p_dome.z);
        if (p_dome.y < wh) ray.origin = vec3_sub(p_dome, vec3(0.0, 1e-3, 0.0));
    }
    return ray;
}

// What the restatement does not cover: textures, bump maps, fog, volumetric
// clouds and sky extras (the GPU renderer rejects the same content).
bool supported(const Scene *s)
{
    if (s->fog.density > 0.0 || s->fog.shadow_steps > 0) return false;
    if (s->sky.cloud_thickness > 1e-4 || s->sky.star_intensity > 0.0 || s->sky.nebula_intensity > 0.0 ||
        s->sky.galaxy_intensity > 0.0)
        return false;
    for (int i = 0; i < s->material_count; ++i)
        if (s->materials[i].texture_kind != 0 || s->materials[i].bump_strength > 1e-6) return false;
    return true;
}

}  // namespace

extern "C" {

/* Parameter count of the adjoint layout: 8 per material, then the sun rgb. */
int mtdual_param_count(void *hp)
{
    return 11 * ((MtRefHandle *)hp)->scene.material_count + 3;
}

/*
 * grad[j] = sum over pixels and samples [s0, s1) of adj(pixel) . scale .
 * dL/dtheta(idx[j]); adj is h x w x 3 floats. value_sum (optional, h x w x 3)
 * receives the per-pixel sum of the sample values. Returns the number of
 * samples whose value differs from the reference's pathtrace_radiance or
 * whose restated BSDF weight differs from the reference's (0 expected), or
 * -1 for content the restatement does not cover.
 */
int mtdual_pathtrace_grad(void *hp, int w, int h, int s0, int s1, int depth, const float *adj, double adj_scale,
                          const int *idx, int n_idx, double *grad, double *value_sum)
{
    MtRefHandle *H = (MtRefHandle *)hp;
    const Scene *scene = &H->scene;
    if (!supported(scene)) return -1;
    const int M = scene->material_count;
    DMat *mats = (DMat *)calloc((size_t)(M > 0 ? M : 1), sizeof(DMat));
    if (!mats) return -1;
    int mismatches = 0;
    for (int j = 0; j < (n_idx > 0 ? n_idx : 1); ++j) {
        const int k = n_idx > 0 ? idx[j] : -1;
        for (int m = 0; m < M; ++m) {
            const Material *src = &scene->materials[m];
            const int b = 8 * m;
            mats[m].albedo = {{src->albedo.x, k == b ? 1.0 : 0.0}, {src->albedo.y, k == b + 1 ? 1.0 : 0.0},
                              {src->albedo.z, k == b + 2 ? 1.0 : 0.0}};
            mats[m].roughness = {src->roughness, k == b + 3 ? 1.0 : 0.0};
            mats[m].metallic = {src->metallic, k == b + 4 ? 1.0 : 0.0};
            mats[m].emissive = {{src->emissive.x, k == b + 5 ? 1.0 : 0.0}, {src->emissive.y, k == b + 6 ? 1.0 : 0.0},
                                {src->emissive.z, k == b + 7 ? 1.0 : 0.0}};
            const int ab = 8 * M + 3 + 3 * m;  // absorption block after the sun
            mats[m].absorption = {{src->absorption.x, k == ab ? 1.0 : 0.0}, {src->absorption.y, k == ab + 1 ? 1.0 : 0.0},
                                  {src->absorption.z, k == ab + 2 ? 1.0 : 0.0}};
        }
        const int sb = 8 * M;
        Params pr{scene, mats,
                  DV3{{scene->sky.sun_color.x, k == sb ? 1.0 : 0.0}, {scene->sky.sun_color.y, k == sb + 1 ? 1.0 : 0.0},
                      {scene->sky.sun_color.z, k == sb + 2 ? 1.0 : 0.0}}};
        double g = 0.0;
        for (int y = 0; y < h; ++y)
            for (int x = 0; x < w; ++x) {
                const float *a = adj + 3 * ((size_t)y * w + x);
                for (int s = s0; s < s1; ++s) {
                    Ray ray = primary_ray(H, w, h, x, y, s);
                    unsigned seed = refpt::pt_hash3((unsigned)x, (unsigned)y, (unsigned)s);
                    int wm = 0;
                    DV3 L = radiance_d(pr, ray, depth, seed, &wm);
                    g += (double)a[0] * adj_scale * L.x.d + (double)a[1] * adj_scale * L.y.d +
                         (double)a[2] * adj_scale * L.z.d;
                    if (j == 0) {
                        Vec3 ref = refpt::refpt_pathtrace_radiance(scene, ray, depth, seed);
                        if (wm || ref.x != L.x.v || ref.y != L.y.v || ref.z != L.z.v) ++mismatches;
                        if (value_sum) {
                            double *o = value_sum + 3 * ((size_t)y * w + x);
                            o[0] += L.x.v;
                            o[1] += L.y.v;
                            o[2] += L.z.v;
                        }
                    }
                }
            }
        if (n_idx > 0) grad[j] = g;
    }
    free(mats);
    return mismatches;
}

}  // extern "C"
