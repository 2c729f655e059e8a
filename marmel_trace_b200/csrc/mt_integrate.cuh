// mt_integrate.cuh - the path tracer and the Whitted renderer on the device.
#pragma once

#include "mt_shade.cuh"

namespace mt {

// Channel constants of the path tracer's random stream (src/pathtrace.c:125-134).
enum : uint32_t {
    PT_KEY = 0x5054u,
    PT_CH_BSDF_A = 0xB501u,
    PT_CH_BSDF_B = 0xB502u,
    PT_CH_LOBE = 0x1001u,
    PT_CH_GLASS = 0x1002u,
    PT_CH_RR = 0x5201u,
    PT_CH_NEE_SUN_A = 0xA101u,
    PT_CH_NEE_SUN_B = 0xA102u,
    PT_CH_NEE_EMIT_A = 0xA201u,
    PT_CH_NEE_EMIT_B = 0xA202u,
};

template <typename R> struct Ray3 {
    V3<R> o, d;
};

// ------------------------------------------------------------------
// Camera (camera_ray / camera_ray_dof, src/camera.c:68-134)
// ------------------------------------------------------------------
template <typename R> MT_D Ray3<R> camera_ray(const DevCamera<R> &c, R u, R v)
{
    Ray3<R> r;
    r.o = mat3(c.position);
    V3<R> point = add(mat3(c.lower_left), add(scale(mat3(c.horizontal), u), scale(mat3(c.vertical), v)));
    r.d = normalize(sub(point, r.o));
    return r;
}

template <typename R> MT_D Ray3<R> camera_ray_dof(const DevCamera<R> &c, R u, R v, R r1, R r2)
{
    if (c.aperture <= R(1e-12)) return camera_ray(c, u, v);
    Ray3<R> pin = camera_ray(c, u, v);
    R fd = c.focus_distance;
    if (fd <= R(0)) fd = R(1);
    V3<R> focal = add(mat3(c.position), scale(pin.d, fd));
    V3<R> right = normalize(mat3(c.horizontal));
    V3<R> up = normalize(mat3(c.vertical));
    R rad = c.aperture * msqrt(r1);
    R theta = R(2) * Const<R>::pi * r2;
    R sq = c.anamorphic_squeeze;
    R st, ct;
    msincos(theta, &st, &ct);
    V3<R> offset;
    if (sq <= R(0) || mfabs(sq - R(1)) < R(1e-12))
        offset = add(scale(right, rad * ct), scale(up, rad * st));
    else
        offset = add(scale(right, (rad / sq) * ct), scale(up, rad * st));
    Ray3<R> r;
    r.o = add(mat3(c.position), offset);
    r.d = normalize(sub(focal, r.o));
    return r;
}

// Primary ray of path-tracer sample s at (x, y): jitter channels 2s / 2s+1,
// lens channels 2s+100 / 2s+101, dome-port adjustment (src/pathtrace.c:1057-1082).
template <typename R>
MT_D Ray3<R> pt_primary(const DevScene<R> &S, const DevCamera<R> &cam, int w, int h, int x, int y, int s)
{
    R jx = rand01<R>((uint32_t)x, (uint32_t)y, (uint32_t)(s * 2 + 0));
    R jy = rand01<R>((uint32_t)x, (uint32_t)y, (uint32_t)(s * 2 + 1));
    R lr1 = rand01<R>((uint32_t)x, (uint32_t)y, (uint32_t)(s * 2 + 100));
    R lr2 = rand01<R>((uint32_t)x, (uint32_t)y, (uint32_t)(s * 2 + 101));
    R uu = (R(x) + jx) / R(w);
    R vv = R(1) - (R(y) + jy) / R(h);
    Ray3<R> ray = camera_ray_dof(cam, uu, vv, lr1, lr2);
    if (cam.dome_radius > R(1e-4) && S.water_material >= 0) {
        V3<R> p_dome = add(ray.o, scale(ray.d, cam.dome_radius));
        R wh = water_height(S, p_dome.x, p_dome.z);
        if (p_dome.y < wh) ray.o = sub(p_dome, v3(R(0), R(1e-3), R(0)));
    }
    return ray;
}

// Whitted sample offset: stratified g x g when spp is a perfect square,
// otherwise uniform (sample_offset, src/render.c:874-889), and lens channels
// 2s+2 / 2s+3 (src/render.c:945-948).
template <typename R>
MT_D Ray3<R> wh_primary(const DevCamera<R> &cam, int w, int h, int spp, int x, int y, int s)
{
    R du, dv;
    int g = (int)(sqrt((double)spp) + 0.5);
    if (g > 0 && g * g == spp) {
        int i = s % g;
        int j = s / g;
        R jx = rand01<R>((uint32_t)x, (uint32_t)y, (uint32_t)(s * 2 + 0));
        R jy = rand01<R>((uint32_t)x, (uint32_t)y, (uint32_t)(s * 2 + 1));
        du = (R(i) + jx) / R(g);
        dv = (R(j) + jy) / R(g);
    } else {
        du = rand01<R>((uint32_t)x, (uint32_t)y, (uint32_t)(s * 2 + 0));
        dv = rand01<R>((uint32_t)x, (uint32_t)y, (uint32_t)(s * 2 + 1));
    }
    R uu = (R(x) + du) / R(w);
    R vv = R(1) - (R(y) + dv) / R(h);
    R lr1 = rand01<R>((uint32_t)x, (uint32_t)y, (uint32_t)(s * 2 + 2));
    R lr2 = rand01<R>((uint32_t)x, (uint32_t)y, (uint32_t)(s * 2 + 3));
    return camera_ray_dof(cam, uu, vv, lr1, lr2);
}

// ------------------------------------------------------------------
// Path tracer
// ------------------------------------------------------------------
template <typename R> MT_D R pt_max_component(V3<R> v)
{
    R m = v.x;
    if (v.y > m) m = v.y;
    if (v.z > m) m = v.z;
    if (!(m > R(0))) m = R(0);
    return m;
}

template <typename R> MT_D R pt_luminance(V3<R> c)
{
    R y = R(0.2126) * c.x + R(0.7152) * c.y + R(0.0722) * c.z;
    return (y > R(0)) ? y : R(0);
}

// pt_apply_medium: water_attenuate twice (white / black inner) and subtract
// (src/pathtrace.c:220-233)
template <typename R>
MT_D void pt_apply_medium(const DevMaterial<R> &m, R dist, V3<R> *beta, V3<R> *radiance)
{
    V3<R> white = water_attenuate(m, v3(R(1), R(1), R(1)), dist);
    V3<R> deep = water_attenuate(m, v3(R(0), R(0), R(0)), dist);
    V3<R> transmittance = sub(white, deep);
    *radiance = add(*radiance, mul(*beta, deep));
    *beta = mul(*beta, transmittance);
}

// pt_occluded_segment: up to 6 chained nearest hits; transparent hits
// (water or transparency > 0.8) pass with Beer-Lambert (src/pathtrace.c:504-532)
template <typename R>
MT_D bool pt_occluded_segment(const DevScene<R> &S, V3<R> o, V3<R> d, R tmin, R tmax, V3<R> *attenuation)
{
    *attenuation = v3(R(1), R(1), R(1));
    V3<R> cur_o = o;
    R remaining = tmax;
    if (S.counters) atomicAdd(&S.counters->shadow_rays, 1ull);
    if (!S.has_passthrough) {
        // No material lets the segment through: the walk below stops at its
        // first hit, so "occluded" is exactly "any hit in [tmin, tmax]".
        return scene_any(S, ray_pre(o, unit_dir(d)), tmin, tmax);
    }
    for (int step = 0; step < 6; ++step) {
        LinkHit<R> h;
        if (!scene_link(S, cur_o, d, tmin, remaining, &h)) return false;
        if (h.material < 0 || h.material >= S.material_count) return true;
        const DevMaterial<R> &m = S.materials[h.material];
        if (m.is_water || m.transparency > R(0.8)) {
            if (m.beer_lambert || m.is_water) {
                V3<R> seg = v3(mexp(-m.absorption[0] * h.t), mexp(-m.absorption[1] * h.t),
                               mexp(-m.absorption[2] * h.t));
                *attenuation = mul(*attenuation, seg);
            }
            cur_o = add(h.point, scale(d, R(1e-3)));
            remaining -= h.t;
            if (remaining <= R(1e-3)) return false;
            tmin = R(1e-3);
            continue;
        }
        return true;
    }
    return true;
}

// pt_fog_segment (src/pathtrace.c:614-730): with fog.shadow_steps > 0 a
// jittered march with a shadow segment toward the sun per step (god rays),
// then the analytic remainder; otherwise the analytic fog_segment.
template <typename R>
MT_NOINLINE void pt_fog_segment(const DevScene<R> &S, V3<R> o, V3<R> d, R dist, uint32_t seed_key, int bounce,
                                R *transmittance, V3<R> *inscatter)
{
    const DevFog<R> &fog = S.fog;
    if (fog.shadow_steps <= 0) {
        fog_segment(fog, S.sky, o, d, dist, transmittance, inscatter);
        return;
    }
    int steps = fog.shadow_steps;
    if (steps < 4) steps = 4;
    if (steps > 128) steps = 128;
    const bool is_sky = dist >= R(1e20);
    const R lambda = fog.height_falloff;
    R max_t;
    if (is_sky) {
        R top_y = (lambda > R(1e-4)) ? (fog.height + R(3) / lambda) : R(25);
        if (o.y >= top_y && d.y >= R(0)) {
            *transmittance = R(1);
            *inscatter = v3(R(0), R(0), R(0));
            return;
        }
        R dy = d.y;
        if (dy > R(0.02)) {
            max_t = (top_y - o.y) / dy;
            if (max_t > R(40)) max_t = R(40);
        } else {
            max_t = R(40);
        }
    } else {
        max_t = (dist > R(60)) ? R(60) : dist;
    }
    const R dt = max_t / R(steps);
    const V3<R> sun_dir = mat3(S.sky.sun_dir);
    R phase_hg = fog_phase_hg(fog, d, sun_dir);
    if (phase_hg > R(6)) phase_hg = R(6);
    const R phase = R(0.70) * phase_hg + R(0.30);
    const V3<R> sun_glow_unit = scale(mat3(S.sky.sun_color), phase * fog.inscatter_strength);
    R T_acc = R(1);
    V3<R> acc = v3(R(0), R(0), R(0));
    const R jitter = rand01<R>(seed_key, (uint32_t)bounce, 0xFE01u);
    for (int i = 0; i < steps; ++i) {
        R t = (R(i) + jitter) * dt;
        V3<R> pos = add(o, scale(d, t));
        R rho = fog.density;
        if (lambda > R(1e-6)) {
            R h_diff = pos.y - fog.height;
            rho *= mexp(-lambda * h_diff);
        }
        if (fog.noise_amount > R(1e-4) && fog.noise_scale > R(1e-4)) rho *= fog_noise_mod(fog, pos);
        if (rho < R(0)) rho = R(0);
        R step_tau = rho * dt;
        R step_T = mexp(-step_tau);
        V3<R> atten;
        bool in_shadow = pt_occluded_segment(S, pos, sun_dir, R(0.05), R(100), &atten);
        if (!in_shadow) atten = scale(atten, cloud_transmittance(S.sky, pos, sun_dir));
        V3<R> col = mat3(fog.color);
        if (!in_shadow) col = add(col, mul(sun_glow_unit, atten));
        V3<R> step_inscatter = scale(col, R(1) - step_T);
        acc = add(acc, scale(step_inscatter, T_acc));
        T_acc *= step_T;
        if (T_acc < R(1e-4)) break;
    }
    if (dist > max_t) {
        R rem_dist = is_sky ? R(1e30) : (dist - max_t);
        V3<R> rem_o = add(o, scale(d, max_t));
        R rem_T;
        V3<R> rem_in;
        fog_segment(fog, S.sky, rem_o, d, rem_dist, &rem_T, &rem_in);
        acc = add(acc, scale(rem_in, T_acc));
        T_acc *= rem_T;
    }
    *transmittance = T_acc;
    *inscatter = acc;
}

// The march of pt_water_segment (src/pathtrace.c:748-795): underwater god
// rays from sun shadow segments.
template <typename R>
MT_NOINLINE void pt_water_march(const DevScene<R> &S, int medium, V3<R> o, V3<R> d, R dist, uint32_t seed_key,
                                int bounce, V3<R> *beta, V3<R> *radiance)
{
    const DevMaterial<R> &m = S.materials[medium];
    int steps = S.fog.shadow_steps;
    if (steps < 4) steps = 4;
    if (steps > 16) steps = 16;
    const R dt = dist / R(steps);
    const V3<R> sun_dir = mat3(S.sky.sun_dir);
    R cos_theta = dot(d, sun_dir);
    const R g = R(0.72);
    R denom = R(1) + g * g - R(2) * g * cos_theta;
    if (denom < R(1e-4)) denom = R(1e-4);
    R phase = (R(1) - g * g) / (denom * msqrt(denom));
    if (phase > R(4.5)) phase = R(4.5);
    const R jitter = rand01<R>(seed_key, (uint32_t)bounce, 0xAC31u);
    const V3<R> step_T = v3(mexp(-m.absorption[0] * dt), mexp(-m.absorption[1] * dt), mexp(-m.absorption[2] * dt));
    for (int i = 0; i < steps; ++i) {
        R t = (R(i) + jitter) * dt;
        V3<R> pos = add(o, scale(d, t));
        V3<R> atten;
        bool in_shadow = pt_occluded_segment(S, pos, sun_dir, R(0.02), R(100), &atten);
        if (!in_shadow) atten = scale(atten, cloud_transmittance(S.sky, pos, sun_dir));
        V3<R> ambient = scale(mat3(m.deep_color), R(0.40));
        V3<R> sun_scat = v3(R(0), R(0), R(0));
        if (!in_shadow) sun_scat = scale(mul(mat3(S.sky.sun_color), atten), phase * R(0.18));
        V3<R> step_col = add(ambient, sun_scat);
        V3<R> step_in = v3(step_col.x * (R(1) - step_T.x), step_col.y * (R(1) - step_T.y), step_col.z * (R(1) - step_T.z));
        *radiance = add(*radiance, mul(*beta, step_in));
        *beta = mul(*beta, step_T);
    }
}

// pt_water_segment (src/pathtrace.c:737-795): a water medium with
// fog.shadow_steps > 0 is marched; otherwise (and for other media) it is
// pt_apply_medium.
template <typename R>
MT_D void pt_water_segment(const DevScene<R> &S, int medium, V3<R> o, V3<R> d, R dist, uint32_t seed_key, int bounce,
                           V3<R> *beta, V3<R> *radiance)
{
    const DevMaterial<R> &m = S.materials[medium];
    if (!m.is_water || S.fog.shadow_steps <= 0 || dist <= R(1e-4)) {
        pt_apply_medium(m, dist, beta, radiance);
        return;
    }
    pt_water_march(S, medium, o, d, dist, seed_key, bounce, beta, radiance);
}

// Distances a shadow segment travels through absorbing (Beer-Lambert)
// materials, for the adjoint: up to two materials, `mat` -1 when unused.
template <typename R> struct AbsorbPath {
    int mat[2];
    R dist[2];
};

// Shadow segments of scenes whose materials can pass shadow rays, with an
// occluder cache entry of opaque blocking leaves (four leaf codes of the main
// tree, newest first). The chain of pt_occluded_segment starts with the
// nearest hit over every primitive, and when that hit is opaque the answer is
// "occluded". A cached opaque blocker hit at t_P makes that certain as soon
// as no pass-through primitive is hit in [tmin, t_P]: the nearest hit is then
// at t <= t_P and opaque. The pass tree (DevScene::pass_root) answers that
// over the pass-through primitives alone; the interval is widened by 1e-5 of
// itself, more than the FP32 rounding of the range tests, so a pass-through
// hit at or next to t_P leaves the segment to the chain.
template <typename R>
MT_D bool pass_cache_occluded(const DevScene<R> &S, const int *entry, const RayPre<R> &rp, R tmin, R tmax)
{
    const R tp = occ_opaque_nearest(S, entry, rp, tmin, tmax);
    return tp >= R(0) && !pass_hit(S, rp, tmin * R(1.0 - 1e-5), tp * R(1.0 + 1e-5));
}

// pt_occluded_segment with the same result and attenuation, also reporting
// the absorbing materials passed and the distance factor of each one: the
// attenuation is prod exp(-absorption * t) over the passed hits, so
// d attenuation / d absorption_c(m) = -attenuation_c * (sum of t over m's hits).
// A third distinct absorbing material on one segment sets ERR_ABSORB.
template <typename R>
MT_D bool pt_occluded_segment_abs(const DevScene<R> &S, V3<R> o, V3<R> d, R tmin, R tmax, V3<R> *attenuation,
                                  AbsorbPath<R> *ab)
{
    ab->mat[0] = ab->mat[1] = -1;
    ab->dist[0] = ab->dist[1] = R(0);
    *attenuation = v3(R(1), R(1), R(1));
    V3<R> cur_o = o;
    R remaining = tmax;
    if (S.counters) atomicAdd(&S.counters->shadow_rays, 1ull);
    if (!S.has_passthrough) return scene_any(S, ray_pre(o, unit_dir(d)), tmin, tmax);
    for (int step = 0; step < 6; ++step) {
        LinkHit<R> h;
        if (!scene_link(S, cur_o, d, tmin, remaining, &h)) return false;
        if (h.material < 0 || h.material >= S.material_count) return true;
        const DevMaterial<R> &m = S.materials[h.material];
        if (m.is_water || m.transparency > R(0.8)) {
            if (m.beer_lambert || m.is_water) {
                V3<R> seg = v3(mexp(-m.absorption[0] * h.t), mexp(-m.absorption[1] * h.t),
                               mexp(-m.absorption[2] * h.t));
                *attenuation = mul(*attenuation, seg);
                int k = ab->mat[0] == h.material ? 0 : ab->mat[1] == h.material ? 1 : ab->mat[0] < 0 ? 0
                                                                                     : ab->mat[1] < 0 ? 1 : -1;
                if (k < 0) {
                    atomicOr(S.err, ERR_ABSORB);
                } else {
                    ab->mat[k] = h.material;
                    ab->dist[k] += h.t;
                }
            }
            cur_o = add(h.point, scale(d, R(1e-3)));
            remaining -= h.t;
            if (remaining <= R(1e-3)) return false;
            tmin = R(1e-3);
            continue;
        }
        return true;
    }
    return true;
}

// pt_nee_sun (src/pathtrace.c:534-556)
// EXTRAS = false: the scene has no volumetric clouds (DevScene::has_extras).
template <typename R, bool EXTRAS = true>
MT_D V3<R> pt_nee_sun(const DevScene<R> &S, const DevMaterial<R> &mm, V3<R> P, V3<R> N, V3<R> V, V3<R> throughput,
                      uint32_t seed_key, int bounce)
{
    V3<R> sun = mat3(S.sky.sun_dir);
    R r1 = rand01<R>(seed_key, (uint32_t)bounce, PT_CH_NEE_SUN_A);
    R r2 = rand01<R>(seed_key, (uint32_t)bounce, PT_CH_NEE_SUN_B);
    V3<R> L = sun_disk_dir(sun, S.sky.sun_radius, r1, r2);
    V3<R> zero = v3(R(0), R(0), R(0));
    if (!finite3(L) || dot(N, L) <= R(0)) return zero;
    V3<R> so = add(P, scale(N, R(1e-3)));
    V3<R> atten;
    if (pt_occluded_segment(S, so, L, R(1e-3), R(1e30), &atten)) return zero;
    if constexpr (EXTRAS) atten = scale(atten, cloud_transmittance(S.sky, so, L));
    if (atten.x < R(1e-4) && atten.y < R(1e-4) && atten.z < R(1e-4)) return zero;
    R rad = S.sky.sun_radius * R(3.14159265358979323846) / R(180);
    R Omega = (S.sky.sun_radius > R(0)) ? R(2) * R(3.14159265358979323846) * (R(1) - mcos(rad)) : R(1);
    V3<R> sun_col = mul(mat3(S.sky.sun_color), atten);
    V3<R> lit = shade(mm, N, L, V, sun_col);
    return mul(throughput, scale(lit, Omega));
}

// pt_nee_emissive (src/pathtrace.c:576-606)
template <typename R>
MT_D V3<R> pt_nee_emissive(const DevScene<R> &S, const DevMaterial<R> &mm, V3<R> P, V3<R> N, V3<R> V,
                           V3<R> throughput, int self_prim, uint32_t seed_key, int bounce)
{
    V3<R> sum = v3(R(0), R(0), R(0));
    for (int li = 0; li < S.light_count; ++li) {
        const DevLight<R> &lt = S.lights[li];
        if (lt.prim == self_prim) continue;
        V3<R> to_c = sub(mat3(lt.center), P);
        R dc2 = length_sq(to_c);
        R dc = msqrt(dc2);
        if (dc <= lt.radius) continue;
        R cos_mx = msqrt(R(1) - (lt.radius * lt.radius) / dc2);
        const R omc = cone_one_minus_cos((lt.radius * lt.radius) / dc2, cos_mx);
        R Omega = R(2) * R(3.14159265358979323846) * omc;
        if (!(Omega > R(0))) continue;
        V3<R> w = scale(to_c, R(1) / dc);
        R u1 = rand01<R>(seed_key ^ (uint32_t)li, (uint32_t)bounce, PT_CH_NEE_EMIT_A);
        R u2 = rand01<R>(seed_key ^ (uint32_t)li, (uint32_t)bounce, PT_CH_NEE_EMIT_B);
        V3<R> wi = light_sphere_sample_dir(w, cos_mx, omc, u1, u2);
        if (!finite3(wi) || dot(N, wi) <= R(0)) continue;
        V3<R> so = add(P, scale(N, R(1e-3)));
        R lt_t;
        if (!light_sphere_t(S, lt.prim, so, wi, R(1e-3), R(1e30), &lt_t)) continue;
        V3<R> atten;
        if (pt_occluded_segment(S, so, wi, R(1e-3), lt_t - R(1e-3), &atten)) continue;
        V3<R> emit_col = mul(mat3(lt.emissive), atten);
        V3<R> lit = shade(mm, N, wi, V, emit_col);
        sum = add(sum, mul(throughput, scale(lit, Omega)));
    }
    return sum;
}

// pt_sample_pbr (src/pathtrace.c:251-322)
template <typename R>
MT_D bool pt_sample_pbr(const DevMaterial<R> &m, V3<R> N, V3<R> d, V3<R> V, R u1, R u2, R u_lobe, V3<R> *wi_out,
                        V3<R> *w_out, int *out_specular)
{
    *out_specular = 0;
    R metallic = pt_clamp01(m.metallic);
    R roughness = pt_clamp01(m.roughness);
    R alpha = roughness_to_alpha(roughness);
    V3<R> albedo = mat3(m.albedo);
    V3<R> f0 = lerp(v3(R(0.04), R(0.04), R(0.04)), albedo, metallic);
    R f0_scalar = pt_luminance(f0);
    R p_spec = specular_probability(metallic, roughness, f0_scalar);
    R ndv = dot(N, V);
    if (!(ndv > R(0))) return false;
    if (u_lobe < p_spec) {
        V3<R> H = ggx_half_vector(N, alpha, u1, u2);
        V3<R> wi = reflect(d, H);
        R ndl = dot(N, wi);
        R ndh = dot(N, H);
        R vdh = dot(V, H);
        if (!(ndl > R(0)) || !(ndh > R(0)) || !(vdh > R(0))) return false;
        const R sin2 = sin2_between(N, H);
        R D = d_ggx_cs(ndh, sin2, alpha);
        R G = g_smith_schlick(ndl, ndv, roughness);
        V3<R> F = sampling_fresnel_schlick_rgb(vdh, f0);
        R pdf = ggx_pdf(ndh, sin2, vdh, alpha);
        if (!(pdf > R(0)) || !(p_spec > R(0))) return false;
        R sc = D * G / (R(4) * ndv * pdf * p_spec);
        *wi_out = wi;
        *w_out = scale(F, sc);
        *out_specular = 1;
        return true;
    }
    R denom = R(1) - p_spec;
    if (!(denom > R(0))) return false;
    V3<R> wi = cosine_hemisphere(N, u1, u2);
    R ndl = dot(N, wi);
    if (!(ndl > R(0))) return false;
    V3<R> F = sampling_fresnel_schlick_rgb(ndv, f0);
    V3<R> kd = scale(sub(v3(R(1), R(1), R(1)), F), R(1) - metallic);
    *wi_out = wi;
    *w_out = scale(mul(kd, albedo), R(1) / denom);
    return true;
}

// pt_sample_legacy (src/pathtrace.c:336-453)
template <typename R>
MT_D bool pt_sample_legacy(const DevMaterial<R> &m, V3<R> N, V3<R> d, V3<R> V, int front_face, R u1, R u2,
                           R u_lobe, R u_glass, V3<R> *wi_out, V3<R> *w_out, int *out_refract, int *out_specular)
{
    *out_refract = 0;
    *out_specular = 0;
    R r_mir = pt_clamp01(m.reflectivity);
    R r_die = pt_clamp01(m.transparency);
    R r_dif = R(1) - r_mir - r_die;
    if (r_dif < R(0)) r_dif = R(0);
    R p_mir = r_mir;
    R p_die = r_die;
    R p_dif = R(1) - p_mir - p_die;
    R norm = R(1);
    if (p_dif < R(0)) {
        R s = p_mir + p_die;
        if (s > R(0)) {
            p_mir /= s;
            p_die /= s;
            if (s > R(1)) norm = s;
        }
        p_dif = R(0);
    }
    if (u_lobe < p_mir) {
        if (!(p_mir > R(0))) return false;
        R w = r_mir / (p_mir * norm);
        *wi_out = reflect(d, N);
        *w_out = v3(w, w, w);
        *out_specular = 1;
        return true;
    }
    if (u_lobe < p_mir + p_die) {
        if (!(p_die > R(0))) return false;
        *out_specular = 1;
        R ior = (m.ior > R(0)) ? m.ior : R(1);
        R eta = front_face ? (R(1) / ior) : ior;
        R cos_i = pt_clamp01(dot(N, V));
        R F = fresnel_dielectric(cos_i, eta);
        R lobe = r_die / (p_die * norm);
        if (F >= R(1)) {
            *wi_out = reflect(d, N);
            *w_out = v3(lobe, lobe, lobe);
            return true;
        }
        R p_r = pt_clamp(F, R(0.05), R(0.95));
        if (u_glass < p_r) {
            R w = lobe * (F / p_r);
            *wi_out = reflect(d, N);
            *w_out = v3(w, w, w);
            return true;
        }
        V3<R> wi;
        if (!sampling_refract(d, N, eta, &wi)) {
            R w = lobe * (F / p_r);
            *wi_out = reflect(d, N);
            *w_out = v3(w, w, w);
            return true;
        }
        R w = lobe * ((R(1) - F) / (R(1) - p_r)) * eta * eta;
        *wi_out = wi;
        *w_out = v3(w, w, w);
        *out_refract = 1;
        return true;
    }
    if (!(p_dif > R(0))) return false;
    V3<R> wi = cosine_hemisphere(N, u1, u2);
    R ndl = dot(N, wi);
    if (!(ndl > R(0))) return false;
    R lobe = r_dif / p_dif;
    *wi_out = wi;
    *w_out = scale(mat3(m.albedo), lobe);
    return true;
}

// Rayleigh limb glow of the primary hit (src/pathtrace.c:924-945, src/render.c:820-838)
template <typename R> MT_D V3<R> atmosphere_term(const DevMaterial<R> &mm, V3<R> N, V3<R> V, V3<R> sun_dir)
{
    R cos_v = mfmax(R(0), dot(N, V));
    R limb = mpow(R(1) - cos_v, R(3.5));
    R sun_dot = dot(N, sun_dir);
    R day_fac = R(0);
    if (sun_dot > R(-0.15)) {
        day_fac = (sun_dot + R(0.15)) / R(0.35);
        if (day_fac > R(1)) day_fac = R(1);
    }
    V3<R> glow_col = mat3(mm.atmosphere_glow);
    if (sun_dot > R(-0.10) && sun_dot < R(0.25)) {
        R sunset_t = R(1) - mfabs(sun_dot - R(0.05)) / R(0.20);
        if (sunset_t > R(0)) {
            V3<R> sunset_col = v3(R(1.0), R(0.45), R(0.15));
            glow_col = lerp(glow_col, sunset_col, sunset_t * R(0.6));
        }
    }
    return scale(glow_col, limb * day_fac * R(2.5));
}

// pathtrace_radiance (src/pathtrace.c:800-1028) without fog (rejected on upload)
// EXTRAS = false: the scene has no fog, marched media, clouds or textures
// (DevScene::has_extras); those paths are then compiled out.
template <typename R, bool EXTRAS = true>
MT_D V3<R> pathtrace_radiance(const DevScene<R> &S, Ray3<R> primary, int max_depth, uint32_t seed_key)
{
    V3<R> radiance = v3(R(0), R(0), R(0));
    if (max_depth < 0) max_depth = 0;
    Ray3<R> r;
    r.o = primary.o;
    r.d = normalize(primary.d);
    if (length_sq(r.d) <= R(0)) return radiance;
    V3<R> throughput = v3(R(1), R(1), R(1));
    int medium = -1;
    if (S.water_material >= 0) {
        R w_h = water_height(S, primary.o.x, primary.o.z);
        if (primary.o.y < w_h && S.water_material < S.material_count) medium = S.water_material;
    }
    int last_bounce_specular = 1;
    for (int b = 0; b <= max_depth; b++) {
        SurfaceHit<R> h;
        if (!scene_intersect(S, r.o, r.d, R(1e-4), R(1e30), &h)) {
            if (medium >= 0) {
                if constexpr (EXTRAS) pt_water_segment(S, medium, r.o, r.d, R(5.0), seed_key, b, &throughput, &radiance);
                else pt_apply_medium(S.materials[medium], R(5.0), &throughput, &radiance);
                medium = -1;
            }
            V3<R> sky_col = sky_sample<R, EXTRAS>(r.d, S.sky);
            if (EXTRAS && S.fog.density > R(0)) {
                R T;
                V3<R> ins;
                if (b == 0) pt_fog_segment(S, r.o, r.d, R(1e30), seed_key, b, &T, &ins);
                else fog_segment(S.fog, S.sky, r.o, r.d, R(1e30), &T, &ins);
                sky_col = add(scale(sky_col, T), ins);
            }
            radiance = add(radiance, mul(throughput, sky_col));
            break;
        }
        if (medium >= 0) {
            if constexpr (EXTRAS) pt_water_segment(S, medium, r.o, r.d, h.t, seed_key, b, &throughput, &radiance);
            else pt_apply_medium(S.materials[medium], h.t, &throughput, &radiance);
        } else if (EXTRAS && S.fog.density > R(0)) {
            R T;
            V3<R> ins;
            if (b == 0) pt_fog_segment(S, r.o, r.d, h.t, seed_key, b, &T, &ins);
            else fog_segment(S.fog, S.sky, r.o, r.d, h.t, &T, &ins);
            radiance = add(radiance, mul(throughput, ins));
            throughput = scale(throughput, T);
        }
        if (h.material < 0 || h.material >= S.material_count) {
            radiance = add(radiance, mul(throughput, sky_sample<R, EXTRAS>(r.d, S.sky)));
            break;
        }
        const DevMaterial<R> &m = S.materials[h.material];
        V3<R> P = h.point;
        V3<R> d = r.d;
        V3<R> N = h.normal;
        if (m.is_water) {
            if (mfabs(h.normal.y) > R(0.999) && mfabs(h.normal.x) < R(1e-4) && mfabs(h.normal.z) < R(1e-4))
                N = water_normal(P.x, P.z, R(0));
        }
        if (dot(N, d) > R(0)) N = neg(N);
        N = normalize(N);
        if (length_sq(N) <= R(0)) break;
        V3<R> V = neg(d);
        // texture-modulated albedo on a local copy (src/pathtrace.c:903-905)
        DevMaterial<R> m_tex;
        const DevMaterial<R> *mp = &m;
        if (EXTRAS && m.texture_kind != 0) {
            m_tex = m;
            V3<R> a = surface_albedo(S, m, r.o, unit_dir(r.d), h);
            m_tex.albedo[0] = a.x;
            m_tex.albedo[1] = a.y;
            m_tex.albedo[2] = a.z;
            mp = &m_tex;
        }
        const DevMaterial<R> &mm = *mp;
        if (b == 0 || last_bounce_specular) radiance = add(radiance, mul(throughput, mat3(mm.emissive)));
        if (b == 0 && length_sq(mat3(mm.atmosphere_glow)) > R(1e-6))
            radiance = add(radiance, mul(throughput, atmosphere_term(mm, N, V, mat3(S.sky.sun_dir))));
        if (S.light_count > 0)
            radiance = add(radiance, pt_nee_emissive(S, mm, P, N, V, throughput, h.prim, seed_key, b));
        if (b == 0 || (b == 1 && medium >= 0 && last_bounce_specular))
            radiance = add(radiance, pt_nee_sun<R, EXTRAS>(S, mm, P, N, V, throughput, seed_key, b));
        uint32_t kb = hash3(seed_key ^ PT_KEY, (uint32_t)b, 0u);
        R u1 = rand01<R>(kb, (uint32_t)b, PT_CH_BSDF_A);
        R u2 = rand01<R>(kb, (uint32_t)b, PT_CH_BSDF_B);
        R u_lobe = rand01<R>(kb, (uint32_t)b, PT_CH_LOBE);
        R u_glass = rand01<R>(kb, (uint32_t)b, PT_CH_GLASS);
        V3<R> wi, w;
        bool ok;
        int refracted = 0;
        int sampled_specular = 0;
        if (mm.pbr)
            ok = pt_sample_pbr(mm, N, d, V, u1, u2, u_lobe, &wi, &w, &sampled_specular);
        else
            ok = pt_sample_legacy(mm, N, d, V, h.front_face, u1, u2, u_lobe, u_glass, &wi, &w, &refracted,
                                  &sampled_specular);
        if (!ok) break;
        last_bounce_specular = sampled_specular;
        throughput = mul(throughput, w);
        if (!finite3(throughput) || !(pt_max_component(throughput) > R(0))) break;
        if (refracted && (m.is_water || m.beer_lambert)) medium = h.front_face ? h.material : -1;
        if (b >= 2) {  // PT_RR_START_BOUNCE (src/pathtrace.c:69)
            R q = pt_clamp01(pt_max_component(throughput));
            if (!(q > R(0))) break;
            R u_rr = rand01<R>(kb, (uint32_t)b, PT_CH_RR);
            if (u_rr >= q) break;
            throughput = scale(throughput, R(1) / q);
        }
        V3<R> offset;
        if (refracted) offset = scale(wi, R(1e-4));
        else offset = scale(N, dot(wi, N) >= R(0) ? R(1e-4) : R(-1e-4));
        r.o = add(P, offset);
        r.d = wi;
    }
    if (!finite3(radiance)) return v3(R(0), R(0), R(0));
    if (radiance.x < R(0)) radiance.x = R(0);
    if (radiance.y < R(0)) radiance.y = R(0);
    if (radiance.z < R(0)) radiance.z = R(0);
    return radiance;
}

// pathtrace_to_byte / to_byte (src/pathtrace.c:464-480, src/render.c:892-907)
template <typename R> MT_D unsigned char to_byte(R linear)
{
    R c = linear;
    if (!(c >= R(0))) c = R(0);
    else if (c > R(1)) c = R(1);
    R v = mpow(c, R(1) / R(2.2)) * R(255);
    int iv = (int)(v + R(0.5));
    if (iv < 0) iv = 0;
    else if (iv > 255) iv = 255;
    return (unsigned char)iv;
}

// ------------------------------------------------------------------
// Whitted renderer: an explicit stack machine that evaluates the reference's
// recursion trace -> trace_hit -> {trace, trace_hit} (src/render.c:585-863)
// in the same order, so every child colour is combined exactly where the
// reference combines it.
// ------------------------------------------------------------------
enum : int {
    WH_TRACE = 0,    // trace(): intersect, then shade
    WH_HIT = 1,      // trace_hit() on a known hit
    WH_GLOSSY = 2,   // waiting for glossy child i
    WH_REFL = 3,     // waiting for the mirror child
    WH_REFR = 4,     // waiting for the refraction child
};

template <typename R> struct WhFrame {
    V3<R> o, d;          // ray
    V3<R> P, N;          // shading point / normal
    V3<R> color;         // local (ambient + sun + emitters)
    V3<R> refl;          // reflection accumulator
    V3<R> alb;           // the hit's (texture-modulated) albedo
    R t;                 // hit distance (refraction child: the exit distance)
    R F;                 // Schlick at cos_t
    R fog_t;             // trace(): distance fog applies over (1e30 for the sky)
    int mat, prim, front;
    int depth, phase, gi, tir;
    int traced;          // entered through trace(): fog_apply on return (src/render.c:842-863)
};

// The hit fields of a Whitted frame, with its albedo (src/render.c:620-621).
template <typename R, bool EXTRAS>
MT_D void wh_set_hit(const DevScene<R> &S, WhFrame<R> &f, V3<R> o, V3<R> d, const SurfaceHit<R> &h)
{
    f.P = h.point;
    f.N = h.normal;
    f.t = h.t;
    f.mat = h.material;
    f.prim = h.prim;
    f.front = h.front_face;
    if constexpr (EXTRAS)
        if (h.material >= 0 && h.material < S.material_count)
            f.alb = surface_albedo(S, S.materials[h.material], o, unit_dir(d), h);
}

template <typename R>
MT_D V3<R> emissive_direct(const DevScene<R> &S, const DevMaterial<R> &mm, V3<R> P, V3<R> N, V3<R> V, int self_prim,
                           uint32_t seed_key)
{
    V3<R> sum = v3(R(0), R(0), R(0));
    V3<R> shadow_o = add(P, scale(N, R(1e-3)));
    for (int li = 0; li < S.light_count; ++li) {
        const DevLight<R> &lt = S.lights[li];
        if (lt.prim == self_prim) continue;
        V3<R> to_c = sub(mat3(lt.center), P);
        R dc2 = length_sq(to_c);
        R dc = msqrt(dc2);
        if (dc <= lt.radius) continue;
        R cos_mx = msqrt(R(1) - (lt.radius * lt.radius) / dc2);
        const R omc = cone_one_minus_cos((lt.radius * lt.radius) / dc2, cos_mx);
        R solid = R(2) * R(3.14159265358979323846) * omc;
        if (!(solid > R(0))) continue;
        V3<R> w = scale(to_c, R(1) / dc);
        for (int si = 0; si < 16; ++si) {  // EMISSIVE_LIGHT_SAMPLES (src/render.c:448)
            uint32_t k = hash3(seed_key ^ 0xE311u, (uint32_t)li, (uint32_t)si);
            R u1 = rand01<R>(k, (uint32_t)si, 0x4c11u);
            R u2 = rand01<R>(k, (uint32_t)si, 0x9d27u);
            V3<R> w_i = light_sphere_sample_dir(w, cos_mx, omc, u1, u2);
            if (dot(N, w_i) <= R(0)) continue;
            R lt_t;
            bool visible;
            if (light_sphere_t(S, lt.prim, shadow_o, w_i, R(1e-3), R(1e30), &lt_t))
                visible = !scene_occluded(S, shadow_o, w_i, R(1e-3), lt_t - R(1e-3));
            else
                visible = false;
            if (!visible) continue;
            V3<R> rad = scale(mat3(lt.emissive), solid);
            sum = add(sum, shade(mm, N, w_i, V, rad));
        }
    }
    return scale(sum, R(1) / R(16));
}

// EXTRAS = false: the scene has no fog, clouds or textures (DevScene::has_extras).
template <typename R, bool EXTRAS = true>
MT_D V3<R> whitted_trace(const DevScene<R> &S, Ray3<R> ray, int max_depth, uint32_t seed_key)
{
    WhFrame<R> st[kWhittedFrames];
    int sp = 0;
    V3<R> ret = v3(R(0), R(0), R(0));
    const V3<R> zero = v3(R(0), R(0), R(0));
    const V3<R> sun_dir = mat3(S.sky.sun_dir);
    const V3<R> sun_color = mat3(S.sky.sun_color);

    st[0].o = ray.o;
    st[0].d = ray.d;
    st[0].depth = 0;
    st[0].phase = WH_TRACE;
    st[0].traced = 0;
    sp = 1;
    // a frame's result, with trace()'s fog when it entered through trace()
    auto fogged = [&](const WhFrame<R> &fr, V3<R> c) {
        return (EXTRAS && fr.traced && S.fog.density > R(0)) ? fog_apply(S.fog, S.sky, fr.o, fr.d, fr.fog_t, c) : c;
    };
    int guard = 0;
    while (sp > 0) {
        if (++guard > (1 << 24)) {
            atomicOr(S.err, ERR_WATCHDOG);
            return zero;
        }
        WhFrame<R> &f = st[sp - 1];
        bool finish = false;   // compute the frame's output colour and pop
        bool refl_done = false;
        switch (f.phase) {
        case WH_TRACE: {
            if (f.depth > max_depth) {
                ret = zero;
                --sp;
                continue;
            }
            SurfaceHit<R> h;
            // The hit point and facing use the normalised direction (inside
            // scene_intersect); everything else sees the ray's own direction,
            // as src/render.c:842-863 passes `r` through unchanged.
            f.traced = 1;
            if (!scene_intersect(S, f.o, f.d, R(1e-4), R(1e30), &h)) {
                f.fog_t = R(1e30);
                ret = fogged(f, sky_sample<R, EXTRAS>(f.d, S.sky));
                --sp;
                continue;
            }
            f.fog_t = h.t;
            wh_set_hit<R, EXTRAS>(S, f, f.o, f.d, h);
        }
        // fall through: shade the hit
        case WH_HIT: {
            if (f.depth > max_depth) {
                ret = zero;
                --sp;
                continue;
            }
            if (f.mat < 0 || f.mat >= S.material_count) {
                ret = fogged(f, sky_sample<R, EXTRAS>(f.d, S.sky));
                --sp;
                continue;
            }
            const DevMaterial<R> &m0 = S.materials[f.mat];
            DevMaterial<R> m_tex;
            const DevMaterial<R> *mp = &m0;
            if (EXTRAS && m0.texture_kind != 0) {
                m_tex = m0;
                m_tex.albedo[0] = f.alb.x;
                m_tex.albedo[1] = f.alb.y;
                m_tex.albedo[2] = f.alb.z;
                mp = &m_tex;
            }
            const DevMaterial<R> &m = *mp;
            if (m.is_water) f.N = water_normal(f.P.x, f.P.z, R(0));
            if (dot(f.N, f.d) > R(0)) f.N = neg(f.N);
            V3<R> V = neg(f.d);
            V3<R> color = material_ambient(m, f.N, S.sky);
            V3<R> shadow_o = add(f.P, scale(f.N, R(1e-3)));
            R sun_radius = S.sky.sun_radius;
            if (sun_radius > R(1e-9)) {
                R lit = R(0);
                for (int i = 0; i < 16; ++i) {  // SUN_SHADOW_SAMPLES (src/render.c:408)
                    uint32_t k = seed_key * 0x9e3779b9u + (uint32_t)i * 2u;
                    R r1 = rand01<R>(k, (uint32_t)i, 0x5a17u);
                    R r2 = rand01<R>(k, (uint32_t)i, 0x7c3du);
                    V3<R> Ld = sun_disk_dir(sun_dir, sun_radius, r1, r2);
                    if (!scene_occluded(S, shadow_o, Ld, R(1e-3), R(1e30))) lit += R(1);
                }
                if (lit > R(0)) color = add(color, scale(shade(m, f.N, sun_dir, V, sun_color), lit / R(16)));
            } else {
                if (!scene_occluded(S, shadow_o, sun_dir, R(1e-3), R(1e30)))
                    color = add(color, shade(m, f.N, sun_dir, V, sun_color));
            }
            if (S.light_count > 0) color = add(color, emissive_direct(S, m, f.P, f.N, V, f.prim, seed_key));
            f.color = color;
            f.refl = zero;
            if (f.depth < max_depth) {
                if (sp >= kWhittedFrames) {
                    atomicOr(S.err, ERR_WHITTED);
                    return zero;
                }
                WhFrame<R> &c = st[sp];
                c.depth = f.depth + 1;
                c.phase = WH_TRACE;
                c.o = add(f.P, scale(f.N, R(1e-3)));
                if (m.pbr != 0 && m.reflectivity > R(0) && m.roughness > R(1e-6)) {
                    f.gi = 0;
                    f.phase = WH_GLOSSY;
                    uint32_t k = seed_key * 0x9e3779b9u + (uint32_t)f.depth * 0x85ebca6bu;
                    R r1 = rand01<R>(k, 0u, 0x9e37u);
                    R r2 = rand01<R>(k, 0u, 0x85ebu);
                    c.d = sample_glossy_dir(m, f.N, f.d, r1, r2);
                } else {
                    f.phase = WH_REFL;
                    c.d = reflect(f.d, f.N);
                }
                ++sp;
                continue;
            }
            refl_done = true;
            break;
        }
        case WH_GLOSSY: {
            const DevMaterial<R> &m = S.materials[f.mat];
            f.refl = add(f.refl, scale(ret, R(1) / R(16)));
            f.gi++;
            if (f.gi < 16) {  // GLOSSY_REFLECTION_SAMPLES (src/render.c:427)
                WhFrame<R> &c = st[sp];
                c.depth = f.depth + 1;
                c.phase = WH_TRACE;
                c.o = add(f.P, scale(f.N, R(1e-3)));
                uint32_t k = seed_key * 0x9e3779b9u + (uint32_t)f.depth * 0x85ebca6bu + (uint32_t)f.gi * 2u;
                R r1 = rand01<R>(k, (uint32_t)f.gi, 0x9e37u);
                R r2 = rand01<R>(k, (uint32_t)f.gi, 0x85ebu);
                c.d = sample_glossy_dir(m, f.N, f.d, r1, r2);
                ++sp;
                continue;
            }
            refl_done = true;
            break;
        }
        case WH_REFL:
            f.refl = ret;
            refl_done = true;
            break;
        case WH_REFR: {
            const DevMaterial<R> &m = S.materials[f.mat];
            V3<R> inner = ret;
            V3<R> refr = (m.is_water || m.beer_lambert) ? water_attenuate(m, inner, f.t) : inner;
            ret = refr;
            finish = true;
            break;
        }
        default:
            return zero;
        }

        if (refl_done) {
            // Fresnel at the refracted cosine, TIR detection (src/render.c:739-763)
            const DevMaterial<R> &m = S.materials[f.mat];
            R f0 = (R(1) - m.ior) / (R(1) + m.ior);
            f0 = f0 * f0;
            V3<R> V = neg(f.d);
            R cos_i = dot(f.N, V);
            if (cos_i < R(0)) cos_i = R(0);
            else if (cos_i > R(1)) cos_i = R(1);
            R eta = (f.front == 1) ? (R(1) / m.ior) : m.ior;
            R sin2_t = eta * eta * (R(1) - cos_i * cos_i);
            f.tir = 0;
            if (sin2_t > R(1)) {
                f.F = R(1);
                f.tir = 1;
            } else {
                R cos_t = msqrt(R(1) - sin2_t);
                f.F = fresnel_schlick(cos_t, f0);
            }
            if (m.transparency > R(0)) {
                if (f.tir) {
                    ret = f.refl;
                    finish = true;
                } else {
                    V3<R> rd = vec3_refract(f.d, f.N, eta);
                    V3<R> ro = add(f.P, scale(rd, R(1e-3)));
                    SurfaceHit<R> h2;
                    if (scene_intersect(S, ro, rd, R(1e-4), R(1e30), &h2)) {
                        if (sp >= kWhittedFrames) {
                            atomicOr(S.err, ERR_WHITTED);
                            return zero;
                        }
                        f.phase = WH_REFR;
                        f.t = h2.t;
                        WhFrame<R> &c = st[sp];
                        c.o = ro;
                        c.d = rd;
                        c.depth = f.depth + 1;
                        c.phase = WH_HIT;
                        c.traced = 0;  // trace_hit directly: no fog (src/render.c:786-790)
                        wh_set_hit<R, EXTRAS>(S, c, ro, rd, h2);
                        ++sp;
                        continue;
                    }
                    V3<R> inner = sky_sample<R, EXTRAS>(rd, S.sky);
                    ret = (m.is_water || m.beer_lambert) ? water_attenuate(m, inner, R(5.0)) : inner;
                    finish = true;
                }
            } else {
                // Opaque: mix with the reflection (src/render.c:813-839)
                V3<R> out = lerp(f.color, f.refl, m.reflectivity);
                if (m.pbr && (m.emissive[0] != R(0) || m.emissive[1] != R(0) || m.emissive[2] != R(0)))
                    out = add(out, mat3(m.emissive));
                if (f.depth == 0 && length_sq(mat3(m.atmosphere_glow)) > R(1e-6))
                    out = add(out, atmosphere_term(m, f.N, V, sun_dir));
                ret = fogged(f, out);
                --sp;
                continue;
            }
        }
        if (finish) {
            // Transparent surface: ret holds refr_col (src/render.c:800-812)
            const DevMaterial<R> &m = S.materials[f.mat];
            V3<R> surface = add(scale(f.refl, f.F), scale(ret, R(1) - f.F));
            V3<R> out = lerp(f.color, surface, m.transparency);
            if (m.pbr && (m.emissive[0] != R(0) || m.emissive[1] != R(0) || m.emissive[2] != R(0)))
                out = add(out, mat3(m.emissive));
            ret = fogged(f, out);
            --sp;
            continue;
        }
    }
    return ret;
}

}  // namespace mt
