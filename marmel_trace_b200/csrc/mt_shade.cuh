// mt_shade.cuh - materials, procedural sky, noise, water and BSDF sampling.
//
// Each function restates the reference function cited beside it in the
// reference's expression order, so the FP64 instantiation reproduces the
// reference's doubles; the FP32 instantiation evaluates the same formulas in
// single precision with CUDA's float math functions.
#pragma once

#include "mt_geom.cuh"

namespace mt {

template <typename R> MT_D V3<R> mat3(const R *p) { return v3(p[0], p[1], p[2]); }

// ------------------------------------------------------------------
// Noise (src/noise.c:31-55,158-187,272-294)
// ------------------------------------------------------------------
MT_D uint32_t noise_mix(uint32_t x)
{
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}

MT_D uint32_t noise_hash(int x, int y, int z, uint32_t seed)
{
    uint32_t h = seed + 0x9e3779b9u;
    h ^= (uint32_t)x * 0x85ebca6bu;
    h ^= (uint32_t)y * 0xc2b2ae35u;
    h ^= (uint32_t)z * 0x27d4eb2fu;
    return noise_mix(h);
}

template <typename R> MT_D R noise_rand01(int x, int y, int z, uint32_t seed)
{
    return R(noise_hash(x, y, z, seed)) / R(4294967295.0);
}

template <typename R> MT_D R noise_fade(R t) { return t * t * t * (t * (t * R(6) - R(15)) + R(10)); }
template <typename R> MT_D R noise_lerp(R a, R b, R t) { return a + t * (b - a); }
template <typename R> MT_D R noise_clamp(R v, R lo, R hi)
{
    if (v < lo) return lo;
    if (v > hi) return hi;
    return v;
}

// noise_perlin2 (src/noise.c:158-187)
template <typename R> MT_D R noise_perlin2(R x, R y, uint32_t seed)
{
    R fx = mfloor(x);
    R fy = mfloor(y);
    int ix = (int)fx;
    int iy = (int)fy;
    R rx = x - fx;
    R ry = y - fy;
    R u = noise_fade(rx);
    R v = noise_fade(ry);
    const R tp = R(2) * Const<R>::pi;
    R a00 = noise_rand01<R>(ix, iy, 0, seed) * tp;
    R a10 = noise_rand01<R>(ix + 1, iy, 0, seed) * tp;
    R a01 = noise_rand01<R>(ix, iy + 1, 0, seed) * tp;
    R a11 = noise_rand01<R>(ix + 1, iy + 1, 0, seed) * tp;
    R s00, c00, s10, c10, s01, c01, s11, c11;
    msincos(a00, &s00, &c00);
    msincos(a10, &s10, &c10);
    msincos(a01, &s01, &c01);
    msincos(a11, &s11, &c11);
    R d00 = c00 * rx + s00 * ry;
    R d10 = c10 * (rx - R(1)) + s10 * ry;
    R d01 = c01 * rx + s01 * (ry - R(1));
    R d11 = c11 * (rx - R(1)) + s11 * (ry - R(1));
    R x0 = noise_lerp(d00, d10, u);
    R x1 = noise_lerp(d01, d11, u);
    R val = noise_lerp(x0, x1, v);
    return noise_clamp(val * R(1.4142135623730951), R(-1), R(1));
}

// noise_fbm2 with lacunarity 2 and gain 0.5 (src/noise.c:272-294)
template <typename R> MT_D R noise_fbm2(R x, R y, int octaves, uint32_t seed)
{
    int n = octaves <= 0 ? 1 : octaves;
    R amp = R(1), freq = R(1), sum = R(0), norm = R(0);
    for (int i = 0; i < n; ++i) {
        sum += amp * noise_perlin2(x * freq, y * freq, seed);
        norm += amp;
        amp *= R(0.5);
        freq *= R(2);
    }
    if (norm <= R(0)) return R(0);
    return noise_clamp(sum / norm, R(-1), R(1));
}

template <typename R> MT_D R noise_rand_signed(int x, int y, int z, uint32_t seed)
{
    return noise_rand01<R>(x, y, z, seed) * R(2) - R(1);
}

// noise_perlin3 (src/noise.c:189-246)
template <typename R> MT_D R noise_perlin3(R x, R y, R z, uint32_t seed)
{
    R fx = mfloor(x), fy = mfloor(y), fz = mfloor(z);
    int ix = (int)fx, iy = (int)fy, iz = (int)fz;
    R rx = x - fx, ry = y - fy, rz = z - fz;
    R u = noise_fade(rx), v = noise_fade(ry), w = noise_fade(rz);
    R dotv[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        int cx = ix + (i & 1), cy = iy + ((i >> 1) & 1), cz = iz + ((i >> 2) & 1);
        R gx = noise_rand_signed<R>(cx, cy, cz, seed);
        R gy = noise_rand_signed<R>(cx, cy, cz, seed ^ 0x68bc21ebu);
        R gz = noise_rand_signed<R>(cx, cy, cz, seed ^ 0x02e5be93u);
        R len = msqrt(gx * gx + gy * gy + gz * gz);
        if (len < R(1e-12)) {
            gx = R(1);
            gy = R(0);
            gz = R(0);
        } else {
            gx /= len;
            gy /= len;
            gz /= len;
        }
        R dx = rx - R(i & 1), dy = ry - R((i >> 1) & 1), dz = rz - R((i >> 2) & 1);
        dotv[i] = gx * dx + gy * dy + gz * dz;
    }
    R x00 = noise_lerp(dotv[0], dotv[1], u);
    R x10 = noise_lerp(dotv[2], dotv[3], u);
    R x01 = noise_lerp(dotv[4], dotv[5], u);
    R x11 = noise_lerp(dotv[6], dotv[7], u);
    R y0 = noise_lerp(x00, x10, v);
    R y1 = noise_lerp(x01, x11, v);
    R val = noise_lerp(y0, y1, w);
    return noise_clamp(val * R(1.1547005383792515), R(-1), R(1));
}

// noise_fbm3 with lacunarity 2 and gain 0.5, the only values its callers use
// (src/noise.c:296-317)
template <typename R> MT_D R noise_fbm3(R x, R y, R z, int octaves, uint32_t seed)
{
    int n = octaves <= 0 ? 1 : octaves;
    R amp = R(1), freq = R(1), sum = R(0), norm = R(0);
    for (int i = 0; i < n; ++i) {
        sum += amp * noise_perlin3(x * freq, y * freq, z * freq, seed);
        norm += amp;
        amp *= R(0.5);
        freq *= R(2);
    }
    if (norm <= R(0)) return R(0);
    return noise_clamp(sum / norm, R(-1), R(1));
}

// ------------------------------------------------------------------
// Sky (sky_sample, src/material.c:473-600,956: gradient, sun glow, volumetric
// or planar clouds; the star / nebula / galaxy terms are rejected on upload)
// ------------------------------------------------------------------
template <typename R> MT_D R smoothstep(R e0, R e1, R x)
{
    R denom = e1 - e0;
    if (denom == R(0)) return x < e0 ? R(0) : R(1);
    R t = mat_clamp01((x - e0) / denom);
    return t * t * (R(3) - R(2) * t);
}

template <typename R> MT_D R pow_nonneg(R base, R e)
{
    if (base <= R(0)) return R(0);
    return mpow(base, e);
}

template <typename R> MT_D void basis(V3<R> n, V3<R> *t, V3<R> *b);

// eval_cloud_density_at (src/material.c:376-408)
template <typename R> MT_D R cloud_density_at(const DevSky<R> &sky, V3<R> p)
{
    if (sky.cloud_thickness <= R(1e-4)) return R(0);
    R y_bot = sky.cloud_height;
    R y_top = y_bot + sky.cloud_thickness;
    if (p.y < y_bot || p.y > y_top) return R(0);
    R h_rel = (p.y - y_bot) / sky.cloud_thickness;
    R vert_profile = smoothstep(R(0), R(0.12), h_rel) * smoothstep(R(1), R(0.60), h_rel);
    if (vert_profile <= R(0)) return R(0);
    int octaves = sky.cloud_octaves;
    if (octaves < 1) octaves = 1;
    if (octaves > 6) octaves = 6;
    R sx = p.x * sky.cloud_scale;
    R sy = (p.y - y_bot) * (sky.cloud_scale * R(1.5));
    R sz = p.z * sky.cloud_scale;
    R raw = noise_fbm3(sx, sy, sz, octaves, sky.seed);
    R d0 = mat_clamp01(R(0.5) * (raw + R(1)));
    R d = d0 * vert_profile;
    R a = sky.cloud_coverage - sky.cloud_softness;
    R b = sky.cloud_coverage + sky.cloud_softness;
    R alpha = smoothstep(a, b, d);
    if (alpha <= R(0)) return R(0);
    alpha = pow_nonneg(alpha, sky.cloud_sharpness);
    R mult = (sky.cloud_density > R(0)) ? sky.cloud_density : R(0.08);
    return alpha * mult;
}

// sky_cloud_transmittance (src/material.c:410-466): grey transmittance of
// the cloud slab from pos along dir, with the crepuscular shaft modulation.
template <typename R> MT_NOINLINE R cloud_transmittance_march(const DevSky<R> &sky, V3<R> pos, V3<R> dir)
{
    if (dir.y <= R(1e-4)) return R(1);
    R y_bot = sky.cloud_height;
    R y_top = y_bot + sky.cloud_thickness;
    R t0 = (y_bot - pos.y) / dir.y;
    R t1 = (y_top - pos.y) / dir.y;
    R t_start = (t0 > R(0)) ? t0 : R(0);
    R t_end = t1;
    if (t_end <= t_start) return R(1);
    R slab_dist = t_end - t_start;
    if (slab_dist > R(3000)) slab_dist = R(3000);
    int steps = sky.cloud_steps / 2;
    if (steps < 4) steps = 4;
    if (steps > 16) steps = 16;
    R dt = slab_dist / R(steps);
    R tau = R(0);
    for (int i = 0; i < steps; ++i) {
        R t = t_start + (R(i) + R(0.5)) * dt;
        V3<R> p = add(pos, scale(dir, t));
        R rho = cloud_density_at(sky, p);
        tau += rho * dt;
        if (tau > R(15)) {
            tau = R(15);
            break;
        }
    }
    R T = mexp(-tau);
    V3<R> u_dir, v_dir;
    basis(mat3(sky.sun_dir), &u_dir, &v_dir);
    R u = dot(pos, u_dir);
    R v = dot(pos, v_dir);
    const R shaft_scale = R(0.22);
    R raw_shaft = noise_fbm2(u * shaft_scale, v * shaft_scale, 3, sky.seed ^ 0x9E3779B9u);
    R shaft = smoothstep(R(-0.25), R(0.35), raw_shaft);
    R beam_factor = R(0.12) + R(0.88) * shaft;
    T *= beam_factor;
    return T;
}

template <typename R> MT_D R cloud_transmittance(const DevSky<R> &sky, V3<R> pos, V3<R> dir)
{
    if (sky.cloud_thickness <= R(1e-4)) return R(1);
    return cloud_transmittance_march(sky, pos, dir);
}

// The volumetric slab of sky_sample (src/material.c:493-556): the cloud march
// blended over `base`.
template <typename R> MT_NOINLINE V3<R> sky_clouds_volumetric(V3<R> dir, const DevSky<R> &sky, V3<R> base, R cos_sun)
{
    if (!(dir.y > R(0.01))) return base;
    const V3<R> sun_color = mat3(sky.sun_color);
    R y_bot = sky.cloud_height;
    R y_top = y_bot + sky.cloud_thickness;
    R t0 = y_bot / dir.y;
    R t1 = y_top / dir.y;
    R slab_dist = t1 - t0;
    if (slab_dist > R(3500)) slab_dist = R(3500);
    int steps = sky.cloud_steps;
    if (steps < 4) steps = 4;
    if (steps > 64) steps = 64;
    R dt = slab_dist / R(steps);
    V3<R> cloud_albedo = v3(R(0.96), R(0.97), R(0.98));
    V3<R> sky_ambient = lerp(mat3(sky.horizon_color), mat3(sky.zenith_color), R(0.55));
    V3<R> ambient_col = scale(mul(cloud_albedo, sky_ambient), R(0.60));
    R lit = (cos_sun > R(0)) ? cos_sun : R(0);
    R silver = R(0.50) * pow_nonneg(mfmax(R(0), cos_sun), R(14));
    R T_acc = R(1);
    V3<R> cloud_inscatter = v3(R(0), R(0), R(0));
    V3<R> sun_dir = mat3(sky.sun_dir);
    for (int i = 0; i < steps; ++i) {
        R tt = t0 + (R(i) + R(0.5)) * dt;
        V3<R> p = scale(dir, tt);
        R rho = cloud_density_at(sky, p);
        if (rho <= R(1e-5)) continue;
        R sun_tau = R(0);
        if (sun_dir.y > R(0.02)) {
            R t_sun_top = (y_top - p.y) / sun_dir.y;
            if (t_sun_top > R(0)) {
                R dt_sun = t_sun_top / R(4);
                for (int k = 0; k < 4; ++k) {
                    V3<R> p_sun = add(p, scale(sun_dir, (R(k) + R(0.5)) * dt_sun));
                    sun_tau += cloud_density_at(sky, p_sun) * dt_sun;
                }
            }
        }
        R T_sun = mexp(-sun_tau) + R(0.25) * mexp(-sun_tau * R(0.30));
        V3<R> sun_lit = scale(sun_color, (R(0.35) * lit + silver) * T_sun);
        V3<R> step_col = add(ambient_col, mul(cloud_albedo, sun_lit));
        R step_tau = rho * dt;
        R step_T = mexp(-step_tau);
        cloud_inscatter = add(cloud_inscatter, scale(step_col, (R(1) - step_T) * T_acc));
        T_acc *= step_T;
        if (T_acc < R(0.005)) break;
    }
    R horizon_fade = smoothstep(R(0.01), R(0.08), dir.y);
    V3<R> combined = add(scale(base, T_acc), cloud_inscatter);
    return lerp(base, combined, horizon_fade);
}

// VOL = false: a caller that knows the sky has no volumetric slab (the
// branch is then compiled out).
template <typename R, bool VOL = true> MT_D V3<R> sky_sample(V3<R> dir, const DevSky<R> &sky)
{
    R h = mat_clamp01(dir.y);
    R t = pow_nonneg(h, sky.gradient_gamma);
    V3<R> base = lerp(mat3(sky.horizon_color), mat3(sky.zenith_color), t);
    V3<R> sun_color = mat3(sky.sun_color);
    R cos_sun = dot(dir, mat3(sky.sun_dir));
    if (cos_sun > R(0)) {
        R glow = pow_nonneg(cos_sun, sky.sun_glow_exponent) * sky.sun_glow_strength;
        base = add(base, scale(sun_color, glow));
    }
    if (VOL && sky.cloud_thickness > R(1e-4)) {
        if constexpr (VOL) base = sky_clouds_volumetric(dir, sky, base, cos_sun);
    } else if (dir.y > R(0.03)) {
        // planar clouds (src/material.c:557-595)
        R tt = sky.cloud_height / dir.y;
        R px = dir.x * tt;
        R pz = dir.z * tt;
        int octaves = sky.cloud_octaves;
        if (octaves < 1) octaves = 1;
        R raw = noise_fbm2(px * sky.cloud_scale, pz * sky.cloud_scale, octaves, sky.seed);
        R density = mat_clamp01(R(0.5) * (raw + R(1)));
        R a = sky.cloud_coverage - sky.cloud_softness;
        R b = sky.cloud_coverage + sky.cloud_softness;
        R alpha = smoothstep(a, b, density);
        alpha = pow_nonneg(alpha, sky.cloud_sharpness);
        alpha *= smoothstep(R(0), R(0.15), dir.y);
        if (alpha > R(0)) {
            R shadow = R(0.6) + R(0.4) * alpha;
            V3<R> cloud_color = scale(v3(R(0.95), R(0.95), R(0.98)), shadow);
            R lit = cos_sun > R(0) ? cos_sun : R(0);
            V3<R> lit_cloud = add(cloud_color, scale(mul(cloud_color, sun_color), R(0.35) * lit));
            base = lerp(base, lit_cloud, alpha);
        }
    }
    if (!(base.x >= R(0))) base.x = R(0);
    if (!(base.y >= R(0))) base.y = R(0);
    if (!(base.z >= R(0))) base.z = R(0);
    return base;
}

// ------------------------------------------------------------------
// Fog (fog_segment / fog_apply, src/material.c:963-1053)
// ------------------------------------------------------------------
// The fBm turbulence factor of fog density at p (src/material.c:1000-1011,
// src/pathtrace.c:674-684).
template <typename R> MT_D R fog_noise_mod(const DevFog<R> &fog, V3<R> p)
{
    R n = noise_fbm3(p.x * fog.noise_scale, p.y * fog.noise_scale, p.z * fog.noise_scale, 3, 1337u);
    R turb = R(0.5) * (n + R(1));
    if (turb < R(0)) turb = R(0);
    if (turb > R(1)) turb = R(1);
    return (R(1) - fog.noise_amount) + fog.noise_amount * turb * R(2);
}

// Henyey-Greenstein phase toward the sun with g clamped to +-0.95.
template <typename R> MT_D R fog_phase_hg(const DevFog<R> &fog, V3<R> dir, V3<R> sun_dir)
{
    R g = fog.sun_anisotropy;
    if (g < R(-0.95)) g = R(-0.95);
    if (g > R(0.95)) g = R(0.95);
    R cos_theta = dot(dir, sun_dir);
    R denom = R(1) + g * g - R(2) * g * cos_theta;
    if (denom < R(1e-4)) denom = R(1e-4);
    return (R(1) - g * g) / (denom * msqrt(denom));
}

template <typename R>
MT_NOINLINE void fog_segment(const DevFog<R> &fog, const DevSky<R> &sky, V3<R> o, V3<R> d, R dist, R *transmittance,
                             V3<R> *inscatter)
{
    *transmittance = R(1);
    *inscatter = v3(R(0), R(0), R(0));
    if (fog.density <= R(0) || dist <= R(1e-7)) return;
    R rho0 = fog.density;
    R lambda = (fog.height_falloff > R(0)) ? fog.height_falloff : R(0);
    R y0 = o.y - fog.height;
    R dy = d.y;
    R tau = R(0);
    bool is_sky = dist >= R(1e20);
    if (lambda <= R(1e-6)) {
        tau = is_sky ? R(1e6) : (rho0 * dist);
    } else {
        R base_density = rho0 * mexp(-lambda * y0);
        if (is_sky) {
            tau = (dy > R(1e-5)) ? base_density / (lambda * dy) : R(1e6);
        } else if (mfabs(dy) < R(1e-5)) {
            tau = base_density * dist;
        } else {
            R term = (R(1) - mexp(-lambda * dy * dist)) / (lambda * dy);
            tau = base_density * term;
        }
    }
    if (tau < R(0)) tau = R(0);
    if (fog.noise_amount > R(1e-4) && fog.noise_scale > R(1e-4)) {
        R eval_dist = is_sky ? R(20) : (dist > R(50) ? R(50) : dist * R(0.5));
        tau *= fog_noise_mod(fog, add(o, scale(d, eval_dist)));
    }
    R T = mexp(-tau);
    if (T < R(0)) T = R(0);
    if (T > R(1)) T = R(1);
    V3<R> inscatter_col = mat3(fog.color);
    if (fog.inscatter_strength > R(0)) {
        R phase = fog_phase_hg(fog, d, mat3(sky.sun_dir));
        inscatter_col = add(inscatter_col, scale(mat3(sky.sun_color), phase * fog.inscatter_strength));
    }
    *transmittance = T;
    *inscatter = scale(inscatter_col, R(1) - T);
}

template <typename R>
MT_D V3<R> fog_apply(const DevFog<R> &fog, const DevSky<R> &sky, V3<R> o, V3<R> d, R dist, V3<R> surface)
{
    if (fog.density <= R(0)) return surface;
    R T;
    V3<R> inscatter;
    fog_segment(fog, sky, o, d, dist, &T, &inscatter);
    return add(scale(surface, T), inscatter);
}

// ------------------------------------------------------------------
// Textures (texture_albedo_uv, src/texture.c:269-327)
// ------------------------------------------------------------------
template <typename R> MT_D R texture_scale_or_default(const DevMaterial<R> &m)
{
    R s = m.texture_scale;
    return (s > R(0)) ? s : R(1);
}

template <typename R> MT_D V3<R> texture_planet_earth(const DevMaterial<R> &m, V3<R> p)
{
    R s = R(1) / texture_scale_or_default(m);
    V3<R> q = scale(p, s);
    R elev = noise_fbm3(q.x * R(1.6), q.y * R(1.6), q.z * R(1.6), 7, 42u);
    V3<R> surf;
    if (elev < R(0)) {
        R t = mat_clamp01((elev + R(0.25)) / R(0.25));
        surf = lerp(v3(R(0.02), R(0.05), R(0.20)), v3(R(0.04), R(0.18), R(0.35)), t);
    } else {
        R t = mat_clamp01(elev / R(0.45));
        const V3<R> land_low = v3(R(0.12), R(0.22), R(0.08)), land_mid = v3(R(0.26), R(0.24), R(0.14));
        const V3<R> land_arid = v3(R(0.42), R(0.35), R(0.20)), snow = v3(R(0.88), R(0.90), R(0.94));
        if (t < R(0.35)) surf = lerp(land_low, land_mid, t / R(0.35));
        else if (t < R(0.70)) surf = lerp(land_mid, land_arid, (t - R(0.35)) / R(0.35));
        else surf = lerp(land_arid, snow, (t - R(0.70)) / R(0.30));
    }
    R warp = noise_fbm3(q.x * R(2.2) + R(7.3), q.y * R(2.2) + R(7.3), q.z * R(2.2) + R(7.3), 4, 101u);
    R c_noise = noise_fbm3(q.x * R(2.6) + warp * R(0.4), q.y * R(2.6) + warp * R(0.4), q.z * R(2.6) + warp * R(0.4),
                           6, 999u);
    R c_cov = smoothstep(R(0.02), R(0.38), c_noise);
    V3<R> result = lerp(surf, v3(R(0.92), R(0.94), R(0.96)), c_cov * R(0.88));
    return mul(mat3(m.albedo), result);
}

template <typename R> MT_D V3<R> texture_planet_moon(const DevMaterial<R> &m, V3<R> p)
{
    R s = R(1) / texture_scale_or_default(m);
    V3<R> q = scale(p, s);
    R maria = noise_fbm3(q.x * R(1.2), q.y * R(1.2), q.z * R(1.2), 5, 77u);
    R crater = noise_fbm3(q.x * R(4.5), q.y * R(4.5), q.z * R(4.5), 6, 555u);
    R micro = noise_fbm3(q.x * R(16), q.y * R(16), q.z * R(16), 4, 888u);
    R m_blend = mat_clamp01((maria + R(0.12)) / R(0.38));
    V3<R> base = lerp(v3(R(0.075), R(0.075), R(0.072)), v3(R(0.165), R(0.160), R(0.150)), m_blend);
    R detail = R(1) + R(0.32) * crater + R(0.14) * micro;
    V3<R> result = scale(base, detail);
    if (crater > R(0.40)) {
        R ray_t = mat_clamp01((crater - R(0.40)) / R(0.25));
        result = lerp(result, v3(R(0.250), R(0.245), R(0.235)), ray_t * R(0.75));
    }
    return mul(mat3(m.albedo), result);
}

// Exact sRGB byte to linear (src/texture.c:57-61).
template <typename R> MT_D R srgb_to_linear(unsigned char byte)
{
    R c = R(byte) / R(255);
    return (c <= R(0.04045)) ? (c / R(12.92)) : mpow((c + R(0.055)) / R(1.055), R(2.4));
}

// texture_image_sample (src/texture.c:212-263): wrapped bilinear lookup.
template <typename R> MT_D V3<R> texture_image_sample(const DevMaterial<R> &m, R u, R v)
{
    const int w = m.texture_width, h = m.texture_height;
    u = u - mfloor(u);
    v = v - mfloor(v);
    R px = u * R(w) - R(0.5);
    R py = (R(1) - v) * R(h) - R(0.5);
    int x0 = (int)mfloor(px), y0 = (int)mfloor(py);
    int x1 = x0 + 1, y1 = y0 + 1;
    R fx = px - R(x0), fy = py - R(y0);
    x0 = ((x0 % w) + w) % w;
    x1 = ((x1 % w) + w) % w;
    y0 = ((y0 % h) + h) % h;
    y1 = ((y1 % h) + h) % h;
    const unsigned char *p00 = m.texture_rgb + ((size_t)y0 * w + x0) * 3;
    const unsigned char *p10 = m.texture_rgb + ((size_t)y0 * w + x1) * 3;
    const unsigned char *p01 = m.texture_rgb + ((size_t)y1 * w + x0) * 3;
    const unsigned char *p11 = m.texture_rgb + ((size_t)y1 * w + x1) * 3;
    R w00 = (R(1) - fx) * (R(1) - fy);
    R w10 = fx * (R(1) - fy);
    R w01 = (R(1) - fx) * fy;
    R w11 = fx * fy;
    R c[3];
    for (int k = 0; k < 3; ++k)
        c[k] = w00 * srgb_to_linear<R>(p00[k]) + w10 * srgb_to_linear<R>(p10[k]) + w01 * srgb_to_linear<R>(p01[k]) +
               w11 * srgb_to_linear<R>(p11[k]);
    return v3(c[0], c[1], c[2]);
}

// Parity bit of floor(x) (as the reference's long long cast, & 1).
template <typename R> MT_D int floor_parity(R x) { return (int)(((long long)mfloor(x)) & 1); }

// Albedo of material m at world point p with hit (u, v).
template <typename R> MT_NOINLINE V3<R> texture_albedo_uv(const DevMaterial<R> &m, V3<R> p, R u, R v)
{
    switch (m.texture_kind) {
    case 1: {  // TEXTURE_CHECKER
        R inv_scale = R(1) / texture_scale_or_default(m);
        int parity = (floor_parity(p.x * inv_scale) + floor_parity(p.y * inv_scale) + floor_parity(p.z * inv_scale)) & 1;
        return mul(mat3(m.albedo), parity ? mat3(m.texture_color_a) : mat3(m.texture_color_b));
    }
    case 2: {  // TEXTURE_STRIPES
        R s = texture_scale_or_default(m);
        R wave = R(0.5) * (R(1) + msin(p.y * s * (R(2) * R(3.14159265358979323846))));
        return mul(mat3(m.albedo), (wave >= R(0.5)) ? mat3(m.texture_color_a) : mat3(m.texture_color_b));
    }
    case 3:
        return texture_planet_earth(m, p);
    case 4:
        return texture_planet_moon(m, p);
    case 5: {  // TEXTURE_NOISE (src/texture.c:154-162)
        R s = R(1) / texture_scale_or_default(m);
        V3<R> q = scale(p, s);
        R n = noise_fbm3(q.x, q.y, q.z, 6, 1337u);
        R t = mat_clamp01(R(0.5) * (n + R(1)));
        return mul(mat3(m.albedo), lerp(mat3(m.texture_color_a), mat3(m.texture_color_b), t));
    }
    case 7: {  // TEXTURE_UV_CHECKER
        R s = texture_scale_or_default(m);
        int parity = (floor_parity(u * s) + floor_parity(v * s)) & 1;
        return mul(mat3(m.albedo), parity ? mat3(m.texture_color_a) : mat3(m.texture_color_b));
    }
    case 6:  // TEXTURE_IMAGE
        if (m.texture_rgb) {
            R s = (m.texture_scale > R(0)) ? m.texture_scale : R(1);
            return mul(mat3(m.albedo), texture_image_sample(m, u * s, v * s));
        }
        return mat3(m.albedo);
    default:
        return mat3(m.albedo);
    }
}

// True for the kinds whose albedo reads the hit's (u, v).
MT_HD bool texture_uses_uv(int kind) { return kind == 6 || kind == 7; }

// The albedo a surface hit shades with: texture_albedo_uv at the hit point
// and the hit's (u, v) (src/pathtrace.c:903-905, src/render.c:620-621).
// o, du: the ray of the hit with its unit direction.
template <typename R>
MT_D V3<R> surface_albedo(const DevScene<R> &S, const DevMaterial<R> &m, V3<R> o, V3<R> du, const SurfaceHit<R> &h)
{
    if (m.texture_kind == 0) return mat3(m.albedo);
    R u = R(0), v = R(0);
    if (texture_uses_uv(m.texture_kind)) {
        Hit<R> th;
        th.t = h.t;
        th.u = h.bu;
        th.v = h.bv;
        th.prim = h.prim;
        th.code = h.code;
        hit_uv(S, o, du, th, &u, &v);
    }
    return texture_albedo_uv(m, h.point, u, v);
}

// sky_basis / sampling_basis: least-aligned world axis, Gram-Schmidt
// (src/material.c:1062-1075, src/sampling.c:52-77; the caller normalises n).
template <typename R> MT_D void basis(V3<R> n, V3<R> *t, V3<R> *b)
{
    V3<R> axis;
    if (mfabs(n.x) <= mfabs(n.y) && mfabs(n.x) <= mfabs(n.z)) axis = v3(R(1), R(0), R(0));
    else if (mfabs(n.y) <= mfabs(n.z)) axis = v3(R(0), R(1), R(0));
    else axis = v3(R(0), R(0), R(1));
    *t = normalize(cross(axis, n));
    *b = cross(n, *t);
}

// sky_sun_disk_dir (src/material.c:1077-1107)
template <typename R> MT_D V3<R> sun_disk_dir(V3<R> sun_dir, R radius_deg, R r1, R r2)
{
    if (radius_deg <= R(0)) return sun_dir;
    V3<R> n = normalize(sun_dir);
    if (length_sq(n) == R(0)) return v3(R(0), R(1), R(0));
    if (r1 < R(0)) r1 = R(0); else if (r1 > R(1)) r1 = R(1);
    if (r2 < R(0)) r2 = R(0); else if (r2 > R(1)) r2 = R(1);
    R radius_rad = radius_deg * (Const<R>::pi / R(180));
    R offset = msqrt(r1) * radius_rad;
    R theta = R(2) * Const<R>::pi * r2;
    V3<R> t, b;
    basis(n, &t, &b);
    R st, ct;
    msincos(theta, &st, &ct);
    V3<R> radial = add(scale(t, ct), scale(b, st));
    V3<R> dir = add(n, scale(radial, mtan(offset)));
    return normalize(dir);
}

// light_sphere_sample_dir (src/material.c:1113-1146)
// omc_max: 1 - cos_alpha_max from cone_one_minus_cos (used by FP32)
template <typename R> MT_D V3<R> light_sphere_sample_dir(V3<R> w, R cos_alpha_max, R omc_max, R u1, R u2)
{
    const R rmax = sizeof(R) == 8 ? R(0.9999999999999999) : R(0.99999994f);
    w = normalize(w);
    if (length_sq(w) == R(0)) return v3(R(0), R(1), R(0));
    if (!(cos_alpha_max >= R(0))) cos_alpha_max = R(0);
    else if (cos_alpha_max > R(1)) cos_alpha_max = R(1);
    if (!(u1 > R(0))) u1 = R(0);
    else if (u1 > rmax) u1 = rmax;
    if (!(u2 > R(0))) u2 = R(0);
    else if (u2 > rmax) u2 = rmax;
    R cos_alpha, sin_alpha;
    if constexpr (sizeof(R) == 4) {
        // y = 1 - cos(alpha) within the cone: sin^2 = y (2 - y), no cancellation
        if (!(omc_max >= R(0))) omc_max = R(0);
        else if (omc_max > R(1)) omc_max = R(1);
        const R y = u1 * omc_max;
        cos_alpha = R(1) - y;
        sin_alpha = msqrt(y * (R(2) - y));
    } else {
        cos_alpha = R(1) - u1 * (R(1) - cos_alpha_max);
        sin_alpha = msqrt(R(1) - cos_alpha * cos_alpha);
    }
    R phi = R(2) * Const<R>::pi * u2;
    V3<R> t, b;
    basis(w, &t, &b);
    R sp, cp;
    msincos(phi, &sp, &cp);
    V3<R> dir = add(add(scale(t, sin_alpha * cp), scale(b, sin_alpha * sp)), scale(w, cos_alpha));
    return normalize(dir);
}

// ------------------------------------------------------------------
// Water (water_normal src/material.c:1171-1217, water_attenuate :1238-1267)
// ------------------------------------------------------------------
template <typename R> MT_D V3<R> water_normal(R x, R z, R time)
{
    // WATER_WAVES (src/material.c:1159-1166): ax, az, w = 2 pi / lambda, amp, speed, phase
    const R tp = R(2) * Const<R>::pi;
    const R ax[4] = {R(0.9584), R(0.7071), R(-0.4061), R(0.2005)};
    const R az[4] = {R(0.2855), R(-0.7071), R(0.9138), R(0.9797)};
    const R w[4] = {tp / R(24), tp / R(13), tp / R(7), tp / R(4)};
    const R amp[4] = {R(0.18), R(0.1), R(0.05), R(0.025)};
    const R speed[4] = {R(1.0), R(1.4), R(2.0), R(2.6)};
    const R phase[4] = {R(0.0), R(1.7), R(3.1), R(0.6)};
    R dhdx = R(0), dhdz = R(0);
    for (int i = 0; i < 4; ++i) {
        R u = (ax[i] * x + az[i] * z) * w[i] + phase[i] + time * speed[i] * w[i];
        R c = mcos(u) * amp[i] * w[i];
        dhdx += c * ax[i];
        dhdz += c * az[i];
    }
    const R freq = R(0.35), namp = R(0.06), e = R(0.02);
    const uint32_t seed = 1337u;
    R hL = noise_fbm2((x - e) * freq, z * freq, 4, seed);
    R hR = noise_fbm2((x + e) * freq, z * freq, 4, seed);
    R hD = noise_fbm2(x * freq, (z - e) * freq, 4, seed);
    R hU = noise_fbm2(x * freq, (z + e) * freq, 4, seed);
    dhdx += namp * (hR - hL) / (R(2) * e);
    dhdz += namp * (hU - hD) / (R(2) * e);
    V3<R> n = normalize(v3(-dhdx, R(1), -dhdz));
    if (length_sq(n) < R(1e-12)) return v3(R(0), R(1), R(0));
    if (n.y < R(0)) n = neg(n);
    return n;
}

template <typename R> MT_D R water_transmittance(R absorption, R depth)
{
    if (absorption == R(0)) return R(1);
    R t = mexp(-absorption * depth);
    if (!(t > R(0))) return R(0);
    if (t > R(1)) return R(1);
    return t;
}

template <typename R> MT_D V3<R> water_attenuate(const DevMaterial<R> &m, V3<R> inner, R depth)
{
    R d = depth > R(0) ? depth : R(0);
    V3<R> tr = v3(water_transmittance(m.absorption[0], d), water_transmittance(m.absorption[1], d),
                  water_transmittance(m.absorption[2], d));
    V3<R> out = v3(inner.x * tr.x + m.deep_color[0] * (R(1) - tr.x),
                   inner.y * tr.y + m.deep_color[1] * (R(1) - tr.y),
                   inner.z * tr.z + m.deep_color[2] * (R(1) - tr.z));
    if (!(out.x >= R(0))) out.x = R(0);
    if (!(out.y >= R(0))) out.y = R(0);
    if (!(out.z >= R(0))) out.z = R(0);
    return out;
}

// scene_water_height (src/scene.c:1109-1153)
template <typename R> MT_D R water_height(const DevScene<R> &S, R x, R z)
{
    if (!S.ocean.enabled) return S.water_level;
    const DevOcean<R> &o = S.ocean;
    R y = o.center[1];
    R dir_x = o.direction[0], dir_z = o.direction[2];
    R dlen = msqrt(dir_x * dir_x + dir_z * dir_z);
    if (dlen > R(1e-12)) {
        dir_x /= dlen;
        dir_z /= dlen;
    } else {
        dir_x = R(1);
        dir_z = R(0);
    }
    R wl = o.wavelength <= R(0) ? R(12) : o.wavelength;
    R amp = o.amplitude;
    R chop_wl = o.chop_wavelength > R(0) ? o.chop_wavelength : wl * R(0.25);
    R chop_amp = o.chop > R(0) ? o.chop : amp * R(0.25);
    R lambda[4] = {wl, wl * R(0.52), chop_wl, chop_wl * R(0.40)};
    R A[4] = {amp, amp * R(0.38), chop_amp, chop_amp * R(0.32)};
    R angle[4] = {R(0.0), R(0.628), R(-0.488), R(1.134)};
    R phi[4] = {R(0.0), R(1.7) + R(o.seed % 100u) * R(0.03), R(3.1) + R((o.seed * 7u) % 100u) * R(0.03),
                R(0.8) + R((o.seed * 13u) % 100u) * R(0.03)};
    for (int h = 0; h < 4; ++h) {
        R ca = mcos(angle[h]);
        R sa = msin(angle[h]);
        R dx_h = ca * dir_x - sa * dir_z;
        R dz_h = sa * dir_x + ca * dir_z;
        R k_h = (R(2) * Const<R>::pi) / lambda[h];
        R theta = k_h * (dx_h * x + dz_h * z) + phi[h];
        y += A[h] * mcos(theta);
    }
    return y;
}

// ------------------------------------------------------------------
// Local shading
// ------------------------------------------------------------------
// material_shade_local: Blinn-Phong without 1/pi (src/material.c:157-188)
template <typename R>
MT_D V3<R> shade_local(const DevMaterial<R> &m, V3<R> N, V3<R> L, V3<R> V, V3<R> light)
{
    R ndl = dot(N, L);
    if (ndl <= R(0)) return v3(R(0), R(0), R(0));
    V3<R> diffuse = scale(mul(mat3(m.albedo), light), ndl);
    V3<R> h = add(L, V);
    V3<R> spec = v3(R(0), R(0), R(0));
    if (length_sq(h) > R(1e-12)) {
        V3<R> H = normalize(h);
        R ndh = dot(N, H);
        if (ndh > R(0)) {
            R spec_term = pow_nonneg(ndh, m.shininess);
            spec = scale(mul(mat3(m.specular), light), spec_term);
        }
    }
    return add(diffuse, spec);
}

// material_roughness_to_alpha (src/material.c:227-232)
template <typename R> MT_D R roughness_to_alpha(R roughness)
{
    R r = mat_clamp01(roughness);
    R a = r * r;
    return a < R(1e-4) ? R(1e-4) : a;
}

template <typename R> MT_D R d_ggx(R ndh, R a)
{
    R a2 = a * a;
    R d = ndh * ndh * (a2 - R(1)) + R(1);
    return a2 / (Const<R>::pi * d * d);
}

// GGX D of a half vector at angle theta from the normal, given cos(theta) =
// ndh and sin^2(theta). The denominator ndh^2 (a^2 - 1) + 1 equals
// a^2 ndh^2 + sin^2(theta). FP64 keeps the reference's form (its bits match
// the reference's); FP32 uses the second form, whose terms are all positive.
// Near the normal the first form subtracts two numbers within an ulp of 1:
// for roughness 0.02 (a^2 = 1.6e-7, about FP32's epsilon) it is off by up to
// a factor of two, so D is off by up to four, which biased FP32 images of
// near-mirror metals bright.
template <typename R> MT_D R d_ggx_cs(R ndh, R sin2, R a)
{
    if constexpr (sizeof(R) == 4) {
        const R a2 = a * a;
        const R d = a2 * ndh * ndh + sin2;
        return a2 / (Const<R>::pi * d * d);
    } else {
        return d_ggx(ndh, a);
    }
}

// sin^2 of the angle between unit vectors n and h, |n x h|^2 (Lagrange's
// identity): accurate where 1 - (n.h)^2 cancels.
template <typename R> MT_D R sin2_between(V3<R> n, V3<R> h) { return length_sq(cross(n, h)); }

// 1 - cos(alpha_max) of the cone a sphere of radius^2 / distance^2 = x
// subtends, given cos(alpha_max) = sqrt(1 - x). FP64: the reference's
// 1 - cos; FP32: x / (1 + cos), the same value without the cancellation that
// costs distant lights (x ~ 1e-4) three decimal digits of their solid angle.
template <typename R> MT_D R cone_one_minus_cos(R x, R cos_max)
{
    if constexpr (sizeof(R) == 4)
        return x / (R(1) + cos_max);
    else
        return R(1) - cos_max;
}

// g_smith_schlick (src/material.c:207-218, same as pt_g_smith_schlick :192-200
// up to the NaN behaviour of the clamp)
template <typename R> MT_D R g_smith_schlick(R ndl, R ndv, R roughness)
{
    R k = (roughness + R(1)) * (roughness + R(1)) / R(8);
    if (k < R(0)) k = R(0);
    else if (k > R(1)) k = R(1);
    R gl = ndl / (ndl * (R(1) - k) + k);
    R gv = ndv / (ndv * (R(1) - k) + k);
    return gl * gv;
}

// fresnel_schlick_rgb (src/material.c:142-151): clamps the cosine only
template <typename R> MT_D V3<R> fresnel_schlick_rgb(R cos_theta, V3<R> f0)
{
    R c = mat_clamp01(cos_theta);
    R mm = R(1) - c;
    R m2 = mm * mm;
    R k = m2 * m2 * mm;
    return v3(f0.x + (R(1) - f0.x) * k, f0.y + (R(1) - f0.y) * k, f0.z + (R(1) - f0.z) * k);
}

// material_shade_pbr: Cook-Torrance GGX + Smith-Schlick + Schlick F at NdotV,
// kD-weighted Lambert (src/material.c:234-290)
template <typename R>
MT_D V3<R> shade_pbr(const DevMaterial<R> &m, V3<R> N, V3<R> L, V3<R> V, V3<R> light)
{
    R ndl = dot(N, L);
    if (ndl <= R(0)) return v3(R(0), R(0), R(0));
    R ndv = dot(N, V);
    if (ndv <= R(0)) return v3(R(0), R(0), R(0));
    R metallic = mat_clamp01(m.metallic);
    R alpha = roughness_to_alpha(m.roughness);
    V3<R> h = add(L, V);
    R ndh = R(0), sin2 = R(1);
    if (length_sq(h) > R(1e-12)) {
        const V3<R> hn = normalize(h);
        ndh = dot(N, hn);
        if (ndh < R(0)) ndh = R(0);
        else sin2 = sin2_between(N, hn);
    }
    V3<R> albedo = mat3(m.albedo);
    V3<R> f0 = lerp(v3(R(0.04), R(0.04), R(0.04)), albedo, metallic);
    V3<R> F = fresnel_schlick_rgb(ndv, f0);
    R D = d_ggx_cs(ndh, sin2, alpha);
    R G = g_smith_schlick(ndl, ndv, mat_clamp01(m.roughness));
    R denom = R(4) * ndl * ndv;
    R spec_scale = (denom > R(0)) ? (D * G / denom) : R(0);
    V3<R> spec = scale(F, spec_scale);
    V3<R> kd = scale(sub(v3(R(1), R(1), R(1)), F), (R(1) - metallic));
    V3<R> f_diff = scale(mul(kd, albedo), R(1) / Const<R>::pi);
    V3<R> f = add(f_diff, spec);
    return scale(mul(light, f), ndl);
}

template <typename R>
MT_D V3<R> shade(const DevMaterial<R> &m, V3<R> N, V3<R> L, V3<R> V, V3<R> light)
{
    return m.pbr ? shade_pbr(m, N, L, V, light) : shade_local(m, N, L, V, light);
}

// fresnel_schlick (scalar, src/material.c:134-140)
template <typename R> MT_D R fresnel_schlick(R cos_theta, R f0)
{
    R c = mat_clamp01(cos_theta);
    R mm = R(1) - c;
    R m2 = mm * mm;
    return f0 + (R(1) - f0) * (m2 * m2 * mm);
}

// material_ambient (src/material.c:351-374)
template <typename R> MT_D V3<R> material_ambient(const DevMaterial<R> &m, V3<R> N, const DevSky<R> &sky)
{
    V3<R> groundish = scale(mat3(sky.horizon_color), R(0.45));
    V3<R> skyish = mat3(sky.zenith_color);
    R w = mat_clamp01(R(0.5) + R(0.5) * N.y);
    V3<R> hemi = lerp(groundish, skyish, w);
    return scale(mul(mat3(m.albedo), hemi), R(0.15));
}

// material_sample_glossy_dir (src/material.c:303-349)
template <typename R>
MT_D V3<R> sample_glossy_dir(const DevMaterial<R> &m, V3<R> N, V3<R> incident, R r1, R r2)
{
    const R rmax = sizeof(R) == 8 ? R(0.9999999999999999) : R(0.99999994f);
    V3<R> mirror = reflect(incident, N);
    if (m.roughness <= R(1e-6)) return mirror;
    R alpha = roughness_to_alpha(m.roughness);
    R a2 = alpha * alpha;
    if (!(r1 > R(0))) r1 = R(0);
    else if (r1 > rmax) r1 = rmax;
    if (!(r2 > R(0))) r2 = R(0);
    else if (r2 > rmax) r2 = rmax;
    R cos_theta, sin_theta;
    if constexpr (sizeof(R) == 4) {
        // cos^2 and sin^2 of the GGX angle as (1 - r1) / den and a2 r1 / den,
        // den = 1 - r1 + a2 r1 (1 - r1 is exact: r1 is a multiple of 2^-24):
        // no cancellation for small alpha (see d_ggx_cs)
        const R omr = R(1) - r1, den = omr + a2 * r1;
        cos_theta = msqrt(omr / den);
        sin_theta = msqrt(a2 * r1 / den);
    } else {
        cos_theta = msqrt((R(1) - r1) / (R(1) + (a2 - R(1)) * r1));
        sin_theta = msqrt(R(1) - cos_theta * cos_theta);
    }
    R phi = R(2) * Const<R>::pi * r2;
    V3<R> t, b;
    basis(N, &t, &b);
    R sp, cp;
    msincos(phi, &sp, &cp);
    V3<R> H = add(add(scale(t, sin_theta * cp), scale(b, sin_theta * sp)), scale(N, cos_theta));
    H = normalize(H);
    V3<R> Rr = reflect(incident, H);
    if (!(dot(Rr, N) > R(0))) return mirror;
    return normalize(Rr);
}

// ------------------------------------------------------------------
// Monte-Carlo sampling (src/sampling.c:40-281)
// ------------------------------------------------------------------
template <typename R> MT_D R clamp_uniform(R u)
{
    const R rmax = sizeof(R) == 8 ? R(0.9999999999999999) : R(0.99999994f);
    if (!(u > R(0))) return R(0);
    if (u > rmax) return rmax;
    return u;
}

// sampling_basis with its defensive normalisation (src/sampling.c:52-77)
template <typename R> MT_D void sampling_basis(V3<R> n, V3<R> *t, V3<R> *b)
{
    V3<R> nn = normalize(n);
    if (length_sq(nn) <= R(0)) nn = v3(R(0), R(1), R(0));
    basis(nn, t, b);
}

// sampling_cosine_hemisphere (src/sampling.c:83-107)
template <typename R> MT_D V3<R> cosine_hemisphere(V3<R> n, R u1, R u2)
{
    V3<R> nn = normalize(n);
    if (length_sq(nn) <= R(0)) nn = v3(R(0), R(1), R(0));
    R r1 = clamp_uniform(u1);
    R r2 = clamp_uniform(u2);
    R r = msqrt(r1);
    R phi = R(2) * Const<R>::pi * r2;
    R sp, cp;
    msincos(phi, &sp, &cp);
    R x = r * cp;
    R y = r * sp;
    R z = msqrt(mfmax(R(0), R(1) - r1));
    V3<R> t, b;
    sampling_basis(nn, &t, &b);
    V3<R> d = add(add(scale(t, x), scale(b, y)), scale(nn, z));
    return normalize(d);
}

// sampling_fresnel_schlick_rgb: clamps cosine AND f0 (src/sampling.c:134-149)
template <typename R> MT_D R sampling_fresnel_schlick(R cos_theta, R f0)
{
    R c = mat_clamp01(cos_theta);
    R f = mat_clamp01(f0);
    R mm = R(1) - c;
    R m2 = mm * mm;
    R k = m2 * m2 * mm;
    return f + (R(1) - f) * k;
}
template <typename R> MT_D V3<R> sampling_fresnel_schlick_rgb(R cos_theta, V3<R> f0)
{
    return v3(sampling_fresnel_schlick(cos_theta, f0.x), sampling_fresnel_schlick(cos_theta, f0.y),
              sampling_fresnel_schlick(cos_theta, f0.z));
}

// sampling_fresnel_dielectric: exact unpolarised Fresnel (src/sampling.c:162-181)
template <typename R> MT_D R fresnel_dielectric(R cos_i, R eta)
{
    R c = mat_clamp01(cos_i);
    R e = eta > R(0) ? eta : R(0);
    R sin2_t = e * e * (R(1) - c * c);
    if (sin2_t >= R(1)) return R(1);
    R cos_t = msqrt(R(1) - sin2_t);
    R rs = (e * c - cos_t) / (e * c + cos_t);
    R rp = (e * cos_t - c) / (e * cos_t + c);
    R f = R(0.5) * (rs * rs + rp * rp);
    return mat_clamp01(f);
}

// sampling_refract (src/sampling.c:183-211)
template <typename R> MT_D bool sampling_refract(V3<R> incident, V3<R> n, R eta, V3<R> *out)
{
    V3<R> i = normalize(incident);
    V3<R> nn = normalize(n);
    if (length_sq(i) <= R(0) || length_sq(nn) <= R(0)) return false;
    R e = eta > R(0) ? eta : R(0);
    R cos_i = -dot(i, nn);
    R sin2_t = e * e * (R(1) - cos_i * cos_i);
    if (sin2_t >= R(1)) return false;
    R cos_t = msqrt(R(1) - sin2_t);
    R k = e * cos_i - cos_t;
    V3<R> t = v3(e * i.x + k * nn.x, e * i.y + k * nn.y, e * i.z + k * nn.z);
    *out = normalize(t);
    return true;
}

// vec3_refract (src/vec3.c:54-66), used by the Whitted renderer
template <typename R> MT_D V3<R> vec3_refract(V3<R> i, V3<R> n, R eta)
{
    R cos_i = -dot(i, n);
    R sin2_t = eta * eta * (R(1) - cos_i * cos_i);
    if (sin2_t > R(1)) return v3(R(0), R(0), R(0));
    R cos_t = msqrt(R(1) - sin2_t);
    R k = eta * cos_i - cos_t;
    return v3(eta * i.x + k * n.x, eta * i.y + k * n.y, eta * i.z + k * n.z);
}

// sampling_specular_probability (src/sampling.c:217-231)
template <typename R> MT_D R specular_probability(R metallic, R roughness, R f0_scalar)
{
    R m = mat_clamp01(metallic);
    R r = mat_clamp01(roughness);
    R f0 = mat_clamp01(f0_scalar);
    R p = f0 + (R(1) - f0) * m;
    p *= R(1) - R(0.5) * r * (R(1) - m);
    return pt_clamp(p, R(1e-3), R(1));
}

// sampling_ggx_half_vector (src/sampling.c:242-268)
template <typename R> MT_D V3<R> ggx_half_vector(V3<R> n, R alpha, R u1, R u2)
{
    V3<R> nn = normalize(n);
    if (length_sq(nn) <= R(0)) nn = v3(R(0), R(1), R(0));
    R a = alpha > R(1e-4) ? alpha : R(1e-4);
    R a2 = a * a;
    R r1 = clamp_uniform(u1);
    R r2 = clamp_uniform(u2);
    R cos_theta, sin_theta;
    if constexpr (sizeof(R) == 4) {
        // the same angle from (1 - r1) / den and a2 r1 / den (see
        // sample_glossy_dir): no cancellation for small alpha
        const R omr = R(1) - r1, den = omr + a2 * r1;
        cos_theta = msqrt(omr / den);
        sin_theta = msqrt(a2 * r1 / den);
    } else {
        cos_theta = msqrt((R(1) - r1) / (R(1) + (a2 - R(1)) * r1));
        sin_theta = msqrt(mfmax(R(0), R(1) - cos_theta * cos_theta));
    }
    R phi = R(2) * Const<R>::pi * r2;
    V3<R> t, b;
    sampling_basis(nn, &t, &b);
    R sp, cp;
    msincos(phi, &sp, &cp);
    V3<R> h = add(add(scale(t, sin_theta * cp), scale(b, sin_theta * sp)), scale(nn, cos_theta));
    return normalize(h);
}

// sampling_ggx_pdf (src/sampling.c:270-281)
// (sin2: sin^2 of the angle between n and h, for the FP32 form of D)
template <typename R> MT_D R ggx_pdf(R n_dot_h, R sin2, R h_dot_v, R alpha)
{
    if (!(h_dot_v > R(0)) || !(n_dot_h > R(0))) return R(0);
    R a = alpha > R(1e-4) ? alpha : R(1e-4);
    R ndh = n_dot_h > R(1) ? R(1) : n_dot_h;
    if (n_dot_h > R(1)) sin2 = R(0);
    R D = d_ggx_cs(ndh, sin2, a);
    return D * ndh / (R(4) * h_dot_v);
}

}  // namespace mt
