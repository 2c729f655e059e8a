// mt_adjoint.cuh - path-replay adjoint of the path tracer.
//
// Parameters: per material m, albedo rgb (8m + 0..2), roughness (8m + 3),
// metallic (8m + 4), emissive rgb (8m + 5..7); then the sun radiance rgb
// (8M + 0..2); then per material the Beer-Lambert absorption rgb
// (8M + 3 + 3m + 0..2), which acts through media (pt_apply_medium) and on
// shadow segments through water / beer_lambert surfaces. Geometry and
// visibility derivatives are out of scope.
//
// Estimator. The path tracer's per-sample value is L = sum_b beta_b E_b,
// where E_b is what vertex b adds (emission, NEE, sky) and
// beta_{b+1} = beta_b * w_b / q_b (w_b the BSDF sample weight, q_b the
// roulette probability). With detached sampling -- directions, lobe
// choices and their probabilities, and roulette probabilities held fixed,
// which keeps the estimator of the gradient of the expectation unbiased --
//   dL/dtheta = sum_b beta_b dE_b/dtheta
//             + sum_k (dw_k/dtheta / w_k) * R_k,   R_k = sum_{b>k} beta_b E_b.
// Path replay (Vicini, Speierer and Jakob, "Path Replay Backpropagation",
// SIGGRAPH 2021): the path is traced once to get L, then replayed from the
// same random stream; at vertex k the remaining radiance is
// R_k = L - (radiance accumulated up to and including vertex k), so no
// vertex is stored.
#pragma once

#include "mt_integrate.cuh"

namespace mt {

static constexpr int kParamsPerMaterial = 8;
static constexpr int kAbsorbPerMaterial = 3;
static constexpr int kAdjMaxMaterials = 256;
static constexpr int kAdjMaxParams = (kParamsPerMaterial + kAbsorbPerMaterial) * kAdjMaxMaterials + 3;
// per NEE connection of a replayed vertex: transmittance rgb, then the
// absorbing materials passed (as R) and their distance sums (AbsorbPath)
static constexpr int kAttStride = 8;

struct AdjCtx {
    float *g;      // gradient accumulator (shared memory)
    int sun;       // index of the sun radiance's red channel
    int absorb;    // index of material 0's absorption red channel
};

MT_D AdjCtx make_adj_ctx(float *g, int material_count)
{
    return AdjCtx{g, kParamsPerMaterial * material_count, kParamsPerMaterial * material_count + 3};
}

MT_D void gadd(const AdjCtx &c, int i, float v)
{
    if (v != 0.0f && isfinite(v)) atomicAdd(&c.g[i], v);
}

template <typename R> MT_D R comp3(V3<R> v, int k) { return k == 0 ? v.x : (k == 1 ? v.y : v.z); }

// d d_ggx_cs(ndh, sin2, a) / d a (the denominator in the precision's form,
// see d_ggx_cs)
template <typename R> MT_D R d_ggx_dalpha(R ndh, R sin2, R a)
{
    R a2 = a * a;
    R d = sizeof(R) == 4 ? a2 * ndh * ndh + sin2 : ndh * ndh * (a2 - R(1)) + R(1);
    R dD_da2 = (d - R(2) * a2 * ndh * ndh) / (Const<R>::pi * d * d * d);
    return dD_da2 * R(2) * a;
}

// d material_roughness_to_alpha(roughness) / d roughness (alpha = max(r^2, 1e-4), r = clamp01)
template <typename R> MT_D R dalpha_drough(R rough)
{
    if (!(rough > R(0)) || !(rough < R(1))) return R(0);
    return rough * rough < R(1e-4) ? R(0) : R(2) * rough;
}

// d g_smith_schlick(ndl, ndv, clamp01(roughness)) / d roughness
template <typename R> MT_D R dG_drough(R ndl, R ndv, R rough)
{
    if (!(rough > R(0)) || !(rough < R(1))) return R(0);
    R k = (rough + R(1)) * (rough + R(1)) / R(8);
    if (!(k > R(0)) || !(k < R(1))) return R(0);
    R dk = (rough + R(1)) / R(4);
    R ql = ndl * (R(1) - k) + k, qv = ndv * (R(1) - k) + k;
    R gl = ndl / ql, gv = ndv / qv;
    R dgl = -ndl * (R(1) - ndl) / (ql * ql), dgv = -ndv * (R(1) - ndv) / (qv * qv);
    return (dgl * gv + gl * dgv) * dk;
}

// The albedo rgb, roughness and metallic terms (offsets 0..4 within the
// material's block) of one surface vertex, summed in registers over its NEE
// connections and its BSDF weight and added to the block's accumulator once:
// five shared-memory atomics per vertex instead of five per connection.
// A non-finite term is dropped on its own, as gadd drops it.
template <typename R> struct VertexSink {
    R g[5] = {R(0), R(0), R(0), R(0), R(0)};
    MT_D void add(int k, R v)
    {
        if (isfinite(v)) g[k] += v;
    }
    MT_D void flush(const AdjCtx &c, int mi, bool dmet) const
    {
        const int base = kParamsPerMaterial * mi;
        for (int k = 0; k < 4; ++k) gadd(c, base + k, (float)g[k]);
        if (dmet) gadd(c, base + 4, (float)g[4]);
    }
};

// d metallic is taken only strictly inside (0, 1), where the clamp passes it
template <typename R> MT_D bool metallic_differentiable(const DevMaterial<R> &m)
{
    return m.metallic > R(0) && m.metallic < R(1);
}

// Accumulate coeff . d shade(m, N, L, V, light) / d(material params) into
// the vertex sink, and return shade(m, N, L, V, 1): the BSDF value both
// terms share, from the same intermediates.
// shade_local (src/material.c:157-188): only the albedo enters.
// shade_pbr (src/material.c:234-290): albedo, metallic, roughness.
// PBR: every material of the scene is a PBR surface (the legacy branch
// compiles out).
template <typename R, bool PBR>
MT_D V3<R> shade_grad(const DevMaterial<R> &m, V3<R> N, V3<R> L, V3<R> V, V3<R> light, V3<R> coeff,
                      VertexSink<R> &sink)
{
    const V3<R> zero = v3(R(0), R(0), R(0));
    R ndl = dot(N, L);
    if (ndl <= R(0)) return zero;
    if (!PBR && !m.pbr) {
        for (int ch = 0; ch < 3; ++ch) sink.add(ch, comp3(coeff, ch) * comp3(light, ch) * ndl);
        return shade_local(m, N, L, V, v3(R(1), R(1), R(1)));
    }
    R ndv = dot(N, V);
    if (ndv <= R(0)) return zero;
    R met = mat_clamp01(m.metallic);
    R alpha = roughness_to_alpha(m.roughness);
    V3<R> h = add(L, V);
    R ndh = R(0), sin2 = R(1);
    if (length_sq(h) > R(1e-12)) {
        const V3<R> hn = normalize(h);
        ndh = dot(N, hn);
        if (ndh < R(0)) ndh = R(0);
        else sin2 = sin2_between(N, hn);
    }
    R cv = mat_clamp01(ndv);
    R mm = R(1) - cv;
    R m2 = mm * mm;
    R k5 = m2 * m2 * mm;
    R D = d_ggx_cs(ndh, sin2, alpha);
    R G = g_smith_schlick(ndl, ndv, mat_clamp01(m.roughness));
    R denom = R(4) * ndl * ndv;
    R specs = denom > R(0) ? D * G / denom : R(0);
    R dspecs = denom > R(0) ? (d_ggx_dalpha(ndh, sin2, alpha) * dalpha_drough(m.roughness) * G +
                               D * dG_drough(ndl, ndv, m.roughness)) / denom
                            : R(0);
    R d_rough = R(0), d_met = R(0);
    R s1[3];
    for (int ch = 0; ch < 3; ++ch) {
        R A = comp3(coeff, ch) * comp3(light, ch) * ndl;
        R alb = m.albedo[ch];
        R f0 = R(0.04) + (alb - R(0.04)) * met;
        R F = f0 + (R(1) - f0) * k5;
        R kd = (R(1) - F) * (R(1) - met);
        // shade_pbr's value for unit light: (kd albedo / pi + F D G / (4 ndl ndv)) ndl
        s1[ch] = ((kd * alb) * (R(1) / Const<R>::pi) + F * specs) * ndl;
        R dF_dalb = (R(1) - k5) * met;
        sink.add(ch, A * ((-dF_dalb * (R(1) - met) * alb + kd) / Const<R>::pi + dF_dalb * specs));
        R dF_dmet = (R(1) - k5) * (alb - R(0.04));
        R dkd_dmet = -dF_dmet * (R(1) - met) - (R(1) - F);
        d_met += A * (dkd_dmet * alb / Const<R>::pi + dF_dmet * specs);
        d_rough += A * F * dspecs;
    }
    sink.add(3, d_rough);
    sink.add(4, d_met);
    return v3(s1[0], s1[1], s1[2]);
}

// d sky_sample(dir) / d sun_color (diagonal): the sun glow and the lit clouds
// are affine in sun_color (src/material.c:480-600).
template <typename R> MT_D V3<R> sky_dsun(V3<R> dir, const DevSky<R> &sky)
{
    R cos_sun = dot(dir, mat3(sky.sun_dir));
    R glow = R(0);
    if (cos_sun > R(0)) glow = pow_nonneg(cos_sun, sky.sun_glow_exponent) * sky.sun_glow_strength;
    V3<R> d = v3(glow, glow, glow);
    if (dir.y > R(0.03)) {
        R tt = sky.cloud_height / dir.y;
        R px = dir.x * tt, pz = dir.z * tt;
        int octaves = sky.cloud_octaves < 1 ? 1 : sky.cloud_octaves;
        R raw = noise_fbm2(px * sky.cloud_scale, pz * sky.cloud_scale, octaves, sky.seed);
        R density = mat_clamp01(R(0.5) * (raw + R(1)));
        R alpha = smoothstep(sky.cloud_coverage - sky.cloud_softness, sky.cloud_coverage + sky.cloud_softness, density);
        alpha = pow_nonneg(alpha, sky.cloud_sharpness);
        alpha *= smoothstep(R(0), R(0.15), dir.y);
        if (alpha > R(0)) {
            R shadow = R(0.6) + R(0.4) * alpha;
            R lit = cos_sun > R(0) ? cos_sun : R(0);
            V3<R> cloud = scale(v3(R(0.95), R(0.95), R(0.98)), shadow);
            d = add(scale(d, R(1) - alpha), scale(cloud, alpha * R(0.35) * lit));
        }
    }
    return d;
}

// The sky seen along `dir` with weight `coeff` (adj * throughput): its sun
// radiance term.
template <typename R> MT_D void sky_sun_grad(const AdjCtx &ctx, V3<R> dir, const DevSky<R> &sky, V3<R> coeff)
{
    V3<R> ds = sky_dsun(dir, sky);
    for (int ch = 0; ch < 3; ++ch) gadd(ctx, ctx.sun + ch, (float)(comp3(coeff, ch) * comp3(ds, ch)));
}

// pt_sample_pbr / pt_sample_legacy plus what the weight derivative needs.
template <typename R> struct LobeInfo {
    int kind;       // 0 none, 1 pbr specular, 2 pbr diffuse, 3 legacy diffuse, 4 delta lobe
    V3<R> H;        // sampled half vector (pbr specular)
    R pdf, p;       // lobe pdf and selection probability (held fixed)
    R lobe;         // legacy diffuse r_dif / p_dif
};

template <typename R, bool PBR>
MT_D bool sample_with_info(const DevMaterial<R> &m, V3<R> N, V3<R> d, V3<R> V, int front_face, R u1, R u2, R u_lobe,
                           R u_glass, V3<R> *wi, V3<R> *w, int *refracted, int *specular, LobeInfo<R> *info)
{
    info->kind = 0;
    if (PBR || m.pbr) {
        *refracted = 0;
        bool ok = pt_sample_pbr(m, N, d, V, u1, u2, u_lobe, wi, w, specular);
        if (ok) {
            R metallic = pt_clamp01(m.metallic);
            R roughness = pt_clamp01(m.roughness);
            V3<R> f0 = lerp(v3(R(0.04), R(0.04), R(0.04)), mat3(m.albedo), metallic);
            R p_spec = specular_probability(metallic, roughness, pt_luminance(f0));
            if (*specular) {
                // the same half vector pt_sample_pbr drew
                info->H = ggx_half_vector(N, roughness_to_alpha(roughness), u1, u2);
                info->pdf = ggx_pdf(dot(N, info->H), sin2_between(N, info->H), dot(V, info->H),
                                    roughness_to_alpha(roughness));
                info->p = p_spec;
                info->kind = 1;
            } else {
                info->p = p_spec;
                info->kind = 2;
            }
        }
        return ok;
    }
    bool ok = pt_sample_legacy(m, N, d, V, front_face, u1, u2, u_lobe, u_glass, wi, w, refracted, specular);
    if (ok) {
        if (*specular) {
            info->kind = 4;
        } else {
            R r_mir = pt_clamp01(m.reflectivity), r_die = pt_clamp01(m.transparency);
            R r_dif = R(1) - r_mir - r_die;
            if (r_dif < R(0)) r_dif = R(0);
            R p_dif = R(1) - r_mir - r_die;
            if (p_dif < R(0)) p_dif = R(0);
            info->lobe = p_dif > R(0) ? r_dif / p_dif : R(0);
            info->kind = 3;
        }
    }
    return ok;
}

// Accumulate sum_c coeff_c d w_c / d theta for the sampled lobe (detached)
// into the vertex sink.
template <typename R>
MT_D void weight_grad(const DevMaterial<R> &m, const LobeInfo<R> &info, V3<R> N, V3<R> V, V3<R> wi, V3<R> coeff,
                      VertexSink<R> &sink)
{
    if (info.kind == 3) {
        for (int ch = 0; ch < 3; ++ch) sink.add(ch, comp3(coeff, ch) * info.lobe);
        return;
    }
    if (info.kind != 1 && info.kind != 2) return;
    R met = pt_clamp01(m.metallic);
    R ndv = dot(N, V);
    if (info.kind == 1) {
        V3<R> H = info.H;
        R ndl = dot(N, wi), ndh = dot(N, H), vdh = dot(V, H);
        R roughness = pt_clamp01(m.roughness);
        R alpha = roughness_to_alpha(roughness);
        R cv = mat_clamp01(vdh);
        R mm = R(1) - cv;
        R m2 = mm * mm;
        R k5 = m2 * m2 * mm;
        const R sin2 = sin2_between(N, H);
        R D = d_ggx_cs(ndh, sin2, alpha);
        R G = g_smith_schlick(ndl, ndv, roughness);
        R S = D * G / (R(4) * ndv * info.pdf * info.p);
        R dS = (d_ggx_dalpha(ndh, sin2, alpha) * dalpha_drough(m.roughness) * G +
                D * dG_drough(ndl, ndv, m.roughness)) /
               (R(4) * ndv * info.pdf * info.p);
        R d_rough = R(0), d_met = R(0);
        for (int ch = 0; ch < 3; ++ch) {
            R alb = m.albedo[ch];
            R f0 = R(0.04) + (alb - R(0.04)) * met;
            bool f_in = f0 > R(0) && f0 < R(1);
            R fc = mat_clamp01(f0);
            R F = fc + (R(1) - fc) * k5;
            R dF_df0 = f_in ? (R(1) - k5) : R(0);
            sink.add(ch, comp3(coeff, ch) * dF_df0 * met * S);
            d_met += comp3(coeff, ch) * dF_df0 * (alb - R(0.04)) * S;
            d_rough += comp3(coeff, ch) * F * dS;
        }
        sink.add(3, d_rough);
        sink.add(4, d_met);
    } else {
        R cv = mat_clamp01(ndv);
        R mm = R(1) - cv;
        R m2 = mm * mm;
        R k5 = m2 * m2 * mm;
        R inv = R(1) / (R(1) - info.p);
        R d_met = R(0);
        for (int ch = 0; ch < 3; ++ch) {
            R alb = m.albedo[ch];
            R f0 = R(0.04) + (alb - R(0.04)) * met;
            bool f_in = f0 > R(0) && f0 < R(1);
            R fc = mat_clamp01(f0);
            R F = fc + (R(1) - fc) * k5;
            R dF_df0 = f_in ? (R(1) - k5) : R(0);
            R kd = (R(1) - F) * (R(1) - met);
            sink.add(ch, comp3(coeff, ch) * (-dF_df0 * met * (R(1) - met) * alb + kd) * inv);
            d_met += comp3(coeff, ch) * (-dF_df0 * (alb - R(0.04)) * (R(1) - met) - (R(1) - F)) * alb * inv;
        }
        sink.add(4, d_met);
    }
}

template <typename R> MT_D V3<R> safe_div(V3<R> a, V3<R> b)
{
    return v3(b.x != R(0) ? a.x / b.x : R(0), b.y != R(0) ? a.y / b.y : R(0), b.z != R(0) ? a.z / b.z : R(0));
}

// Gradient of one medium segment (pt_apply_medium, src/pathtrace.c:220-233)
// w.r.t. the medium's absorption: the segment adds beta * deep * (1 - T) and
// scales the throughput by T = exp(-a d) (water_transmittance); `beta` is the
// throughput entering the segment and `after` = L - radiance once the
// segment's own term is in, i.e. what the scaled throughput carries.
template <typename R>
MT_D void medium_grad(const AdjCtx &ctx, const DevMaterial<R> &m, int mi, R dist, V3<R> beta, V3<R> after, V3<R> adj)
{
    const R d = dist > R(0) ? dist : R(0);
    for (int ch = 0; ch < 3; ++ch) {
        const R a = m.absorption[ch];
        const R T = water_transmittance(a, d);
        // exp(-a d) clamped to [0, 1]: derivative -d T inside, 0 where clamped
        const R dT = (a >= R(0) && T > R(0)) ? -d * T : R(0);
        if (dT == R(0)) continue;
        const R g = comp3(adj, ch) * (-comp3(beta, ch) * m.deep_color[ch] * dT) +
                    comp3(adj, ch) * comp3(after, ch) * (dT / T);
        gadd(ctx, ctx.absorb + kAbsorbPerMaterial * mi + ch, (float)g);
    }
}

// Absorption part of one NEE connection: contribution c (adj-weighted, per
// channel) times -(distance through each absorbing material).
template <typename R> MT_D void nee_absorb_grad(const AdjCtx &ctx, const R *slot, V3<R> c)
{
    for (int k = 0; k < 2; ++k) {
        const int am = (int)slot[5 + k];
        const R dist = slot[3 + k];
        if (am < 0 || dist == R(0)) continue;
        for (int ch = 0; ch < 3; ++ch)
            gadd(ctx, ctx.absorb + kAbsorbPerMaterial * am + ch, (float)(-dist * comp3(c, ch)));
    }
}

// Fill one NEE connection record from a shadow walk's result.
template <typename R> MT_D void set_att(R *slot, V3<R> atten, const AbsorbPath<R> &ab)
{
    slot[0] = atten.x;
    slot[1] = atten.y;
    slot[2] = atten.z;
    slot[3] = ab.dist[0];
    slot[4] = ab.dist[1];
    slot[5] = R(ab.mat[0]);
    slot[6] = R(ab.mat[1]);
    slot[7] = R(0);
}

// A surface vertex of a replayed path, held until its NEE visibility and the
// radiance the path gathers after it are known. Everything else the
// vertex's gradient needs is re-drawn from the path's random stream.
template <typename R> struct AdjVertex {
    R p[3], n[3], v[3];
    R beta[3];     // throughput arriving at the vertex (the NEE weight)
    int mat;       // material index; -1: no vertex pending
    int b;         // bounce index
    int flags;     // kVertFront | kVertSun | the connections made (vert_conn_bit)
    int pad;
};
static constexpr int kVertFront = 1;  // front-face hit (legacy glass sampling)
static constexpr int kVertSun = 2;    // the vertex draws a sun NEE sample
// Bit of AdjVertex::flags saying that NEE connection `li` (a light, or
// kMaxLights: the sun) was queued, so that its transmittance record holds
// this vertex's result. Records of connections not made are never read,
// which spares clearing them between vertices.
MT_HD constexpr int vert_conn_bit(int li) { return 1 << (2 + li); }
static constexpr int kVertConnAll = ((1 << kNeeSlots) - 1) << 2;

// Gradient terms of one vertex: NEE to every sphere light and to the sun,
// given each made connection's record att[kAttStride * slot] (transmittance
// zero where it was occluded or dark: such a connection adds nothing), and
// the BSDF weight term against `remaining` = L - radiance through this
// vertex. The vertex material's albedo / roughness / metallic terms are
// summed in a VertexSink and added once.
// Light sampling follows pt_nee_emissive / pt_nee_sun (src/pathtrace.c:534-606)
// and the BSDF sample pt_sample_* (src/pathtrace.c:961-1000), from the same
// random channels as the primal pass.
// PBR: every material is a PBR surface without media or absorption
// (DevScene::pbr_only); the legacy and absorption terms compile out.
// WARP: the caller runs all 32 lanes of the warp through this call together
// (`active` false where a lane has no vertex). A connection's emitter terms
// then go to the same three parameters for every lane of the warp (one light
// per iteration), so they are summed across the warp with shuffles and added
// by one lane: the vertex kernels were bound by these shared-memory atomics.
// Without WARP (the one-thread-per-pixel replay, whose lanes diverge) each
// lane adds its own.
template <typename R, bool PBR = false, bool WARP = false>
MT_D void vertex_adjoint(const DevScene<R> &S, const AdjVertex<R> &vx, const R *att, uint32_t seed_key,
                         V3<R> remaining, V3<R> adj, const AdjCtx &ctx, bool active = true)
{
    const int mi = active ? vx.mat : 0;
    const DevMaterial<R> &mm = S.materials[mi];
    const V3<R> P = v3(vx.p[0], vx.p[1], vx.p[2]);
    const V3<R> N = v3(vx.n[0], vx.n[1], vx.n[2]);
    const V3<R> V = v3(vx.v[0], vx.v[1], vx.v[2]);
    const V3<R> nee_w = mul(adj, v3(vx.beta[0], vx.beta[1], vx.beta[2]));
    const int b = vx.b;
    VertexSink<R> sink;
    // the lights in order, then the sun (slot kMaxLights) as one more pass of
    // the same loop, so the gradient code is emitted once: the replay kernels
    // are bound by instruction fetch. Under WARP every lane takes every pass.
    const bool sun_wanted = active && (vx.flags & kVertSun);
    const int n_conn = S.light_count + ((WARP || sun_wanted) ? 1 : 0);
    for (int k = 0; k < n_conn; ++k) {
        const bool sun = k == S.light_count;
        const int li = sun ? kMaxLights : k;
        V3<R> e = v3(R(0), R(0), R(0));  // the emitter's radiance term of this lane
        int pidx;  // first parameter of the emitter's radiance: its material's emissive rgb, or the sun's
        if (!sun) {
            const int lmat = __ldg(S.prim_info + S.lights[li].prim).y;
            pidx = (lmat >= 0 && lmat < S.material_count) ? kParamsPerMaterial * lmat + 5 : -1;
        } else {
            pidx = ctx.sun;
        }
        const bool made = active && (!sun || sun_wanted) && (vx.flags & vert_conn_bit(li));
        const R *slot = att + kAttStride * li;
        const V3<R> a = made ? v3(slot[0], slot[1], slot[2]) : v3(R(0), R(0), R(0));
        if (a.x != R(0) || a.y != R(0) || a.z != R(0)) {
            V3<R> wi, emit;
            R Omega;
            if (!sun) {
                const DevLight<R> &lt = S.lights[li];
                V3<R> to_c = sub(mat3(lt.center), P);
                R dc2 = length_sq(to_c);
                R dc = msqrt(dc2);
                R cos_mx = msqrt(R(1) - (lt.radius * lt.radius) / dc2);
                const R omc = cone_one_minus_cos((lt.radius * lt.radius) / dc2, cos_mx);
                Omega = R(2) * R(3.14159265358979323846) * omc;
                V3<R> w = scale(to_c, R(1) / dc);
                R u1 = rand01<R>(seed_key ^ (uint32_t)li, (uint32_t)b, PT_CH_NEE_EMIT_A);
                R u2 = rand01<R>(seed_key ^ (uint32_t)li, (uint32_t)b, PT_CH_NEE_EMIT_B);
                wi = light_sphere_sample_dir(w, cos_mx, omc, u1, u2);
                emit = mat3(lt.emissive);
            } else {
                R r1 = rand01<R>(seed_key, (uint32_t)b, PT_CH_NEE_SUN_A);
                R r2 = rand01<R>(seed_key, (uint32_t)b, PT_CH_NEE_SUN_B);
                wi = sun_disk_dir(mat3(S.sky.sun_dir), S.sky.sun_radius, r1, r2);
                R rad = S.sky.sun_radius * R(3.14159265358979323846) / R(180);
                Omega = (S.sky.sun_radius > R(0)) ? R(2) * R(3.14159265358979323846) * (R(1) - mcos(rad)) : R(1);
                emit = mat3(S.sky.sun_color);
            }
            const V3<R> coeff = scale(nee_w, Omega);
            const V3<R> s1 = shade_grad<R, PBR>(mm, N, wi, V, mul(emit, a), coeff, sink);
            e = mul(mul(coeff, a), s1);
            if (!PBR) nee_absorb_grad(ctx, slot, mul(mul(coeff, s1), mul(emit, a)));
        }
        if constexpr (WARP) {
            // a non-finite term is dropped before the sum, as gadd drops it
            float ev[3] = {(float)e.x, (float)e.y, (float)e.z};
            bool any = false;
            for (int ch = 0; ch < 3; ++ch) {
                if (!isfinite(ev[ch])) ev[ch] = 0.0f;
                any |= ev[ch] != 0.0f;
            }
            if (__any_sync(0xffffffffu, any) && pidx >= 0) {
                for (int ch = 0; ch < 3; ++ch)
                    for (int o = 16; o > 0; o >>= 1) ev[ch] += __shfl_xor_sync(0xffffffffu, ev[ch], o);
                if ((threadIdx.x & 31) == 0)
                    for (int ch = 0; ch < 3; ++ch) gadd(ctx, pidx + ch, ev[ch]);
            }
        } else if (pidx >= 0) {
            for (int ch = 0; ch < 3; ++ch) gadd(ctx, pidx + ch, (float)comp3(e, ch));
        }
    }
    if (!active) return;
    uint32_t kb = hash3(seed_key ^ PT_KEY, (uint32_t)b, 0u);
    R u1 = rand01<R>(kb, (uint32_t)b, PT_CH_BSDF_A);
    R u2 = rand01<R>(kb, (uint32_t)b, PT_CH_BSDF_B);
    R u_lobe = rand01<R>(kb, (uint32_t)b, PT_CH_LOBE);
    R u_glass = rand01<R>(kb, (uint32_t)b, PT_CH_GLASS);
    V3<R> wi, w;
    int refracted = 0, sampled_specular = 0;
    LobeInfo<R> info;
    if (sample_with_info<R, PBR>(mm, N, neg(V), V, (vx.flags & kVertFront) ? 1 : 0, u1, u2, u_lobe, u_glass, &wi,
                                 &w, &refracted, &sampled_specular, &info))
        weight_grad(mm, info, N, V, wi, mul(adj, safe_div(remaining, w)), sink);
    sink.flush(ctx, mi, metallic_differentiable(mm));
}

// Replay of pathtrace_radiance (src/pathtrace.c:800-1028) that accumulates
// adj . dL/dtheta, given the path's value L from the first pass.
template <typename R>
MT_D void pathtrace_adjoint(const DevScene<R> &S, Ray3<R> primary, int max_depth, uint32_t seed_key, V3<R> L,
                            V3<R> adj, const AdjCtx &ctx)
{
    V3<R> radiance = v3(R(0), R(0), R(0));
    if (max_depth < 0) max_depth = 0;
    Ray3<R> r;
    r.o = primary.o;
    r.d = normalize(primary.d);
    if (length_sq(r.d) <= R(0)) return;
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
                const V3<R> beta_in = throughput;
                pt_apply_medium(S.materials[medium], R(5.0), &throughput, &radiance);
                medium_grad(ctx, S.materials[medium], medium, R(5.0), beta_in, sub(L, radiance), adj);
                medium = -1;
            }
            sky_sun_grad(ctx, r.d, S.sky, mul(adj, throughput));
            return;
        }
        if (medium >= 0) {
            const V3<R> beta_in = throughput;
            pt_apply_medium(S.materials[medium], h.t, &throughput, &radiance);
            medium_grad(ctx, S.materials[medium], medium, h.t, beta_in, sub(L, radiance), adj);
        }
        if (h.material < 0 || h.material >= S.material_count) {
            sky_sun_grad(ctx, r.d, S.sky, mul(adj, throughput));
            return;
        }
        const int mi = h.material;
        const DevMaterial<R> &m = S.materials[mi];
        V3<R> P = h.point;
        V3<R> d = r.d;
        V3<R> N = h.normal;
        if (m.is_water) {
            if (mfabs(h.normal.y) > R(0.999) && mfabs(h.normal.x) < R(1e-4) && mfabs(h.normal.z) < R(1e-4))
                N = water_normal(P.x, P.z, R(0));
        }
        if (dot(N, d) > R(0)) N = neg(N);
        N = normalize(N);
        if (length_sq(N) <= R(0)) return;
        V3<R> V = neg(d);
        const DevMaterial<R> &mm = m;
        if (b == 0 || last_bounce_specular) {
            radiance = add(radiance, mul(throughput, mat3(mm.emissive)));
            for (int ch = 0; ch < 3; ++ch)
                gadd(ctx, kParamsPerMaterial * mi + 5 + ch, (float)(comp3(adj, ch) * comp3(throughput, ch)));
        }
        if (b == 0 && length_sq(mat3(mm.atmosphere_glow)) > R(1e-6))
            radiance = add(radiance, mul(throughput, atmosphere_term(mm, N, V, mat3(S.sky.sun_dir))));
        AdjVertex<R> vx;
        vx.p[0] = P.x; vx.p[1] = P.y; vx.p[2] = P.z;
        vx.n[0] = N.x; vx.n[1] = N.y; vx.n[2] = N.z;
        vx.v[0] = V.x; vx.v[1] = V.y; vx.v[2] = V.z;
        vx.beta[0] = throughput.x; vx.beta[1] = throughput.y; vx.beta[2] = throughput.z;
        vx.mat = mi;
        vx.b = b;
        // the local records below start cleared: every connection's record is valid
        vx.flags = (h.front_face ? kVertFront : 0) |
                   ((b == 0 || (b == 1 && medium >= 0 && last_bounce_specular)) ? kVertSun : 0) | kVertConnAll;
        vx.pad = 0;
        R att[kNeeSlots * kAttStride];
        for (int k = 0; k < kNeeSlots * kAttStride; ++k) att[k] = R(0);
        // ---- emissive-sphere NEE (pt_nee_emissive, src/pathtrace.c:576-606) ----
        if (S.light_count > 0) {
            V3<R> sum = v3(R(0), R(0), R(0));
            for (int li = 0; li < S.light_count; ++li) {
                const DevLight<R> &lt = S.lights[li];
                if (lt.prim == h.prim) continue;
                V3<R> to_c = sub(mat3(lt.center), P);
                R dc2 = length_sq(to_c);
                R dc = msqrt(dc2);
                if (dc <= lt.radius) continue;
                R cos_mx = msqrt(R(1) - (lt.radius * lt.radius) / dc2);
                const R omc = cone_one_minus_cos((lt.radius * lt.radius) / dc2, cos_mx);
                R Omega = R(2) * R(3.14159265358979323846) * omc;
                if (!(Omega > R(0))) continue;
                V3<R> w = scale(to_c, R(1) / dc);
                R u1 = rand01<R>(seed_key ^ (uint32_t)li, (uint32_t)b, PT_CH_NEE_EMIT_A);
                R u2 = rand01<R>(seed_key ^ (uint32_t)li, (uint32_t)b, PT_CH_NEE_EMIT_B);
                V3<R> wi = light_sphere_sample_dir(w, cos_mx, omc, u1, u2);
                if (!finite3(wi) || dot(N, wi) <= R(0)) continue;
                V3<R> so = add(P, scale(N, R(1e-3)));
                R lt_t;
                if (!light_sphere_t(S, lt.prim, so, wi, R(1e-3), R(1e30), &lt_t)) continue;
                V3<R> atten;
                AbsorbPath<R> ab;
                if (pt_occluded_segment_abs(S, so, wi, R(1e-3), lt_t - R(1e-3), &atten, &ab)) continue;
                V3<R> lit = shade(mm, N, wi, V, mul(mat3(lt.emissive), atten));
                sum = add(sum, mul(throughput, scale(lit, Omega)));
                set_att(att + kAttStride * li, atten, ab);
            }
            radiance = add(radiance, sum);
        }
        // ---- sun NEE (pt_nee_sun, src/pathtrace.c:534-556) ----
        if (b == 0 || (b == 1 && medium >= 0 && last_bounce_specular)) {
            V3<R> sun = mat3(S.sky.sun_dir);
            R r1 = rand01<R>(seed_key, (uint32_t)b, PT_CH_NEE_SUN_A);
            R r2 = rand01<R>(seed_key, (uint32_t)b, PT_CH_NEE_SUN_B);
            V3<R> Ls = sun_disk_dir(sun, S.sky.sun_radius, r1, r2);
            if (finite3(Ls) && dot(N, Ls) > R(0)) {
                V3<R> so = add(P, scale(N, R(1e-3)));
                V3<R> atten;
                AbsorbPath<R> ab;
                if (!pt_occluded_segment_abs(S, so, Ls, R(1e-3), R(1e30), &atten, &ab)) {
                    if (!(atten.x < R(1e-4) && atten.y < R(1e-4) && atten.z < R(1e-4))) {
                        R rad = S.sky.sun_radius * R(3.14159265358979323846) / R(180);
                        R Omega = (S.sky.sun_radius > R(0)) ? R(2) * R(3.14159265358979323846) * (R(1) - mcos(rad)) : R(1);
                        V3<R> lit = shade(mm, N, Ls, V, mul(mat3(S.sky.sun_color), atten));
                        radiance = add(radiance, mul(throughput, scale(lit, Omega)));
                        set_att(att + kAttStride * kMaxLights, atten, ab);
                    }
                }
            }
        }
        // ---- this vertex's gradient; L - radiance is what the path adds after it ----
        vertex_adjoint(S, vx, att, seed_key, sub(L, radiance), adj, ctx);
        // ---- BSDF sample (pt_sample_*), continue the path ----
        uint32_t kb = hash3(seed_key ^ PT_KEY, (uint32_t)b, 0u);
        R u1 = rand01<R>(kb, (uint32_t)b, PT_CH_BSDF_A);
        R u2 = rand01<R>(kb, (uint32_t)b, PT_CH_BSDF_B);
        R u_lobe = rand01<R>(kb, (uint32_t)b, PT_CH_LOBE);
        R u_glass = rand01<R>(kb, (uint32_t)b, PT_CH_GLASS);
        V3<R> wi, w;
        int refracted = 0, sampled_specular = 0;
        bool ok = mm.pbr ? pt_sample_pbr(mm, N, d, V, u1, u2, u_lobe, &wi, &w, &sampled_specular)
                         : pt_sample_legacy(mm, N, d, V, h.front_face, u1, u2, u_lobe, u_glass, &wi, &w, &refracted,
                                            &sampled_specular);
        if (!ok) return;
        last_bounce_specular = sampled_specular;
        throughput = mul(throughput, w);
        if (!finite3(throughput) || !(pt_max_component(throughput) > R(0))) return;
        if (refracted && (m.is_water || m.beer_lambert)) medium = h.front_face ? mi : -1;
        if (b >= 2) {
            R q = pt_clamp01(pt_max_component(throughput));
            if (!(q > R(0))) return;
            R u_rr = rand01<R>(kb, (uint32_t)b, PT_CH_RR);
            if (u_rr >= q) return;
            throughput = scale(throughput, R(1) / q);
        }
        V3<R> offset;
        if (refracted) offset = scale(wi, R(1e-4));
        else offset = scale(N, dot(wi, N) >= R(0) ? R(1e-4) : R(-1e-4));
        r.o = add(P, offset);
        r.d = wi;
    }
}

// One thread per pixel: both passes for each of the pixel's samples, then
// the block's gradient is flushed with one atomic per parameter.
template <typename R>
__global__ void __launch_bounds__(128) k_adjoint(const __grid_constant__ DevScene<R> S, const DevCamera<R> cam, int w, int h, int s0,
                                                 int s1, int depth, const float *adj_img, double adj_scale,
                                                 double *grad_out, int n_params)
{
    __shared__ float g[kAdjMaxParams];
    for (int i = threadIdx.x; i < n_params; i += blockDim.x) g[i] = 0.0f;
    __syncthreads();
    const AdjCtx ctx = make_adj_ctx(g, S.material_count);
    int pix = blockIdx.x * blockDim.x + threadIdx.x;
    if (pix < w * h) {
        V3<R> adj = v3<R>((R)(adj_img[3 * (size_t)pix] * adj_scale), (R)(adj_img[3 * (size_t)pix + 1] * adj_scale),
                          (R)(adj_img[3 * (size_t)pix + 2] * adj_scale));
        if (adj.x != R(0) || adj.y != R(0) || adj.z != R(0)) {
            int x = pix % w, y = pix / w;
            for (int s = s0; s < s1; ++s) {
                Ray3<R> ray = pt_primary(S, cam, w, h, x, y, s);
                uint32_t seed_key = hash3((uint32_t)x, (uint32_t)y, (uint32_t)s);
                V3<R> L = pathtrace_radiance<R, false>(S, ray, depth, seed_key);  // no extras: rejected on entry
                pathtrace_adjoint(S, ray, depth, seed_key, L, adj, ctx);
            }
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < n_params; i += blockDim.x)
        if (g[i] != 0.0f) atomicAdd(&grad_out[i], (double)g[i]);
}

}  // namespace mt
