// mt_wavefront.cuh - wavefront path tracer: per-bounce stage kernels over
// compacted queues (device side).
//
// A batch holds every pixel of the image times `batch_spp` samples. Bounce b
// of all live paths runs as three kernels:
//   extend  : nearest hit of every queued ray (pure traversal, few registers)
//   shade   : medium / emission / NEE set-up / BSDF sample / Russian roulette
//             (pathtrace_radiance's loop body, src/pathtrace.c:835-1018); NEE
//             connections go to the shadow queue, surviving paths to the next
//             ray queue. Both queues are compacted with one atomicAdd per
//             warp (ballot + popc), so terminated paths stop occupying lanes.
//   shadow  : pt_occluded_segment for every NEE connection; the visible
//             contribution lands in the path's NEE slot for that light.
// The NEE slots are summed into the path radiance in light order (then the
// sun) at the path's next shade or at the end of the batch, which is the
// order the reference adds them. Per-sample radiance is reduced into the
// pixel accumulator in sample order, as pt_render_pixel sums it.
#pragma once

#include "mt_adjoint.cuh"
#include "mt_launch.h"

namespace mt {

// 16-byte aligned records (and 8 for paths) so that a record moves in vector
// loads and stores, not one instruction per word.
template <typename R> struct alignas(16) WfRay {
    R o[3];
    R d[3];
    int slot;
    int pad;
};

template <typename R> struct WfHit {
    R t, u, v;
    int prim;
    int code;
};

template <typename R> struct alignas(8) WfPath {
    R throughput[3];
    R radiance[3];
    uint32_t seed_key;
    int medium;
    int last_specular;
    int pad;
};

template <typename R> struct alignas(16) WfShadow {
    R o[3];
    R d[3];
    R tmax;
    R contrib[3];
    int slot;
    int li;
};

// Parameters that change between calls live in device memory, so one
// captured CUDA graph serves every call with the same shape.
template <typename R> struct WfParams {
    DevCamera<R> cam;
    void *out;
    int w, h, wh;
    int s0;            // first sample of the window
    int spp_window;    // samples in the window
    int out_kind;
    // adjoint pass: dL/dimage (h, w, 3), its scale, the gradient (float64)
    const float *adj_img;
    double *grad;
    double adj_scale;
    int n_params;
};

// Buffers of the adjoint replay pass.
template <typename R> struct WfAdj {
    AdjVertex<R> *verts;  // the vertex each path holds until its NEE is resolved
    R *att;               // per path: kNeeSlots records of kAttStride (transmittance, absorbing distances)
    const R *L;           // per-sample radiance of the primal pass
    const WfParams<R> *P;
};

// Block-local gradient accumulator: zeroed at kernel start, flushed to the
// float64 gradient with one atomic per nonzero parameter at kernel end.
template <typename R> MT_D void adj_block_begin(float *g, const WfParams<R> *P)
{
    for (int i = threadIdx.x; i < P->n_params; i += blockDim.x) g[i] = 0.0f;
    __syncthreads();
}
template <typename R> MT_D void adj_block_end(const float *g, const WfParams<R> *P)
{
    __syncthreads();
    for (int i = threadIdx.x; i < P->n_params; i += blockDim.x)
        if (g[i] != 0.0f) atomicAdd(&P->grad[i], (double)g[i]);
}

template <typename R> MT_D V3<R> adj_of_path(const WfParams<R> *P, int slot)
{
    const int pix = slot % P->wh;
    const float *a = P->adj_img + 3 * (size_t)pix;
    const double sc = P->adj_scale;
    return v3<R>((R)(a[0] * sc), (R)(a[1] * sc), (R)(a[2] * sc));
}

// Stage kernels run with 64 or 128 (default) threads per block; the register
// allocation is tuned for the 128-thread bound.
static constexpr int kWfMaxBlock = 128;

// Blocks of 128 per SM the binary-tree walks are compiled for (the register
// budget, 65536 / (128 * blocks)): extend and the any-hit shadow walk.
#ifndef MT_EXTEND_MIN_BLOCKS
#define MT_EXTEND_MIN_BLOCKS 0
#endif
#ifndef MT_SHADOW_MIN_BLOCKS
#define MT_SHADOW_MIN_BLOCKS 7
#endif
// the chained pass-through walk (scenes with water or glass)
#ifndef MT_PASS_MIN_BLOCKS
#define MT_PASS_MIN_BLOCKS 7
#endif

struct WfCounters {
    int ray_count[2];
    int shadow_count;
    int shadow_fetch;  // next shadow ray handed out by the dynamic-fetch kernel
    int ray_fetch;     // next ray handed out by the dynamic-fetch extend kernel
    int sorted;        // this bounce's extend results were sorted by material
    int walk_count;    // shadow rays whose cached occluder missed (k_wf_shadow_cache)
    int pad;
    int link_count[6]; // pass-through chains continuing after link k (k_wf_shadow_link)
    int pad2[2];
};
// Ints from shadow_count that are zeroed before every shade stage.
static constexpr int kWfBounceCounters = 12;

// Warp-aggregated queue append: one atomicAdd per warp, lanes get
// consecutive slots in lane order.
MT_D int warp_append(int *counter, bool want)
{
    unsigned mask = __activemask();
    unsigned ballot = __ballot_sync(mask, want);
    if (!ballot) return -1;
    int lane = threadIdx.x & 31;
    int leader = __ffs(ballot) - 1;
    int base = 0;
    if (lane == leader) base = atomicAdd(counter, __popc(ballot));
    base = __shfl_sync(mask, base, leader);
    if (!want) return -1;
    return base + __popc(ballot & ((1u << lane) - 1u));
}

// Query log (mt_trace_log_enable): one record of 3 float4 per traversal
// query the stages answer, so a test can put the same query to the oracle:
//   (o.x, o.y, o.z, d.x) (d.y, d.z, t, result) (kind, bounce, light, 0)
// kind 0: extension ray, t = hit distance, result = prim index (-1: miss);
// kind 1: shadow connection over [1e-3, t = tmax], result = 1 if occluded.
// result / kind / bounce / light are int bit patterns. Records past
// trace_cap are counted but not kept.
template <typename R>
MT_D void trace_put(const DevScene<R> &S, V3<R> o, V3<R> d, R t, int result, int kind, int b, int li)
{
    const unsigned at = atomicAdd(S.trace_count, 1u);
    if (at >= (unsigned)S.trace_cap) return;
    float4 *r = S.trace_rec + 3 * (size_t)at;
    r[0] = make_float4((float)o.x, (float)o.y, (float)o.z, (float)d.x);
    r[1] = make_float4((float)d.y, (float)d.z, (float)t, __int_as_float(result));
    r[2] = make_float4(__int_as_float(kind), __int_as_float(b), __int_as_float(li), 0.0f);
}

// ------------------------------------------------------------------
// generate: primary rays of a batch (pt_render_pixel, src/pathtrace.c:1053-1086)
// ------------------------------------------------------------------
template <typename R>
__global__ void k_wf_generate(const __grid_constant__ DevScene<R> S, const WfParams<R> *P, int batch, int batch_spp, int n_paths,
                              WfPath<R> *paths, WfRay<R> *rays, WfCounters *C, R *nee, WfAdj<R> A, bool zero_nee)
{
    const WfParams<R> p = *P;
    const int n_round = (n_paths + gridDim.x * blockDim.x - 1) / (gridDim.x * blockDim.x) * (gridDim.x * blockDim.x);
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n_round; q += gridDim.x * blockDim.x) {
        if (q >= n_paths) {
            warp_append(&C->ray_count[0], false);
            continue;
        }
        int s = p.s0 + batch * batch_spp + q / p.wh;
        int pix = q % p.wh;
        int x = pix % p.w, y = pix / p.w;
        Ray3<R> ray = pt_primary(S, p.cam, p.w, p.h, x, y, s);
        WfPath<R> st;
        for (int k = 0; k < 3; ++k) {
            st.throughput[k] = R(1);
            st.radiance[k] = R(0);
        }
        st.seed_key = hash3((uint32_t)x, (uint32_t)y, (uint32_t)s);
        st.last_specular = 1;
        st.pad = 0;
        // medium if the eye is under water (src/pathtrace.c:821-826)
        st.medium = -1;
        if (S.water_material >= 0) {
            R w_h = water_height(S, ray.o.x, ray.o.z);
            if (ray.o.y < w_h && S.water_material < S.material_count) st.medium = S.water_material;
        }
        V3<R> d = normalize(ray.d);
        if (zero_nee)
            for (int k = 0; k < kNeeSlots * 3; ++k) nee[(size_t)q * kNeeSlots * 3 + k] = R(0);
        // adjoint replay: no vertex pending (a vertex reads only the records of
        // the connections it made, so the records need no clearing)
        if (A.verts) A.verts[q].mat = -1;
        paths[q] = st;
        bool live = length_sq(d) > R(0);  // degenerate primary ray: zero radiance
        int at = warp_append(&C->ray_count[0], live);
        if (live) {
            WfRay<R> r;
            r.o[0] = ray.o.x; r.o[1] = ray.o.y; r.o[2] = ray.o.z;
            r.d[0] = d.x; r.d[1] = d.y; r.d[2] = d.z;
            r.slot = q;
            r.pad = 0;
            rays[at] = r;
        }
    }
    if (S.counters && blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&S.counters->primary_rays, (unsigned long long)n_paths);
}

// ------------------------------------------------------------------
// extend: nearest hit (scene_intersect, src/scene.c:767 -> src/bvh.c:557)
// ------------------------------------------------------------------
template <typename R, int W>
__global__ void __launch_bounds__(kWfMaxBlock, W == 2 ? MT_EXTEND_MIN_BLOCKS : 0) k_wf_extend(const __grid_constant__ DevScene<R> S, const WfRay<R> *rays, const WfCounters *C,
                                                   int which, WfHit<R> *hits)
{
    const int n = C->ray_count[which];
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
        const WfRay<R> r = rays[q];
        V3<R> o = v3(r.o[0], r.o[1], r.o[2]);
        V3<R> d = unit_dir(v3(r.d[0], r.d[1], r.d[2]));
        RayPre<R> rp = ray_pre(o, d);
        Hit<R> h;
        WfHit<R> out;
        if (scene_nearest<R, W>(S, rp, R(1e-4), R(1e30), &h)) {
            out.t = h.t;
            out.u = h.u;
            out.v = h.v;
            out.prim = h.prim;
            out.code = h.code;
        } else {
            out.t = R(0);
            out.u = R(0);
            out.v = R(0);
            out.prim = -1;
            out.code = 0;
        }
        hits[q] = out;
        if (S.trace_rec) trace_put(S, o, d, out.t, out.prim, 0, 0, 0);
    }
    if (S.counters && blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&S.counters->extension_rays, (unsigned long long)n);
}

template <typename R> MT_D void gather_nee(const DevScene<R> &S, R *nee_slot, V3<R> *radiance)
{
    V3<R> sum = v3(R(0), R(0), R(0));
    for (int li = 0; li < S.light_count; ++li)
        sum = add(sum, v3(nee_slot[3 * li], nee_slot[3 * li + 1], nee_slot[3 * li + 2]));
    if (S.light_count > 0) *radiance = add(*radiance, sum);
    *radiance = add(*radiance, v3(nee_slot[3 * kMaxLights], nee_slot[3 * kMaxLights + 1], nee_slot[3 * kMaxLights + 2]));
    for (int k = 0; k < kNeeSlots * 3; ++k) nee_slot[k] = R(0);
}

template <typename R>
MT_D void push_shadow(WfShadow<R> *sq, WfCounters *C, bool want, V3<R> o, V3<R> d, R tmax, V3<R> contrib, int slot,
                      int li)
{
    int at = warp_append(&C->shadow_count, want);
    if (want) {
        WfShadow<R> s;
        s.o[0] = o.x; s.o[1] = o.y; s.o[2] = o.z;
        s.d[0] = d.x; s.d[1] = d.y; s.d[2] = d.z;
        s.tmax = tmax;
        s.contrib[0] = contrib.x; s.contrib[1] = contrib.y; s.contrib[2] = contrib.z;
        s.slot = slot;
        s.li = li;
        sq[at] = s;
    }
}

// ------------------------------------------------------------------
// shade: one bounce of pathtrace_radiance (src/pathtrace.c:835-1018)
// ------------------------------------------------------------------
//
// ADJ: the replay pass of the adjoint. The path's previous vertex (held in
// A.verts) gets its gradient terms once its NEE results are gathered, with
// the remaining radiance L - radiance: from bounce 1 on k_wf_vertex_adj does
// both for the queue before this kernel runs, so the gradient code of a
// vertex is not part of this kernel. Emission and sky terms are taken where
// they occur. The radiance bookkeeping is the primal pass's, so the replay
// reproduces it exactly.
//
// When the bounce's extend results were sorted by material (C->sorted), the
// kernel reads the sorted copies instead.
//
// EXTRAS: the scene has fog, marched media, volumetric clouds or a textured
// material (DevScene::has_extras). Without them those paths are compiled out:
// their out-of-line calls would otherwise constrain the kernel's registers.
// The FP32 forward kernel is held to 7 blocks of 128 per SM (72 registers):
// left alone the compiler takes 79 and the SM runs 6 blocks, which measured
// 22.2 vs 27.0 ms of shading per 16-spp torus-field frame.
//
// PBR: every material of the scene is a PBR surface without water, media or
// atmosphere glow (DevScene::pbr_only). Such a path never enters a medium and
// never takes the legacy BSDF, so those branches compile out and the kernel's
// code (and its instruction-cache footprint) shrinks; the arithmetic of the
// remaining branches is unchanged. The replay (ADJ) kernel takes the same
// specialisation, which also drops the absorption terms of vertex_adjoint;
// each replayed vertex records in its flags which NEE connections it queued,
// so no transmittance record is cleared between vertices. With both, the
// backward of the 512x512, 32-spp adjoint configuration measured 70.1 ms
// against 100.7 ms, gradients equal to 2e-6 relative (float sum order).
// The FP32 replay kernels are held to 7 blocks of 128 per SM as well: for
// the PBR scene (72 registers, 16 bytes of spills) backward 49.3 ms against
// 52.7 at 91 registers and 5 blocks, 53.4 at 6 blocks; with the vertex
// kernels bounded the same way, the water scene's backward (legacy and
// medium terms) took 53.1 ms against 61.2.
template <typename R, bool ADJ, bool EXTRAS, bool PBR = false>
__global__ void __launch_bounds__(kWfMaxBlock, (sizeof(R) == 4 && !EXTRAS) ? 7 : 0) k_wf_shade(const __grid_constant__ DevScene<R> S, const WfRay<R> *rays_in, const WfHit<R> *hits,
                                                  WfCounters *C, int which, int b, int max_depth, WfPath<R> *paths,
                                                  R *nee, WfRay<R> *rays_out, WfShadow<R> *sq, WfAdj<R> A,
                                                  const WfRay<R> *sorted_rays, const WfHit<R> *sorted_hits)
{
    if (!ADJ && sorted_rays && C->sorted) {
        rays_in = sorted_rays;
        hits = sorted_hits;
    }
    __shared__ float adj_g[ADJ ? kAdjMaxParams : 1];
    const AdjCtx ctx = make_adj_ctx(adj_g, S.material_count);
    if constexpr (ADJ) adj_block_begin(adj_g, A.P);
    const int n = C->ray_count[which];
    const int stride = gridDim.x * blockDim.x;
    // Every lane of a warp walks the same number of iterations, so the
    // warp-wide queue appends below always see the whole warp.
    const int n_round = (n + stride - 1) / stride * stride;
    const V3<R> zero = v3(R(0), R(0), R(0));
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n_round; q += stride) {
        const bool active = q < n;
        WfPath<R> st;
        int slot = -1, prim = -1;
        V3<R> throughput = zero, radiance = zero;
        V3<R> beta = zero;       // throughput before the BSDF update: NEE weight
        V3<R> P = zero, N = zero, V = zero;
        V3<R> next_o = zero, next_d = zero;
        int mat = -1, vflags = 0;
        bool shade_hit = false, do_sun = false, cont = false;
        // the material the hit shades with: a local copy with the texture's
        // albedo (src/pathtrace.c:903-905), else the scene's
        DevMaterial<R> m_tex;
        const DevMaterial<R> *msh = S.materials;
        if (active) {
            const WfRay<R> r = rays_in[q];
            const WfHit<R> hh = hits[q];
            slot = r.slot;
            prim = hh.prim;
            st = paths[slot];
            throughput = v3(st.throughput[0], st.throughput[1], st.throughput[2]);
            radiance = v3(st.radiance[0], st.radiance[1], st.radiance[2]);
            // ADJ: k_wf_vertex_adj has gathered this path's NEE results into
            // its radiance and taken its previous vertex's gradient
            if (!ADJ && b > 0) gather_nee(S, nee + (size_t)slot * kNeeSlots * 3, &radiance);
            V3<R> adj = zero, Lp = zero;
            if constexpr (ADJ) {
                adj = adj_of_path(A.P, slot);
                const R *Lq = A.L + 3 * (size_t)slot;
                Lp = v3(Lq[0], Lq[1], Lq[2]);
            }
            const V3<R> ro = v3(r.o[0], r.o[1], r.o[2]);
            const V3<R> d = v3(r.d[0], r.d[1], r.d[2]);
            if (hh.prim < 0) {
                // escaped: medium fallback depth then the sky, through the fog
                // (src/pathtrace.c:837-857)
                if (!PBR && st.medium >= 0) {
                    const V3<R> beta_in = throughput;
                    if constexpr (EXTRAS)
                        pt_water_segment(S, st.medium, ro, d, R(5.0), st.seed_key, b, &throughput, &radiance);
                    else
                        pt_apply_medium(S.materials[st.medium], R(5.0), &throughput, &radiance);
                    if constexpr (ADJ)
                        medium_grad(ctx, S.materials[st.medium], st.medium, R(5.0), beta_in, sub(Lp, radiance), adj);
                    st.medium = -1;
                }
                V3<R> sky_col = sky_sample<R, EXTRAS>(d, S.sky);
                if (EXTRAS && S.fog.density > R(0)) {
                    R T;
                    V3<R> ins;
                    if (b == 0) pt_fog_segment(S, ro, d, R(1e30), st.seed_key, b, &T, &ins);
                    else fog_segment(S.fog, S.sky, ro, d, R(1e30), &T, &ins);
                    sky_col = add(scale(sky_col, T), ins);
                }
                radiance = add(radiance, mul(throughput, sky_col));
                if constexpr (ADJ) sky_sun_grad(ctx, d, S.sky, mul(adj, throughput));
            } else {
                Hit<R> th;
                th.t = hh.t;
                th.u = hh.u;
                th.v = hh.v;
                th.prim = hh.prim;
                th.code = hh.code;
                SurfaceHit<R> h;
                finish_hit(S, ro, unit_dir(d), th, &h);
                if (!PBR && st.medium >= 0) {
                    const V3<R> beta_in = throughput;
                    if constexpr (EXTRAS)
                        pt_water_segment(S, st.medium, ro, d, h.t, st.seed_key, b, &throughput, &radiance);
                    else
                        pt_apply_medium(S.materials[st.medium], h.t, &throughput, &radiance);
                    if constexpr (ADJ)
                        medium_grad(ctx, S.materials[st.medium], st.medium, h.t, beta_in, sub(Lp, radiance), adj);
                } else if (EXTRAS && S.fog.density > R(0)) {
                    R T;
                    V3<R> ins;
                    if (b == 0) pt_fog_segment(S, ro, d, h.t, st.seed_key, b, &T, &ins);
                    else fog_segment(S.fog, S.sky, ro, d, h.t, &T, &ins);
                    radiance = add(radiance, mul(throughput, ins));
                    throughput = scale(throughput, T);
                }
                if (h.material < 0 || h.material >= S.material_count) {
                    radiance = add(radiance, mul(throughput, sky_sample<R, EXTRAS>(d, S.sky)));
                    if constexpr (ADJ) sky_sun_grad(ctx, d, S.sky, mul(adj, throughput));
                } else {
                    const DevMaterial<R> &m = S.materials[h.material];
                    msh = S.materials + h.material;
                    if (EXTRAS && m.texture_kind != 0) {
                        m_tex = m;
                        const V3<R> a = surface_albedo(S, m, ro, unit_dir(d), h);
                        m_tex.albedo[0] = a.x;
                        m_tex.albedo[1] = a.y;
                        m_tex.albedo[2] = a.z;
                        msh = &m_tex;
                    }
                    P = h.point;
                    N = h.normal;
                    if (!PBR && m.is_water) {
                        if (mfabs(h.normal.y) > R(0.999) && mfabs(h.normal.x) < R(1e-4) && mfabs(h.normal.z) < R(1e-4))
                            N = water_normal(P.x, P.z, R(0));
                    }
                    if (dot(N, d) > R(0)) N = neg(N);
                    N = normalize(N);
                    if (length_sq(N) > R(0)) {
                        V = neg(d);
                        mat = h.material;
                        shade_hit = true;
                        beta = throughput;
                        if (b == 0 || st.last_specular) {
                            radiance = add(radiance, mul(throughput, mat3(m.emissive)));
                            if constexpr (ADJ)
                                for (int ch = 0; ch < 3; ++ch)
                                    gadd(ctx, kParamsPerMaterial * mat + 5 + ch,
                                         (float)(comp3(adj, ch) * comp3(throughput, ch)));
                        }
                        if (!PBR && b == 0 && length_sq(mat3(m.atmosphere_glow)) > R(1e-6))
                            radiance = add(radiance, mul(throughput, atmosphere_term(m, N, V, mat3(S.sky.sun_dir))));
                        do_sun = (b == 0 || (b == 1 && st.medium >= 0 && st.last_specular));
                        vflags = (h.front_face ? kVertFront : 0) | (do_sun ? kVertSun : 0);
                        // BSDF sample, throughput update, medium, roulette, advance
                        uint32_t kb = hash3(st.seed_key ^ PT_KEY, (uint32_t)b, 0u);
                        R u1 = rand01<R>(kb, (uint32_t)b, PT_CH_BSDF_A);
                        R u2 = rand01<R>(kb, (uint32_t)b, PT_CH_BSDF_B);
                        R u_lobe = rand01<R>(kb, (uint32_t)b, PT_CH_LOBE);
                        R u_glass = rand01<R>(kb, (uint32_t)b, PT_CH_GLASS);
                        V3<R> wi, w;
                        int refracted = 0, sampled_specular = 0;
                        bool ok;
                        if (PBR || m.pbr)
                            ok = pt_sample_pbr(*msh, N, d, V, u1, u2, u_lobe, &wi, &w, &sampled_specular);
                        else
                            ok = pt_sample_legacy(*msh, N, d, V, h.front_face, u1, u2, u_lobe, u_glass, &wi, &w,
                                                  &refracted, &sampled_specular);
                        if (ok) {
                            st.last_specular = sampled_specular;
                            throughput = mul(throughput, w);
                            if (finite3(throughput) && pt_max_component(throughput) > R(0)) {
                                if (!PBR && refracted && (m.is_water || m.beer_lambert))
                                    st.medium = h.front_face ? h.material : -1;
                                bool alive = true;
                                if (b >= 2) {  // PT_RR_START_BOUNCE (src/pathtrace.c:69)
                                    R qv = pt_clamp01(pt_max_component(throughput));
                                    if (!(qv > R(0))) {
                                        alive = false;
                                    } else {
                                        R u_rr = rand01<R>(kb, (uint32_t)b, PT_CH_RR);
                                        if (u_rr >= qv) alive = false;
                                        else throughput = scale(throughput, R(1) / qv);
                                    }
                                }
                                if (alive && b < max_depth) {
                                    V3<R> offset = refracted ? scale(wi, R(1e-4))
                                                             : scale(N, dot(wi, N) >= R(0) ? R(1e-4) : R(-1e-4));
                                    next_o = add(P, offset);
                                    next_d = wi;
                                    cont = true;
                                }
                            }
                        }
                    }
                }
            }
        }
        // ---- NEE connections of this bounce (lights in order, then the sun) ----
        // pt_nee_emissive (src/pathtrace.c:576-606)
        for (int li = 0; li < S.light_count; ++li) {
            bool want = false;
            V3<R> so = zero, wi = zero, contrib = zero;
            R tmax = R(0);
            if (shade_hit) {
                const DevLight<R> &lt = S.lights[li];
                if (lt.prim != prim) {
                    V3<R> to_c = sub(mat3(lt.center), P);
                    R dc2 = length_sq(to_c);
                    R dc = msqrt(dc2);
                    if (dc > lt.radius) {
                        R cos_mx = msqrt(R(1) - (lt.radius * lt.radius) / dc2);
                        const R omc = cone_one_minus_cos((lt.radius * lt.radius) / dc2, cos_mx);
                        R Omega = R(2) * R(3.14159265358979323846) * omc;
                        if (Omega > R(0)) {
                            V3<R> w = scale(to_c, R(1) / dc);
                            R u1 = rand01<R>(st.seed_key ^ (uint32_t)li, (uint32_t)b, PT_CH_NEE_EMIT_A);
                            R u2 = rand01<R>(st.seed_key ^ (uint32_t)li, (uint32_t)b, PT_CH_NEE_EMIT_B);
                            wi = light_sphere_sample_dir(w, cos_mx, omc, u1, u2);
                            if (finite3(wi) && dot(N, wi) > R(0)) {
                                so = add(P, scale(N, R(1e-3)));
                                R lt_t;
                                if (light_sphere_t(S, lt.prim, so, wi, R(1e-3), R(1e30), &lt_t)) {
                                    V3<R> lit = PBR ? shade_pbr(*msh, N, wi, V, mat3(lt.emissive))
                                                    : shade(*msh, N, wi, V, mat3(lt.emissive));
                                    contrib = mul(beta, scale(lit, Omega));
                                    tmax = lt_t - R(1e-3);
                                    want = true;
                                    vflags |= vert_conn_bit(li);
                                }
                            }
                        }
                    }
                }
            }
            push_shadow(sq, C, want, so, wi, tmax, contrib, slot, li);
        }
        {
            // pt_nee_sun (src/pathtrace.c:534-556)
            bool want = false;
            V3<R> so = zero, L = zero, contrib = zero;
            if (shade_hit && do_sun) {
                R r1 = rand01<R>(st.seed_key, (uint32_t)b, PT_CH_NEE_SUN_A);
                R r2 = rand01<R>(st.seed_key, (uint32_t)b, PT_CH_NEE_SUN_B);
                L = sun_disk_dir(mat3(S.sky.sun_dir), S.sky.sun_radius, r1, r2);
                if (finite3(L) && dot(N, L) > R(0)) {
                    so = add(P, scale(N, R(1e-3)));
                    R rad = S.sky.sun_radius * R(3.14159265358979323846) / R(180);
                    R Omega = (S.sky.sun_radius > R(0)) ? R(2) * R(3.14159265358979323846) * (R(1) - mcos(rad)) : R(1);
                    V3<R> lit = PBR ? shade_pbr(*msh, N, L, V, mat3(S.sky.sun_color))
                                    : shade(*msh, N, L, V, mat3(S.sky.sun_color));
                    contrib = mul(beta, scale(lit, Omega));
                    want = true;
                    vflags |= vert_conn_bit(kMaxLights);
                }
            }
            push_shadow(sq, C, want, so, L, R(1e30), contrib, slot, kMaxLights);
        }
        // ---- next ray ----
        int at = warp_append(&C->ray_count[which ^ 1], cont);
        if (cont) {
            WfRay<R> nr;
            nr.o[0] = next_o.x; nr.o[1] = next_o.y; nr.o[2] = next_o.z;
            nr.d[0] = next_d.x; nr.d[1] = next_d.y; nr.d[2] = next_d.z;
            nr.slot = slot;
            nr.pad = 0;
            rays_out[at] = nr;
        }
        if (active) {
            st.throughput[0] = throughput.x;
            st.throughput[1] = throughput.y;
            st.throughput[2] = throughput.z;
            st.radiance[0] = radiance.x;
            st.radiance[1] = radiance.y;
            st.radiance[2] = radiance.z;
            paths[slot] = st;
            if constexpr (ADJ) {
                AdjVertex<R> vx;
                vx.p[0] = P.x; vx.p[1] = P.y; vx.p[2] = P.z;
                vx.n[0] = N.x; vx.n[1] = N.y; vx.n[2] = N.z;
                vx.v[0] = V.x; vx.v[1] = V.y; vx.v[2] = V.z;
                vx.beta[0] = beta.x; vx.beta[1] = beta.y; vx.beta[2] = beta.z;
                vx.mat = shade_hit ? mat : -1;
                vx.b = b;
                vx.flags = vflags;
                vx.pad = 0;
                A.verts[slot] = vx;
            }
        }
    }
    if constexpr (ADJ) adj_block_end(adj_g, A.P);
}

// ------------------------------------------------------------------
// sort by material and place: a counting sort of one bounce's extend results
// by (material hit, Morton cell of the hit point), bucket M = no surface, so
// that the shade kernel's warps see one material, hence one BSDF code path, at
// a time, and consecutive paths sit close together in the scene. The shade
// kernel appends each warp's NEE connections light by light, so the shadow
// queue then holds runs of up to 32 rays toward one light from nearby points,
// which walk nearly the same nodes. The cells split the root box into
// 2^bits per axis; bits shrinks as the material count grows so the bucket
// count stays <= kSortMaxBuckets. It runs only when the queue holds at least
// `threshold` rays (decided on the device). Queue order never changes a
// path's result: every path keeps its own slot, NEE slots and sample index.
// Lanes of a warp with the same key share one atomicAdd.
// ------------------------------------------------------------------
static constexpr int kSortMaxBuckets = 1 << 16;
static constexpr int kSortMaxCellBits = 4;

// Cell bits per axis for `keys` material keys (materials + 1).
MT_HD int sort_cell_bits(int keys)
{
    int b = kSortMaxCellBits;
    while (b > 0 && ((long long)keys << (3 * b)) > kSortMaxBuckets) --b;
    return b;
}

// Buckets of the sort: material keys x cells.
MT_HD int sort_buckets(int keys) { return keys << (3 * sort_cell_bits(keys)); }

// Morton cell (bits per axis) of point p in the root box of the tree.
template <typename R> MT_D int sort_cell(const DevScene<R> &S, R px, R py, R pz, int bits)
{
    if (bits == 0 || S.node_count <= 0) return 0;
    const float4 q0 = __ldg(S.nodes), q1 = __ldg(S.nodes + 1), q2 = __ldg(S.nodes + 2);
    const float lo[3] = {fminf(q0.x, q1.x), fminf(q0.z, q1.z), fminf(q2.x, q2.z)};
    const float hi[3] = {fmaxf(q0.y, q1.y), fmaxf(q0.w, q1.w), fmaxf(q2.y, q2.w)};
    const float p[3] = {(float)px, (float)py, (float)pz};
    const int top = (1 << bits) - 1;
    int cell = 0;
    for (int k = 0; k < 3; ++k) {
        const float ext = hi[k] - lo[k];
        const float f = ext > 0.f ? (p[k] - lo[k]) * ((float)(1 << bits) / ext) : 0.f;
        int v = f > 0.f ? (int)f : 0;  // NaN and points below the box go to cell 0
        v = v > top ? top : v;
        for (int j = 0; j < bits; ++j) cell |= ((v >> j) & 1) << (3 * j + k);
    }
    return cell;
}

MT_D int warp_add_by_key(int *counters, int key, bool want)
{
    const unsigned active = __ballot_sync(0xffffffffu, want);
    if (!want) return 0;
    const unsigned peers = __match_any_sync(active, key);
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(peers) - 1;
    int base = 0;
    if (lane == leader) base = atomicAdd(&counters[key], __popc(peers));
    base = __shfl_sync(peers, base, leader);
    return base + __popc(peers & ((1u << lane) - 1u));
}

template <typename R>
__global__ void k_wf_sort_count(const __grid_constant__ DevScene<R> S, WfCounters *C, int which, const WfRay<R> *rays,
                                const WfHit<R> *hits, int *keys, int *buckets, int threshold)
{
    const int n = C->ray_count[which];
    if (blockIdx.x == 0 && threadIdx.x == 0) C->sorted = n >= threshold;
    if (n < threshold) return;
    const int M = S.material_count;
    const int bits = sort_cell_bits(M + 1);
    const int stride = gridDim.x * blockDim.x;
    const int n_round = (n + stride - 1) / stride * stride;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n_round; q += stride) {
        int key = M << (3 * bits);
        if (q < n) {
            const WfHit<R> hq = hits[q];
            if (hq.prim >= 0) {
                const int m = __ldg(S.prim_info + hq.prim).y;
                if (m >= 0 && m < M) {
                    const WfRay<R> &r = rays[q];
                    key = (m << (3 * bits)) | sort_cell(S, r.o[0] + hq.t * r.d[0], r.o[1] + hq.t * r.d[1],
                                                        r.o[2] + hq.t * r.d[2], bits);
                }
            }
            keys[q] = key;
        }
        warp_add_by_key(buckets, key, q < n);
    }
}

// Exclusive scan of the nb bucket counts into the cursors (buckets[nb..2nb)):
// one block of kSortScanThreads, each thread a contiguous run of buckets.
static constexpr int kSortScanThreads = 1024;
template <typename R>
__global__ void __launch_bounds__(kSortScanThreads) k_wf_sort_scan(const WfCounters *C, int *buckets, int nb)
{
    __shared__ int warp_sum[kSortScanThreads / 32];
    if (!C->sorted) return;
    const int per = (nb + kSortScanThreads - 1) / kSortScanThreads;
    const int b0 = threadIdx.x * per;
    const int b1 = min(b0 + per, nb);
    int sum = 0;
    for (int k = b0; k < b1; ++k) sum += buckets[k];
    // inclusive scan of the thread sums: within the warp, then across warps
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int x = sum;
    for (int off = 1; off < 32; off <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, off);
        if (lane >= off) x += y;
    }
    if (lane == 31) warp_sum[wid] = x;
    __syncthreads();
    if (wid == 0) {
        int w = warp_sum[lane];
        for (int off = 1; off < 32; off <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, w, off);
            if (lane >= off) w += y;
        }
        warp_sum[lane] = w;
    }
    __syncthreads();
    int acc = x - sum + (wid > 0 ? warp_sum[wid - 1] : 0);
    for (int k = b0; k < b1; ++k) {
        buckets[nb + k] = acc;
        acc += buckets[k];
    }
}

template <typename R>
__global__ void k_wf_sort_scatter(const WfCounters *C, int which, const WfRay<R> *rays, const WfHit<R> *hits,
                                  const int *keys, int *buckets, int nb, WfRay<R> *sorted_rays,
                                  WfHit<R> *sorted_hits)
{
    if (!C->sorted) return;
    const int n = C->ray_count[which];
    int *cursors = buckets + nb;
    const int stride = gridDim.x * blockDim.x;
    const int n_round = (n + stride - 1) / stride * stride;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n_round; q += stride) {
        const int key = q < n ? keys[q] : 0;
        const int pos = warp_add_by_key(cursors, key, q < n);
        if (q < n) {
            sorted_rays[pos] = rays[q];
            sorted_hits[pos] = hits[q];
        }
    }
}

// ------------------------------------------------------------------
// shadow: pt_occluded_segment (src/pathtrace.c:504-532) per NEE connection
// ------------------------------------------------------------------
// ADJ: also keep the connection's transmittance (zero when it adds no light)
// for the replay's gradient terms.
//
// PASS: some material of the scene lets shadow rays through (has_passthrough),
// so connections take the chained walk; otherwise one any-hit query each.
//
// In a scene without pass-through materials the stage runs in two passes
// over the occluder cache, which holds for each connection's entry (see
// occ_entry) the kOccWays BVH leaves that most recently blocked a connection
// there: k_wf_shadow_cache tests the primitives of every connection's cached
// leaves (a hit there is a hit of the any-hit query, so the answer cannot
// change), resolves the blocked ones and appends the others to `walk`;
// k_wf_shadow then walks the tree for `walk` only and pushes each blocking leaf
// it finds to the front of the entry (scene_any_cached); a probe that hits a
// later way moves that leaf to the front (occ_ways_hit). Cache hits (a few
// primitive tests) and walks (the whole tree) therefore do not share warps.

// Occluder cache entry of a connection. At bounce 0, per pixel and NEE slot:
// the samples of a pixel shade nearly the same point. Later, a hash of (cell
// of the origin, NEE slot) into kOccHash entries after the per-pixel part,
// with 2^kOccCellBits cells per axis of the root box: nearby origins toward
// one light tend to share a blocker. A collision only costs a primitive test,
// since an entry is just a candidate. (On the 1M-triangle torus field 256
// cells per axis did best: 64 and 4096 were both slower.)
static constexpr int kOccHashBits = 22;
static constexpr int kOccHash = 1 << kOccHashBits;
static constexpr int kOccCellBits = 8;
// Blocking leaves kept per entry, newest first: the samples of a pixel toward
// one light meet a handful of blockers (on the torus field 1 / 2 / 4 / 8 ways:
// 59.7 / 46.4 / 39.5 / 45.5 ms of shadow stage per 16-spp frame).
static constexpr int kOccWays = 4;

// ints of the occluder cache for `wh` pixels
inline size_t occ_cache_ints(size_t wh) { return (wh * kNeeSlots + kOccHash) * kOccWays; }
template <typename R> MT_D int *occ_entry(const DevScene<R> &S, int *occ_cache, int wh, int b, const WfShadow<R> &s)
{
    if (b == 0) return occ_cache + ((size_t)(s.slot % wh) * kNeeSlots + s.li) * kOccWays;
    unsigned c[3] = {0u, 0u, 0u};
    if (S.node_count > 0) {
        const float4 q0 = __ldg(S.nodes), q1 = __ldg(S.nodes + 1), q2 = __ldg(S.nodes + 2);
        const float lo[3] = {fminf(q0.x, q1.x), fminf(q0.z, q1.z), fminf(q2.x, q2.z)};
        const float hi[3] = {fmaxf(q0.y, q1.y), fmaxf(q0.w, q1.w), fmaxf(q2.y, q2.w)};
        const int top = (1 << kOccCellBits) - 1;
        for (int k = 0; k < 3; ++k) {
            const float ext = hi[k] - lo[k];
            const float f = ext > 0.f ? ((float)s.o[k] - lo[k]) * ((float)(1 << kOccCellBits) / ext) : 0.f;
            int v = f > 0.f ? (int)f : 0;
            c[k] = (unsigned)(v > top ? top : v);
        }
    }
    unsigned h = c[0] * 73856093u ^ c[1] * 19349663u ^ c[2] * 83492791u ^ (unsigned)s.li * 2654435761u;
    h ^= h >> 15;
    h *= 2246822519u;
    h ^= h >> 13;
    return occ_cache + ((size_t)wh * kNeeSlots + (h & (kOccHash - 1))) * kOccWays;
}

// Result of one connection: its NEE slot (and, ADJ, its transmittance record).
template <typename R, bool ADJ>
MT_D void shadow_result(const WfShadow<R> &s, bool occ, V3<R> atten, const AbsorbPath<R> &ab, R *nee, R *att)
{
    V3<R> res = v3(R(0), R(0), R(0));
    bool lit = false;
    if (!occ) {
        bool dark = s.li == kMaxLights && atten.x < R(1e-4) && atten.y < R(1e-4) && atten.z < R(1e-4);
        if (!dark) {
            res = mul(v3(s.contrib[0], s.contrib[1], s.contrib[2]), atten);
            lit = true;
        }
    }
    const size_t at = ((size_t)s.slot * kNeeSlots + s.li) * 3;
    R *slot = nee + at;
    slot[0] = res.x;
    slot[1] = res.y;
    slot[2] = res.z;
    if constexpr (ADJ) {
        R *rec = att + ((size_t)s.slot * kNeeSlots + s.li) * kAttStride;
        if (lit) {
            set_att(rec, atten, ab);
        } else {  // the reader tests the transmittance first
            rec[0] = R(0);
            rec[1] = R(0);
            rec[2] = R(0);
        }
    }
}

// State of a pass-through chain between two of its links (the loop of
// pt_occluded_segment, src/pathtrace.c:504-532): the next link's origin,
// the length left, the attenuation so far and the connection sq[q].
template <typename R> struct __align__(16) WfLink {
    R o[3];
    R remaining;
    R att[3];
    int q;
};

// One link (step `step`, 0..5) of pt_occluded_segment's chain. Returns 0 (not
// occluded), 1 (occluded) or 2 (passed a transparent hit: cur_o, tmin,
// remaining and atten hold the next link). `leaf`: see scene_link.
template <typename R>
MT_D int chain_link(const DevScene<R> &S, V3<R> &cur_o, V3<R> d, R &tmin, R &remaining, V3<R> &atten, int step,
                    int *leaf = nullptr)
{
    LinkHit<R> h;
    if (!scene_link(S, cur_o, d, tmin, remaining, &h, leaf)) return 0;
    if (h.material < 0 || h.material >= S.material_count) return 1;
    const DevMaterial<R> &m = S.materials[h.material];
    if (!(m.is_water || m.transparency > R(0.8))) return 1;
    if (m.beer_lambert || m.is_water) {
        V3<R> seg = v3(mexp(-m.absorption[0] * h.t), mexp(-m.absorption[1] * h.t), mexp(-m.absorption[2] * h.t));
        atten = mul(atten, seg);
    }
    cur_o = add(h.point, scale(d, R(1e-3)));
    remaining -= h.t;
    if (remaining <= R(1e-3)) return 0;
    tmin = R(1e-3);
    return step < 5 ? 2 : 1;  // six links at most, then occluded
}

// Append chain state to the link queue `out`. Its capacity `cap` is the
// stage's shadow-connection capacity, and every launch appends at most one
// record per connection it reads, so it cannot fill; if it ever did, the
// error word says so (ERR_QUEUE) and the record is dropped.
template <typename R>
MT_D void push_link(const DevScene<R> &S, WfLink<R> *out, int *count, int cap, V3<R> o, R remaining, V3<R> atten,
                    int q)
{
    const int at = warp_append(count, true);
    if (at >= cap) {
        atomicOr(S.err, ERR_QUEUE);
        return;
    }
    WfLink<R> L;
    L.o[0] = o.x;
    L.o[1] = o.y;
    L.o[2] = o.z;
    L.remaining = remaining;
    L.att[0] = atten.x;
    L.att[1] = atten.y;
    L.att[2] = atten.z;
    L.q = q;
    out[at] = L;
}

// `walk` (may be NULL): the connections to process are sq[walk[0 .. C->walk_count)]
// and their cached occluder has already missed; otherwise sq[0 .. C->shadow_count).
template <typename R, bool ADJ, int W, bool PASS, bool LINKED = false>
// (binary tree: at most 72 registers, so 7 blocks of 128 fit an SM; the
// pass-through instantiation would otherwise take 80 and run 6)
//
// PASS and LINKED (not the adjoint): only the chain's first link runs here;
// chains that pass a transparent hit go to the link queue (link_count[0]) and
// k_wf_shadow_link runs their next links, one launch per link, so that the
// lanes of a warp do not wait for the longest chain among them.
__global__ void __launch_bounds__(kWfMaxBlock, W == 2 ? (PASS ? MT_PASS_MIN_BLOCKS : MT_SHADOW_MIN_BLOCKS) : 1) k_wf_shadow(const __grid_constant__ DevScene<R> S, const WfShadow<R> *sq, WfCounters *C,
                                                   R *nee, R *att, int *occ_cache, int wh, int b, const int *walk,
                                                   WfLink<R> *link, int link_cap)
{
    const int n = walk ? C->walk_count : C->shadow_count;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
        const int qs = walk ? walk[q] : q;
        const WfShadow<R> s = sq[qs];
        V3<R> o = v3(s.o[0], s.o[1], s.o[2]);
        V3<R> d = v3(s.d[0], s.d[1], s.d[2]);
        V3<R> atten;
        AbsorbPath<R> ab;
        ab.mat[0] = ab.mat[1] = -1;
        ab.dist[0] = ab.dist[1] = R(0);
        bool occ;
        if constexpr (PASS) {
            // with `walk`, the connections whose cached blockers did not
            // settle them (k_wf_shadow_pass_cache): the chain records the
            // blocker it meets; the adjoint keeps the plain chain
            if constexpr (ADJ) {
                occ = pt_occluded_segment_abs(S, o, d, R(1e-3), s.tmax, &atten, &ab);
            } else {
                // pt_occluded_segment's chain, link by link; the first link's
                // opaque blocker goes to the front of the entry
                int *entry = walk ? occ_entry(S, occ_cache, wh, b, s) : nullptr;
                if (S.counters && !walk) atomicAdd(&S.counters->shadow_rays, 1ull);
                atten = v3(R(1), R(1), R(1));
                V3<R> cur_o = o;
                R tmin = R(1e-3), remaining = s.tmax;
                int leaf = -1;
                int r = chain_link(S, cur_o, d, tmin, remaining, atten, 0, &leaf);
                if (r == 1 && entry && leaf != -1) {
                    const int4 e = *reinterpret_cast<const int4 *>(entry);
                    if (e.x != leaf) *reinterpret_cast<int4 *>(entry) = make_int4(leaf, e.x, e.y, e.z);
                }
                if (LINKED) {
                    if (r == 2) {
                        push_link(S, link, &C->link_count[0], link_cap, cur_o, remaining, atten, qs);
                        continue;
                    }
                } else {
                    for (int step = 1; r == 2; ++step) r = chain_link(S, cur_o, d, tmin, remaining, atten, step);
                }
                occ = r == 1;
            }
        } else {
            // No material lets a shadow ray through: the chained nearest-hit
            // walk stops at its first hit, so it equals an any-hit query.
            atten = v3(R(1), R(1), R(1));
            if (S.counters && !walk) atomicAdd(&S.counters->shadow_rays, 1ull);
            if (occ_cache)
                occ = scene_any_cached<R, W, kOccWays>(S, ray_pre(o, unit_dir(d)), R(1e-3), s.tmax,
                                             occ_entry(S, occ_cache, wh, b, s), !walk);
            else
                occ = scene_any<R, W>(S, ray_pre(o, unit_dir(d)), R(1e-3), s.tmax);
        }
        // the sun through volumetric clouds (pt_nee_sun, src/pathtrace.c:545-546)
        if (!occ && s.li == kMaxLights) atten = scale(atten, cloud_transmittance(S.sky, o, d));
        shadow_result<R, ADJ>(s, occ, atten, ab, nee, att);
        if (S.trace_rec) trace_put(S, o, unit_dir(d), s.tmax, occ ? 1 : 0, 1, b, s.li);
    }
}

// Link `step` (1..5) of the pass-through chains queued by the previous link
// (in[0 .. min(link_count[step - 1], cap))); chains that pass another
// transparent hit go to `out` (link_count[step]), the others write their
// connection's result. LAST: every chain runs to its end here (the few
// long chains left would otherwise pay one launch per link).
template <typename R, bool LAST>
__global__ void __launch_bounds__(kWfMaxBlock, MT_PASS_MIN_BLOCKS) k_wf_shadow_link(const __grid_constant__ DevScene<R> S, const WfShadow<R> *sq,
                                                                   WfCounters *C, R *nee, int b, int step,
                                                                   const WfLink<R> *in, WfLink<R> *out, int cap)
{
    const int c = C->link_count[step - 1];
    const int n = c < cap ? c : cap;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const WfLink<R> L = in[i];
        const WfShadow<R> s = sq[L.q];
        const V3<R> d = v3(s.d[0], s.d[1], s.d[2]);
        V3<R> cur_o = v3(L.o[0], L.o[1], L.o[2]);
        V3<R> atten = v3(L.att[0], L.att[1], L.att[2]);
        R tmin = R(1e-3), remaining = L.remaining;
        int r = chain_link(S, cur_o, d, tmin, remaining, atten, step);
        if constexpr (LAST) {
            for (int k = step + 1; r == 2; ++k) r = chain_link(S, cur_o, d, tmin, remaining, atten, k);
        } else if (r == 2) {
            push_link(S, out, &C->link_count[step], cap, cur_o, remaining, atten, L.q);
            continue;
        }
        const bool occ = r == 1;
        const V3<R> o = v3(s.o[0], s.o[1], s.o[2]);
        // the sun through volumetric clouds (pt_nee_sun, src/pathtrace.c:545-546)
        if (!occ && s.li == kMaxLights) atten = scale(atten, cloud_transmittance(S.sky, o, d));
        AbsorbPath<R> ab;
        ab.mat[0] = ab.mat[1] = -1;
        ab.dist[0] = ab.dist[1] = R(0);
        shadow_result<R, false>(s, occ, atten, ab, nee, nullptr);
        if (S.trace_rec) trace_put(S, o, unit_dir(d), s.tmax, occ ? 1 : 0, 1, b, s.li);
    }
}

// First pass of bounce 0 (scenes without pass-through materials): the cached
// occluder of every connection; misses go to `walk` (warp-aggregated appends).
// Held to 64 registers (8 blocks of 128 per SM), as it compiles without the
// query log.
template <typename R, bool ADJ>
__global__ void __launch_bounds__(kWfMaxBlock, 8) k_wf_shadow_cache(const __grid_constant__ DevScene<R> S, const WfShadow<R> *sq,
                                                         WfCounters *C, R *nee, R *att, int *occ_cache, int wh,
                                                         int b, int *walk)
{
    const int n = C->shadow_count;
    const int stride = gridDim.x * blockDim.x;
    const int n_round = (n + stride - 1) / stride * stride;
    AbsorbPath<R> ab;
    ab.mat[0] = ab.mat[1] = -1;
    ab.dist[0] = ab.dist[1] = R(0);
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n_round; q += stride) {
        bool miss = false;
        if (q < n) {
            const WfShadow<R> s = sq[q];
            if (S.counters) atomicAdd(&S.counters->shadow_rays, 1ull);
            const bool blocked =
                occ_ways_hit<R, kOccWays, true>(
                    S, occ_entry(S, occ_cache, wh, b, s),
                    ray_pre(v3(s.o[0], s.o[1], s.o[2]), unit_dir(v3(s.d[0], s.d[1], s.d[2]))), R(1e-3), s.tmax) >= 0;
            if (blocked) {
                if (S.counters) atomicAdd(&S.counters->any_prim_tests, 1ull);
                shadow_result<R, ADJ>(s, true, v3(R(1), R(1), R(1)), ab, nee, att);
                if (S.trace_rec)
                    trace_put(S, v3(s.o[0], s.o[1], s.o[2]), unit_dir(v3(s.d[0], s.d[1], s.d[2])), s.tmax, 1, 1, b,
                              s.li);
            } else {
                miss = true;
            }
        }
        const int at = warp_append(&C->walk_count, miss);
        if (miss) walk[at] = q;
    }
}

// First pass of the shadow stage of a scene with pass-through materials
// (pass tree built, occluder cache on): connections that a cached opaque
// blocker settles (pass_cache_occluded) are answered here; the rest go to
// `walk` for the chain (k_wf_shadow, PASS).
template <typename R>
__global__ void __launch_bounds__(kWfMaxBlock, MT_SHADOW_MIN_BLOCKS) k_wf_shadow_pass_cache(const __grid_constant__ DevScene<R> S, const WfShadow<R> *sq,
                                                                          WfCounters *C, R *nee, int *occ_cache,
                                                                          int wh, int b, int *walk)
{
    const int n = C->shadow_count;
    const int stride = gridDim.x * blockDim.x;
    const int n_round = (n + stride - 1) / stride * stride;
    AbsorbPath<R> ab;
    ab.mat[0] = ab.mat[1] = -1;
    ab.dist[0] = ab.dist[1] = R(0);
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n_round; q += stride) {
        bool miss = false;
        if (q < n) {
            const WfShadow<R> s = sq[q];
            if (S.counters) atomicAdd(&S.counters->shadow_rays, 1ull);
            const V3<R> o = v3(s.o[0], s.o[1], s.o[2]);
            const V3<R> du = unit_dir(v3(s.d[0], s.d[1], s.d[2]));
            if (pass_cache_occluded(S, occ_entry(S, occ_cache, wh, b, s), ray_pre(o, du), R(1e-3), s.tmax)) {
                if (S.counters) atomicAdd(&S.counters->any_prim_tests, 1ull);
                shadow_result<R, false>(s, true, v3(R(1), R(1), R(1)), ab, nee, nullptr);
                if (S.trace_rec) trace_put(S, o, du, s.tmax, 1, 1, b, s.li);
            } else {
                miss = true;
            }
        }
        const int at = warp_append(&C->walk_count, miss);
        if (miss) walk[at] = q;
    }
}

// ------------------------------------------------------------------
// Dynamic ray fetch (persistent threads with per-lane refill; Aila and
// Laine, HPG 2009): every lane walks its ray one leaf at a time (trav_step)
// and, once it is done, takes the next ray of the queue, so lanes whose rays
// end early do not idle until the warp's longest walk is over. Refills are
// warp-aggregated: one atomicAdd hands out consecutive rays to every idle
// lane, once at least kFetchMin lanes are idle or no lane is busy. Results
// are those of the grid-stride kernels above; only the ray-to-lane schedule
// differs.
// ------------------------------------------------------------------
static constexpr int kFetchMin = 8;

// One refill round. Returns the ray this lane takes (-1: none this round);
// sets *more = false once the queue of `n` rays is drained for this lane.
MT_D int fetch_round(int *counter, int n, bool idle, bool busy_lane, bool *more)
{
    const unsigned want = __ballot_sync(0xffffffffu, idle);
    const unsigned busy = __ballot_sync(0xffffffffu, busy_lane);
    if (!want || (busy && __popc(want) < kFetchMin)) return -1;
    const int leader = __ffs(want) - 1;
    const int lane = threadIdx.x & 31;
    int base = 0;
    if (lane == leader) base = atomicAdd(counter, __popc(want));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (!idle) return -1;
    const int mine = base + __popc(want & ((1u << lane) - 1u));
    if (mine >= n) {
        *more = false;
        return -1;
    }
    return mine;
}

template <typename R, int W>
__global__ void __launch_bounds__(kWfMaxBlock) k_wf_extend_dyn(const __grid_constant__ DevScene<R> S, const WfRay<R> *rays, WfCounters *C,
                                                       int which, WfHit<R> *hits)
{
    const int n = C->ray_count[which];
    int *stk = mt_stack_smem + threadIdx.x;
    const int stride = blockDim.x;
    int q = -1;
    bool more = true;
    Trav<R> tv;
    Hit<R> best;
    TravCount cnt;
    while (__any_sync(0xffffffffu, q >= 0 || more)) {
        const int f = fetch_round(&C->ray_fetch, n, q < 0 && more, q >= 0, &more);
        if (f >= 0) {
            q = f;
            const WfRay<R> r = rays[q];
            V3<R> d = unit_dir(v3(r.d[0], r.d[1], r.d[2]));
            trav_init<R, false>(S, tv, ray_pre(v3(r.o[0], r.o[1], r.o[2]), d), R(1e-4), R(1e30), &best, cnt);
        }
        if (q >= 0) {
            if (tv.node == kEmpty || !trav_step<R, false, W>(S, tv, stk, stride, &best, cnt)) {
                WfHit<R> out;
                out.t = tv.found ? best.t : R(0);
                out.u = tv.found ? best.u : R(0);
                out.v = tv.found ? best.v : R(0);
                out.prim = tv.found ? best.prim : -1;
                out.code = tv.found ? best.code : 0;
                hits[q] = out;
                q = -1;
            }
        }
    }
    trav_count_flush<R, false>(S, cnt);
    if (S.counters && blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&S.counters->extension_rays, (unsigned long long)n);
}

// Shadow rays of a scene without pass-through materials: a pure any-hit
// query per connection (see k_wf_shadow).
template <typename R, bool ADJ, int W>
__global__ void __launch_bounds__(kWfMaxBlock) k_wf_shadow_dyn(const __grid_constant__ DevScene<R> S, const WfShadow<R> *sq, WfCounters *C,
                                                       R *nee, R *att)
{
    const int n = C->shadow_count;
    int *stk = mt_stack_smem + threadIdx.x;
    const int stride = blockDim.x;
    int q = -1;
    bool more = true;
    Trav<R> tv;
    Hit<R> unused;
    TravCount cnt;
    while (__any_sync(0xffffffffu, q >= 0 || more)) {
        const int f = fetch_round(&C->shadow_fetch, n, q < 0 && more, q >= 0, &more);
        if (f >= 0) {
            q = f;
            const WfShadow<R> s = sq[q];
            V3<R> d = unit_dir(v3(s.d[0], s.d[1], s.d[2]));
            trav_init<R, true>(S, tv, ray_pre(v3(s.o[0], s.o[1], s.o[2]), d), R(1e-3), s.tmax, &unused, cnt);
        }
        if (q >= 0) {
            if (tv.node == kEmpty || !trav_step<R, true, W>(S, tv, stk, stride, &unused, cnt)) {
                const WfShadow<R> &s = sq[q];
                V3<R> atten = v3(R(1), R(1), R(1));
                if (!tv.found && s.li == kMaxLights)
                    atten = scale(atten, cloud_transmittance(S.sky, v3(s.o[0], s.o[1], s.o[2]),
                                                             v3(s.d[0], s.d[1], s.d[2])));
                AbsorbPath<R> ab;
                ab.mat[0] = ab.mat[1] = -1;
                ab.dist[0] = ab.dist[1] = R(0);
                shadow_result<R, ADJ>(s, tv.found, atten, ab, nee, att);
                if (S.trace_rec)
                    trace_put(S, v3(s.o[0], s.o[1], s.o[2]), unit_dir(v3(s.d[0], s.d[1], s.d[2])), s.tmax, tv.found ? 1 : 0, 1, -1,
                              s.li);
                q = -1;
            }
        }
    }
    trav_count_flush<R, true>(S, cnt);
    if (S.counters && blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&S.counters->shadow_rays, (unsigned long long)n);
}

// ------------------------------------------------------------------
// finalize + reduce: per-sample radiance (final clamp of
// src/pathtrace.c:1020-1027) and the per-pixel sum in sample order
// ------------------------------------------------------------------
// The final radiance of path q: its last bounce's NEE gathered, then the
// reference's final NaN -> 0 and negative clamp (src/pathtrace.c:1020-1027).
template <typename R> MT_D V3<R> finalize_path(const DevScene<R> &S, const WfPath<R> *paths, R *nee, size_t q)
{
    const WfPath<R> st = paths[q];
    V3<R> radiance = v3(st.radiance[0], st.radiance[1], st.radiance[2]);
    gather_nee(S, nee + q * kNeeSlots * 3, &radiance);
    if (!finite3(radiance)) radiance = v3(R(0), R(0), R(0));
    if (radiance.x < R(0)) radiance.x = R(0);
    if (radiance.y < R(0)) radiance.y = R(0);
    if (radiance.z < R(0)) radiance.z = R(0);
    return radiance;
}

template <typename R>
__global__ void k_wf_finalize(const __grid_constant__ DevScene<R> S, int n_paths, const WfPath<R> *paths, R *nee, R *sample_buf)
{
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n_paths; q += gridDim.x * blockDim.x) {
        const V3<R> radiance = finalize_path(S, paths, nee, (size_t)q);
        sample_buf[3 * (size_t)q] = radiance.x;
        sample_buf[3 * (size_t)q + 1] = radiance.y;
        sample_buf[3 * (size_t)q + 2] = radiance.z;
    }
}

// Adjoint replay, before the shade of bounce b >= 1: every path of the
// bounce's ray queue gathers its NEE results into its radiance (written back;
// the shade kernel then skips the gather) and its previous vertex takes its
// gradient terms against L - radiance. Kept out of k_wf_shade: with the
// gradient code inside, the replay shade was bound by instruction fetch.
// PBR as in k_wf_shade. The FP32 kernels are held to 7 blocks of 128 per SM
// (72 registers, 88 bytes of spills for PBR): backward 46.9 ms against 49.2
// at 91 registers and 5 blocks; 6 blocks measured no change.
template <typename R, bool PBR>
__global__ void __launch_bounds__(kWfMaxBlock, sizeof(R) == 4 ? 7 : 0) k_wf_vertex_adj(const __grid_constant__ DevScene<R> S, const WfRay<R> *rays_in, const WfCounters *C,
                                int which, WfPath<R> *paths, R *nee, WfAdj<R> A)
{
    __shared__ float adj_g[kAdjMaxParams];
    const AdjCtx ctx = make_adj_ctx(adj_g, S.material_count);
    adj_block_begin(adj_g, A.P);
    const int n = C->ray_count[which];
    const int stride = gridDim.x * blockDim.x;
    // every lane of a warp takes the same iterations: vertex_adjoint sums
    // across the warp
    const int n_round = (n + stride - 1) / stride * stride;
    const V3<R> zero = v3(R(0), R(0), R(0));
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n_round; q += stride) {
        AdjVertex<R> pv = {};
        pv.mat = -1;
        int slot = 0;
        uint32_t seed_key = 0;
        V3<R> remaining = zero, adj = zero;
        if (q < n) {
            slot = rays_in[q].slot;
            WfPath<R> *sp = paths + slot;
            V3<R> radiance = v3(sp->radiance[0], sp->radiance[1], sp->radiance[2]);
            gather_nee(S, nee + (size_t)slot * kNeeSlots * 3, &radiance);
            sp->radiance[0] = radiance.x;
            sp->radiance[1] = radiance.y;
            sp->radiance[2] = radiance.z;
            pv = A.verts[slot];
            seed_key = sp->seed_key;
            const R *Lq = A.L + 3 * (size_t)slot;
            remaining = sub(v3(Lq[0], Lq[1], Lq[2]), radiance);
            adj = adj_of_path(A.P, slot);
        }
        vertex_adjoint<R, PBR, true>(S, pv, A.att + (size_t)slot * kNeeSlots * kAttStride, seed_key, remaining, adj,
                                     ctx, pv.mat >= 0);
    }
    adj_block_end(adj_g, A.P);
}

// Adjoint replay: the vertex each path still holds (its last) takes its
// gradient terms against the radiance the path ends with. PBR as in k_wf_shade.
// Paths whose last vertex is pending are gathered first, chunk by chunk of
// 8 x blockDim paths, into a list in shared memory (warp-aggregated appends),
// so the gradient code runs on full warps instead of on the scattered lanes
// of a grid-stride loop over every path (paths that escaped hold none).
// Held to 7 blocks per SM like k_wf_vertex_adj (backward 46.8 -> 46.5 ms).
static constexpr int kFinalizeChunkPerThread = 8;
template <typename R, bool PBR>
__global__ void __launch_bounds__(kWfMaxBlock, sizeof(R) == 4 ? 7 : 0) k_wf_finalize_adj(const __grid_constant__ DevScene<R> S, int n_paths, const WfPath<R> *paths, R *nee, WfAdj<R> A)
{
    __shared__ float adj_g[kAdjMaxParams];
    __shared__ int pending[kFinalizeChunkPerThread * kWfMaxBlock];
    __shared__ int n_pending;
    const AdjCtx ctx = make_adj_ctx(adj_g, S.material_count);
    adj_block_begin(adj_g, A.P);
    const int chunk = kFinalizeChunkPerThread * (int)blockDim.x;
    for (long long base = (long long)blockIdx.x * chunk; base < n_paths; base += (long long)gridDim.x * chunk) {
        if (threadIdx.x == 0) n_pending = 0;
        __syncthreads();
        // every lane runs the same iterations (chunk is a multiple of the
        // block, the block of the warp), so each append sees the whole warp
        for (int i = threadIdx.x; i < chunk; i += blockDim.x) {
            const long long q = base + i;
            const bool want = q < n_paths && A.verts[q].mat >= 0;
            const int at = warp_append(&n_pending, want);
            if (want) pending[at] = (int)q;
        }
        __syncthreads();
        const int np = n_pending;
        // every lane of the block takes the same iterations (vertex_adjoint
        // sums across the warp); lanes past the list take part inactive
        const int np_round = (np + (int)blockDim.x - 1) / (int)blockDim.x * (int)blockDim.x;
        const V3<R> zero = v3(R(0), R(0), R(0));
        for (int i = threadIdx.x; i < np_round; i += blockDim.x) {
            AdjVertex<R> pv = {};
            pv.mat = -1;
            int q = 0;
            uint32_t seed_key = 0;
            V3<R> remaining = zero, adj = zero;
            if (i < np) {
                q = pending[i];
                pv = A.verts[q];
                const WfPath<R> st = paths[q];
                V3<R> radiance = v3(st.radiance[0], st.radiance[1], st.radiance[2]);
                gather_nee(S, nee + (size_t)q * kNeeSlots * 3, &radiance);
                seed_key = st.seed_key;
                const R *Lq = A.L + 3 * (size_t)q;
                remaining = sub(v3(Lq[0], Lq[1], Lq[2]), radiance);
                adj = adj_of_path(A.P, q);
            }
            vertex_adjoint<R, PBR, true>(S, pv, A.att + (size_t)q * kNeeSlots * kAttStride, seed_key, remaining,
                                         adj, ctx, i < np);
        }
        __syncthreads();  // the list is rebuilt for the next chunk
    }
    adj_block_end(adj_g, A.P);
}

// Per pixel: each of its batch_spp paths finalised (finalize_path) and summed
// in sample order, without a round trip through a per-sample buffer.
template <typename R>
__global__ void k_wf_reduce(const __grid_constant__ DevScene<R> S, const WfParams<R> *P, int batch_spp, int first_batch,
                            int last_batch, R *acc, const WfPath<R> *paths, R *nee)
{
    const WfParams<R> p = *P;
    for (int pix = blockIdx.x * blockDim.x + threadIdx.x; pix < p.wh; pix += gridDim.x * blockDim.x) {
        V3<R> a = v3(R(0), R(0), R(0));
        if (!first_batch) a = v3(acc[3 * (size_t)pix], acc[3 * (size_t)pix + 1], acc[3 * (size_t)pix + 2]);
        for (int j = 0; j < batch_spp; ++j) a = add(a, finalize_path(S, paths, nee, (size_t)j * p.wh + pix));
        if (!last_batch) {
            acc[3 * (size_t)pix] = a.x;
            acc[3 * (size_t)pix + 1] = a.y;
            acc[3 * (size_t)pix + 2] = a.z;
            continue;
        }
        size_t o = 3 * (size_t)pix;
        if (p.out_kind == OUT_RGB8) {
            V3<R> mean = scale(a, R(1) / R(p.spp_window));
            unsigned char *op = (unsigned char *)p.out + o;
            op[0] = to_byte(mean.x);
            op[1] = to_byte(mean.y);
            op[2] = to_byte(mean.z);
        } else if (p.out_kind == OUT_MEAN_F32) {
            V3<R> mean = scale(a, R(1) / R(p.spp_window));
            float *op = (float *)p.out + o;
            op[0] = (float)mean.x;
            op[1] = (float)mean.y;
            op[2] = (float)mean.z;
        } else if (p.out_kind == OUT_SUM_F32) {
            float *op = (float *)p.out + o;
            op[0] = (float)a.x;
            op[1] = (float)a.y;
            op[2] = (float)a.z;
        } else {
            float *op = (float *)p.out + o;
            op[0] += (float)a.x;
            op[1] += (float)a.y;
            op[2] += (float)a.z;
        }
    }
}

}  // namespace mt
