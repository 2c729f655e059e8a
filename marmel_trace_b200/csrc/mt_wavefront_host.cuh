// mt_wavefront_host.cuh - host driver of the wavefront integrator (one
// arithmetic type per translation unit).
//
// The whole sample window [s0, s1) of a frame is captured once into a CUDA
// graph: for every batch, generate -> (extend, shade, shadow) x (depth + 1)
// -> finalize -> reduce, plus the queue-counter resets. Values that change
// from call to call (camera, window start, output pointer) are read by the
// kernels from a device-side parameter block that is refreshed by one
// asynchronous copy before each graph launch, so a graph is re-captured only
// when the frame's shape changes (size, batch split, depth).
#pragma once

#include <limits.h>

#include <string.h>

#include <string>

#include "mt_wavefront.cuh"
#include "mt_wavefront.h"

namespace mt {

struct WavefrontState {
    int elem = 0;              // sizeof(R) of the buffers below
    size_t cap_paths = 0;      // path slots allocated
    int light_count = -1;
    void *paths = nullptr, *rays[2] = {nullptr, nullptr}, *hits = nullptr, *nee = nullptr, *shadow = nullptr;
    void *sample_buf = nullptr, *acc = nullptr, *params = nullptr;
    WfCounters *counters = nullptr;
    size_t acc_pixels = 0;
    void *h_params = nullptr;  // pinned host copy of the parameter block
    cudaStream_t cap_stream = nullptr;
    cudaGraphExec_t exec = nullptr;
    std::string key;
    // adjoint replay: pending vertex and NEE transmittance per path slot, and
    // the graph of the primal + replay window
    void *adj_verts = nullptr, *adj_att = nullptr;
    cudaGraphExec_t adj_exec = nullptr;
    std::string adj_key;
    // sort by material: sorted copies of a bounce's rays and hits, keys, and
    // bucket counts + cursors (2 x buckets ints)
    void *sorted_rays = nullptr, *sorted_hits = nullptr, *sort_keys = nullptr, *sort_buckets = nullptr;
    int sort_bucket_cap = 0;
    int grid_block = 0;        // block size the persistent grid was sized for
    // occluder cache (occ_entry): per pixel and NEE slot for bounce 0, then a
    // hash of (origin cell, NEE slot); only for a state that serves one scene
    // (a batch lane renders several, so it turns this off)
    void *occ_cache = nullptr;
    bool occ_cache_on = true;
    // scenes with pass-through materials use the cache (cache pass with the
    // pass tree) only when asked for (mt_options.occluder_cache = 1)
    bool pass_cache_on = false;
    // the NEE slots hold zeros between windows: they are zeroed at
    // allocation, and every slot a shadow connection writes is gathered (and
    // zeroed) by the next shade or by finalize; a state whose buffers are
    // carved from shared memory of changing layout leaves this false and has
    // k_wf_generate zero them
    bool nee_clean = false;
    void *walk = nullptr;      // shadow rays left to walk after the occluder-cache pass
    // link queues of pass-through chains (wf_reserve_links), `link_cap`
    // records of WfLink<R> each; NULL: chains run whole in k_wf_shadow
    void *link[2] = {nullptr, nullptr};
    int link_cap = 0;
    int grid = 0;              // persistent grid (blocks) of the stage kernels
    cudaEvent_t kev[64];       // per-kernel timing events (profiling mode)
    bool kev_init = false;
    double kernel_ms[4] = {0, 0, 0, 0};  // extend, shade, shadow, other (profiling mode)
    long long kernel_launches[4] = {0, 0, 0, 0};
};

namespace wfdetail {
inline std::string &last_error()
{
    static thread_local std::string e;
    return e;
}
inline int fail(int code, const char *what, cudaError_t e)
{
    last_error() = std::string(what) + ": " + cudaGetErrorString(e);
    return code;
}
}  // namespace wfdetail

#define WF_CK(call, what)                                                                               \
    do {                                                                                                \
        cudaError_t e_ = (call);                                                                        \
        if (e_ != cudaSuccess)                                                                          \
            return wfdetail::fail(e_ == cudaErrorMemoryAllocation ? MT_ERR_OOM : MT_ERR_LAUNCH, what, e_); \
    } while (0)

inline void wf_free(WavefrontState *st)
{
    void **bufs[] = {&st->paths,       &st->rays[0],    &st->rays[1],     &st->hits,        &st->nee,
                     &st->shadow,      &st->sample_buf, &st->acc,         &st->params,      &st->adj_verts,
                     &st->adj_att,     &st->sorted_rays, &st->sorted_hits, &st->sort_keys, &st->sort_buckets,
                     &st->occ_cache,   &st->walk,       &st->link[0],     &st->link[1]};
    for (void **b : bufs) {
        if (*b) cudaFree(*b);
        *b = nullptr;
    }
    if (st->counters) cudaFree(st->counters);
    st->counters = nullptr;
    if (st->exec) cudaGraphExecDestroy(st->exec);
    st->exec = nullptr;
    st->key.clear();
    if (st->adj_exec) cudaGraphExecDestroy(st->adj_exec);
    st->adj_exec = nullptr;
    st->adj_key.clear();
    st->cap_paths = 0;
    st->acc_pixels = 0;
    st->sort_bucket_cap = 0;
    st->link_cap = 0;
    st->nee_clean = false;
}

// Batch size of a window of `spp` samples over `wh` pixels: the largest
// divisor of spp whose paths fit the queue capacity (default kDefaultQueuePaths,
// at least one sample of every pixel).
// Default path slots of a batch: 2^25 (about 25 GB of queues when a window
// fills them; a window allocates only pixels x batch spp). Larger batches
// leave fewer deep-bounce tails with a half-empty GPU: on the 1080p torus
// field a 16-spp frame takes 161 / 156 / 154 ms with 8 M / 16 M / 33 M slots.
static constexpr long long kDefaultQueuePaths = 1ll << 25;

inline void wf_batch_split(int wh, int spp, long long capacity, int *batch_spp, int *n_batches)
{
    long long cap = capacity > 0 ? capacity : kDefaultQueuePaths;
    if (cap < wh) cap = wh;
    *batch_spp = 1;
    for (int d = spp; d >= 1; --d)
        if (spp % d == 0 && (long long)wh * d <= cap) {
            *batch_spp = d;
            break;
        }
    *n_batches = spp / *batch_spp;
}

// the pinned host staging block of the parameters is 256 bytes
static_assert(sizeof(WfParams<double>) <= 256 && sizeof(WfParams<float>) <= 256, "parameter block size");

// Grow the buffers to hold `n_paths` path slots and `wh` pixels.
template <typename R> int wf_reserve(WavefrontState *st, size_t n_paths, size_t wh, int light_count)
{
    if (st->elem == (int)sizeof(R) && st->cap_paths >= n_paths && st->acc_pixels >= wh && st->light_count == light_count)
        return 0;
    wf_free(st);
    st->elem = sizeof(R);
    st->light_count = light_count;
    size_t nshadow = n_paths * (size_t)(light_count + 1);
    WF_CK(cudaMalloc(&st->paths, n_paths * sizeof(WfPath<R>)), "cudaMalloc(paths)");
    WF_CK(cudaMalloc(&st->rays[0], n_paths * sizeof(WfRay<R>)), "cudaMalloc(rays)");
    WF_CK(cudaMalloc(&st->rays[1], n_paths * sizeof(WfRay<R>)), "cudaMalloc(rays)");
    WF_CK(cudaMalloc(&st->hits, n_paths * sizeof(WfHit<R>)), "cudaMalloc(hits)");
    WF_CK(cudaMalloc(&st->nee, n_paths * kNeeSlots * 3 * sizeof(R)), "cudaMalloc(nee)");
    WF_CK(cudaMemset(st->nee, 0, n_paths * kNeeSlots * 3 * sizeof(R)), "cudaMemset(nee)");
    st->nee_clean = true;
    WF_CK(cudaMalloc(&st->shadow, (nshadow ? nshadow : 1) * sizeof(WfShadow<R>)), "cudaMalloc(shadow)");
    WF_CK(cudaMalloc(&st->acc, wh * 3 * sizeof(R)), "cudaMalloc(acc)");
    WF_CK(cudaMalloc(&st->params, sizeof(WfParams<R>)), "cudaMalloc(params)");
    WF_CK(cudaMalloc((void **)&st->counters, sizeof(WfCounters)), "cudaMalloc(counters)");
    WF_CK(cudaMalloc(&st->occ_cache, occ_cache_ints(wh) * sizeof(int)), "cudaMalloc(occluder cache)");
    WF_CK(cudaMemset(st->occ_cache, 0xFF, occ_cache_ints(wh) * sizeof(int)), "cudaMemset(occluder cache)");
    WF_CK(cudaMalloc(&st->walk, (nshadow ? nshadow : 1) * sizeof(int)), "cudaMalloc(shadow walk list)");
    if (!st->h_params) WF_CK(cudaMallocHost(&st->h_params, 256), "cudaMallocHost(params)");
    st->cap_paths = n_paths;
    st->acc_pixels = wh;
    return 0;
}

// Link queues of the pass-through chains (scenes with water or transparency
// > 0.8): two buffers, each for every shadow connection of the reserved path
// slots (a launch appends at most one record per connection). Optional: when
// the allocation fails the chains run whole in k_wf_shadow (same results).
template <typename R> void wf_reserve_links(WavefrontState *st)
{
    if (st->link[0] && st->link[1]) return;
    const size_t nshadow = st->cap_paths * (size_t)(st->light_count + 1);
    size_t cap = nshadow;
    if (cap < 1) cap = 1;
    if (cap > (size_t)INT_MAX) cap = (size_t)INT_MAX;
    for (int k = 0; k < 2; ++k)
        if (!st->link[k] && cudaMalloc(&st->link[k], cap * sizeof(WfLink<R>)) != cudaSuccess) st->link[k] = nullptr;
    if (!st->link[0] || !st->link[1]) {
        for (int k = 0; k < 2; ++k) {
            if (st->link[k]) cudaFree(st->link[k]);
            st->link[k] = nullptr;
        }
        cudaGetLastError();
        st->link_cap = 0;
        return;
    }
    st->link_cap = (int)cap;
}

// The adjoint replay's per-path buffers, sized to the reserved path slots.
template <typename R> int wf_reserve_adj(WavefrontState *st)
{
    // each buffer on its own, so that a failed allocation is retried next call
    // each sample's primal radiance (k_wf_finalize), the replay's target
    if (!st->sample_buf)
        WF_CK(cudaMalloc(&st->sample_buf, st->cap_paths * 3 * sizeof(R)), "cudaMalloc(samples)");
    if (!st->adj_verts)
        WF_CK(cudaMalloc(&st->adj_verts, st->cap_paths * sizeof(AdjVertex<R>)), "cudaMalloc(adjoint vertices)");
    if (!st->adj_att)
        WF_CK(cudaMalloc(&st->adj_att, st->cap_paths * kNeeSlots * kAttStride * sizeof(R)), "cudaMalloc(adjoint nee)");
    return 0;
}

// Traversal stage launches for the tree width W (2: binary nodes; 4 / 8: the
// wide tree, FP32 only). `smem` is the stack of that tree.
template <typename R, int W>
void launch_extend(bool dyn, int g, int block, size_t smem, cudaStream_t s, const DevScene<R> &S,
                   const WfRay<R> *rays, WfCounters *C, int which, WfHit<R> *hits)
{
    if (dyn)
        k_wf_extend_dyn<R, W><<<g, block, smem, s>>>(S, rays, C, which, hits);
    else
        k_wf_extend<R, W><<<g, block, smem, s>>>(S, rays, C, which, hits);
}

// Link queues of the pass-through chains (k_wf_shadow_link): two buffers of
// `cap` records, NULL when the state has none (the chain then runs whole in
// k_wf_shadow).
struct WfLinkQueues {
    void *q[2];
    int cap;
};

// Kernels of one shadow stage in a scene with pass-through materials and
// link queues: the first link, then one launch per further link up to
// kWfLinkLaunches, the last of which runs the chains left to their end.
#ifndef MT_LINK_LAUNCHES
#define MT_LINK_LAUNCHES 3
#endif
static constexpr int kWfLinkLaunches = MT_LINK_LAUNCHES;
static_assert(kWfLinkLaunches >= 1 && kWfLinkLaunches <= 5, "link launches");

template <typename R, bool ADJ, int W>
void launch_shadow(bool dyn, int g, int block, size_t smem, cudaStream_t s, const DevScene<R> &S,
                   const WfShadow<R> *sq, WfCounters *C, R *nee, R *att, int *occ, int wh, int b, int *walk,
                   const WfLinkQueues &lq)
{
    if (S.has_passthrough) {
        WfLink<R> *l0 = ADJ || !lq.cap ? nullptr : (WfLink<R> *)lq.q[0];
        const bool cached = !ADJ && occ && walk && S.pass_root != kNoPassTree;
        // cached opaque blockers first (with the pass tree), then the chain
        // for the rest
        if (cached) k_wf_shadow_pass_cache<R><<<g, block, smem, s>>>(S, sq, C, nee, occ, wh, b, walk);
        int *w = cached ? walk : nullptr;
        if constexpr (!ADJ) {
            if (l0) {
                k_wf_shadow<R, false, 2, true, true><<<g, block, smem, s>>>(S, sq, C, nee, att, occ, wh, b, w, l0,
                                                                            lq.cap);
                for (int step = 1; step <= kWfLinkLaunches; ++step) {
                    const WfLink<R> *in = (const WfLink<R> *)lq.q[(step - 1) & 1];
                    WfLink<R> *out = (WfLink<R> *)lq.q[step & 1];
                    if (step == kWfLinkLaunches)
                        k_wf_shadow_link<R, true><<<g, block, smem, s>>>(S, sq, C, nee, b, step, in, out, lq.cap);
                    else
                        k_wf_shadow_link<R, false><<<g, block, smem, s>>>(S, sq, C, nee, b, step, in, out, lq.cap);
                }
                return;
            }
        }
        k_wf_shadow<R, ADJ, 2, true><<<g, block, smem, s>>>(S, sq, C, nee, att, occ, wh, b, w, nullptr, 0);
    } else if (dyn) {
        k_wf_shadow_dyn<R, ADJ, W><<<g, block, smem, s>>>(S, sq, C, nee, att);
    } else if (occ && walk) {
        // cached occluders first, then the tree walk for the misses
        k_wf_shadow_cache<R, ADJ><<<g, block, 0, s>>>(S, sq, C, nee, att, occ, wh, b, walk);
        k_wf_shadow<R, ADJ, W, false><<<g, block, smem, s>>>(S, sq, C, nee, att, occ, wh, b, walk, nullptr, 0);
    } else {
        k_wf_shadow<R, ADJ, W, false><<<g, block, smem, s>>>(S, sq, C, nee, att, occ, wh, b, nullptr, nullptr, 0);
    }
}

template <typename R, bool ADJ>
void launch_shadow_w(int W, bool dyn, int g, int block, size_t smem, cudaStream_t s, const DevScene<R> &S,
                     const WfShadow<R> *sq, WfCounters *C, R *nee, R *att, int *occ, int wh, int b, int *walk,
                     const WfLinkQueues &lq)
{
    if constexpr (sizeof(R) == 4) {
        if (W == 4)
            return launch_shadow<R, ADJ, 4>(dyn, g, block, smem, s, S, sq, C, nee, att, occ, wh, b, walk, lq);
        if (W == 8)
            return launch_shadow<R, ADJ, 8>(dyn, g, block, smem, s, S, sq, C, nee, att, occ, wh, b, walk, lq);
    }
    launch_shadow<R, ADJ, 2>(dyn, g, block, smem, s, S, sq, C, nee, att, occ, wh, b, walk, lq);
}

template <typename R>
void launch_extend_w(int W, bool dyn, int g, int block, size_t smem, cudaStream_t s, const DevScene<R> &S,
                     const WfRay<R> *rays, WfCounters *C, int which, WfHit<R> *hits)
{
    if constexpr (sizeof(R) == 4) {
        if (W == 4) return launch_extend<R, 4>(dyn, g, block, smem, s, S, rays, C, which, hits);
        if (W == 8) return launch_extend<R, 8>(dyn, g, block, smem, s, S, rays, C, which, hits);
    }
    launch_extend<R, 2>(dyn, g, block, smem, s, S, rays, C, which, hits);
}

// Buffers of the sort-by-material stage for `buckets` keys.
template <typename R> int wf_reserve_sort(WavefrontState *st, int buckets)
{
    if (!st->sorted_rays) {
        WF_CK(cudaMalloc(&st->sorted_rays, st->cap_paths * sizeof(WfRay<R>)), "cudaMalloc(sorted rays)");
        WF_CK(cudaMalloc(&st->sorted_hits, st->cap_paths * sizeof(WfHit<R>)), "cudaMalloc(sorted hits)");
        WF_CK(cudaMalloc(&st->sort_keys, st->cap_paths * sizeof(int)), "cudaMalloc(sort keys)");
    }
    if (st->sort_bucket_cap < buckets) {
        if (st->sort_buckets) cudaFree(st->sort_buckets);
        st->sort_buckets = nullptr;
        WF_CK(cudaMalloc(&st->sort_buckets, 2 * (size_t)buckets * sizeof(int)), "cudaMalloc(sort buckets)");
        st->sort_bucket_cap = buckets;
    }
    return 0;
}

// Enqueue one frame window. In profiling mode (`prof`), every stage kernel is
// bracketed by CUDA events and its time is added to st->kernel_ms.
// `adjoint`: per batch, the primal pass leaves every sample's radiance in
// sample_buf, then the replay pass re-traces the same paths and accumulates
// the parameter gradient (no image is written).
//
// `dyn`: the extend stage, and the shadow stage of scenes without
// pass-through materials, use the dynamic-fetch traversal kernels.
//
// `params` (default: the state's own block) is the device parameter block the
// kernels read, so several windows can share one state's queues.
template <typename R>
int wf_enqueue(WavefrontState *st, const DevScene<R> &S, int w, int h, int batch_spp, int n_batches, int depth,
               cudaStream_t s, bool prof, int block, bool adjoint = false, bool dyn = false,
               const void *params = nullptr, int sort_threshold = 0)
{
    const int wh = w * h;
    const int n_paths = wh * batch_spp;
    WfPath<R> *paths = (WfPath<R> *)st->paths;
    WfRay<R> *rays[2] = {(WfRay<R> *)st->rays[0], (WfRay<R> *)st->rays[1]};
    WfHit<R> *hits = (WfHit<R> *)st->hits;
    R *nee = (R *)st->nee;
    WfShadow<R> *sq = (WfShadow<R> *)st->shadow;
    R *sample_buf = (R *)st->sample_buf;
    R *acc = (R *)st->acc;
    const WfParams<R> *P = (const WfParams<R> *)(params ? params : st->params);
    WfCounters *C = st->counters;
    const int g = st->grid;
    // tree width of the traversal stages; the pass-through shadow walk
    // (pt_occluded_segment) stays on the binary tree
    const int W = (sizeof(R) == 4 && S.wnodes) ? S.bvh_width : 2;
    const size_t smem = (size_t)(S.stack_depth > 0 ? S.stack_depth : 1) * block * sizeof(int);
    const size_t smem_w = W == 2 ? smem : (size_t)S.wide_stack_depth * block * sizeof(int);
    const int Ws = S.has_passthrough ? 2 : W;
    const size_t smem_s = Ws == 2 ? smem : smem_w;
    // marched media (fog or water with fog.shadow_steps > 0) cast shadow
    // segments from the shade stage: it then needs the binary-tree stack
    const size_t smem_shade = S.fog.shadow_steps > 0 ? smem : 0;
    int ev = 0;
    auto tic = [&]() {
        if (prof) cudaEventRecord(st->kev[ev & 63], s);
    };
    auto toc = [&](int kind) {
        if (!prof) return;
        cudaEventRecord(st->kev[(ev + 1) & 63], s);
        cudaEventSynchronize(st->kev[(ev + 1) & 63]);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, st->kev[ev & 63], st->kev[(ev + 1) & 63]);
        st->kernel_ms[kind] += ms;
        st->kernel_launches[kind] += 1;
        ev += 2;
    };
    int *occ = st->occ_cache_on && (!S.has_passthrough || st->pass_cache_on) ? (int *)st->occ_cache : nullptr;
    const WfLinkQueues lq{{st->link[0], st->link[1]}, st->link[0] && st->link[1] ? st->link_cap : 0};
    const WfAdj<R> none{nullptr, nullptr, nullptr, P};
    const WfAdj<R> A{(AdjVertex<R> *)st->adj_verts, (R *)st->adj_att, sample_buf, P};
    // generate -> (extend, shade, shadow) x (depth + 1); the replay pass uses
    // the ADJ stage kernels
    auto bounces = [&](int batch, bool replay) -> int {
        WF_CK(cudaMemsetAsync(C, 0, sizeof(WfCounters), s), "memset(counters)");
        tic();
        k_wf_generate<R><<<g, block, 0, s>>>(S, P, batch, batch_spp, n_paths, paths, rays[0], C, nee,
                                             replay ? A : none, replay || !st->nee_clean);
        toc(3);
        int which = 0;
        for (int b = 0; b <= depth; ++b) {
            tic();
            launch_extend_w<R>(W, dyn, g, block, smem_w, s, S, rays[which], C, which, hits);
            toc(0);
            WF_CK(cudaMemsetAsync(&C->ray_count[which ^ 1], 0, sizeof(int), s), "memset(ray_count)");
            // shadow_count, shadow_fetch, ray_fetch (the next extend's), sorted
            // and walk_count
            WF_CK(cudaMemsetAsync(&C->shadow_count, 0, kWfBounceCounters * sizeof(int), s), "memset(shadow_count)");
            const bool sort = sort_threshold > 0 && !replay && st->sorted_rays;
            if (sort) {
                const int nb = sort_buckets(S.material_count + 1);
                WF_CK(cudaMemsetAsync(st->sort_buckets, 0, 2 * (size_t)nb * sizeof(int), s), "memset(buckets)");
                tic();
                k_wf_sort_count<R><<<g, block, 0, s>>>(S, C, which, rays[which], hits, (int *)st->sort_keys,
                                                       (int *)st->sort_buckets, sort_threshold);
                k_wf_sort_scan<R><<<1, kSortScanThreads, 0, s>>>(C, (int *)st->sort_buckets, nb);
                k_wf_sort_scatter<R><<<g, block, 0, s>>>(C, which, rays[which], hits, (const int *)st->sort_keys,
                                                         (int *)st->sort_buckets, nb, (WfRay<R> *)st->sorted_rays,
                                                         (WfHit<R> *)st->sorted_hits);
                toc(3);
            }
            tic();
            if (replay) {
                // the adjoint rejects every scene extra
                if (b > 0) {
                    if (sizeof(R) == 4 && S.pbr_only)
                        k_wf_vertex_adj<R, sizeof(R) == 4><<<g, block, 0, s>>>(S, rays[which], C, which, paths, nee,
                                                                               A);
                    else
                        k_wf_vertex_adj<R, false><<<g, block, 0, s>>>(S, rays[which], C, which, paths, nee, A);
                }
                if (sizeof(R) == 4 && S.pbr_only)
                    k_wf_shade<R, true, false, sizeof(R) == 4><<<g, block, smem_shade, s>>>(
                        S, rays[which], hits, C, which, b, depth, paths, nee, rays[which ^ 1], sq, A, nullptr,
                        nullptr);
                else
                    k_wf_shade<R, true, false><<<g, block, smem_shade, s>>>(S, rays[which], hits, C, which, b,
                                                                            depth, paths, nee, rays[which ^ 1], sq, A,
                                                                            nullptr, nullptr);
            } else {
                const WfRay<R> *srays = sort ? (const WfRay<R> *)st->sorted_rays : nullptr;
                if (S.has_extras)
                    k_wf_shade<R, false, true><<<g, block, smem_shade, s>>>(S, rays[which], hits, C, which, b, depth,
                                                                            paths, nee, rays[which ^ 1], sq, none,
                                                                            srays, (const WfHit<R> *)st->sorted_hits);
                else if (sizeof(R) == 4 && S.pbr_only)
                    k_wf_shade<R, false, false, sizeof(R) == 4><<<g, block, smem_shade, s>>>(
                        S, rays[which], hits, C, which, b, depth, paths, nee, rays[which ^ 1], sq, none, srays,
                        (const WfHit<R> *)st->sorted_hits);
                else
                    k_wf_shade<R, false, false><<<g, block, smem_shade, s>>>(S, rays[which], hits, C, which, b, depth,
                                                                             paths, nee, rays[which ^ 1], sq, none,
                                                                             srays, (const WfHit<R> *)st->sorted_hits);
            }
            toc(1);
            tic();
            if (replay)
                launch_shadow_w<R, true>(Ws, dyn, g, block, smem_s, s, S, sq, C, nee, A.att, occ, wh, b,
                                         (int *)st->walk, lq);
            else
                launch_shadow_w<R, false>(Ws, dyn, g, block, smem_s, s, S, sq, C, nee, nullptr, occ, wh, b,
                                          (int *)st->walk, lq);
            toc(2);
            which ^= 1;
        }
        return 0;
    };
    for (int batch = 0; batch < n_batches; ++batch) {
        int rc = bounces(batch, false);
        if (rc) return rc;
        tic();
        if (adjoint) {
            k_wf_finalize<R><<<g, block, 0, s>>>(S, n_paths, paths, nee, sample_buf);
        } else {
            // one thread per pixel finalises its batch_spp paths and sums them
            k_wf_reduce<R><<<g, block, 0, s>>>(S, P, batch_spp, batch == 0, batch == n_batches - 1, acc, paths, nee);
        }
        toc(3);
        if (adjoint) {
            if ((rc = bounces(batch, true))) return rc;
            tic();
            if (sizeof(R) == 4 && S.pbr_only)
                k_wf_finalize_adj<R, sizeof(R) == 4><<<g, block, 0, s>>>(S, n_paths, paths, nee, A);
            else
                k_wf_finalize_adj<R, false><<<g, block, 0, s>>>(S, n_paths, paths, nee, A);
            toc(3);
        }
    }
    WF_CK(cudaGetLastError(), "wavefront launch");
    return 0;
}

template <typename R>
int wavefront_render_impl(WavefrontState *&st, const DevScene<R> &S, const DevCamera<R> &cam, int w, int h, int s0,
                          int s1, int depth, int out_kind, void *out, cudaStream_t stream, const mt_options *opts,
                          cudaEvent_t ev0, cudaEvent_t ev1, int32_t *launches, const WfAdjointCall *adj = nullptr)
{
    if (!st) st = new WavefrontState();
    const int wh = w * h;
    const int spp = s1 - s0;
    int batch_spp = 1, n_batches = 1;
    wf_batch_split(wh, spp, opts ? opts->queue_capacity : 0, &batch_spp, &n_batches);
    int rc = wf_reserve<R>(st, (size_t)wh * batch_spp, (size_t)wh, S.light_count);
    if (rc) return rc;
    const bool adjoint = adj != nullptr;
    if (adjoint && (rc = wf_reserve_adj<R>(st))) return rc;
    if (S.has_passthrough) wf_reserve_links<R>(st);
    const int block = (opts && opts->block_size == 64) ? 64 : 128;
    const int sort_threshold = (!adjoint && opts && opts->sort_threshold > 0) ? opts->sort_threshold : 0;
    if (sort_threshold && (rc = wf_reserve_sort<R>(st, sort_buckets(S.material_count + 1)))) return rc;
    if (!st->grid || st->grid_block != block) {
        st->grid_block = block;
        int dev = 0, sms = 0, per_sm = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_wf_extend<R, 2>, block,
                                                      (size_t)(S.stack_depth > 0 ? S.stack_depth : 1) * block * 4);
        if (per_sm < 1) per_sm = 1;
        st->grid = sms * per_sm;
    }
    // parameter block
    WfParams<R> hp;
    memset(&hp, 0, sizeof hp);
    hp.cam = cam;
    hp.out = out;
    hp.w = w;
    hp.h = h;
    hp.wh = wh;
    hp.s0 = s0;
    hp.spp_window = spp;
    hp.out_kind = out_kind;
    if (adjoint) {
        hp.adj_img = adj->adj_img;
        hp.grad = adj->grad;
        hp.adj_scale = adj->scale;
        hp.n_params = adj->n_params;
    }
    bool prof = opts && opts->use_graph < 0;   // profiling mode: no graph, per-kernel events
    bool use_graph = !prof && (!opts || opts->use_graph != 0);
    if (prof && !st->kev_init) {
        for (int i = 0; i < 64; ++i) cudaEventCreate(&st->kev[i]);
        st->kev_init = true;
    }
    if (ev0) WF_CK(cudaEventRecord(ev0, stream), "cudaEventRecord");
    // The parameter copy is ordered on `stream` before the graph / kernels.
    cudaStreamSynchronize(stream);  // the pinned block may still be in use by a previous copy
    memcpy(st->h_params, &hp, sizeof hp);
    WF_CK(cudaMemcpyAsync(st->params, st->h_params, sizeof hp, cudaMemcpyHostToDevice, stream), "params copy");
    // the occluder cache can be switched off per scene (mt_options.occluder_cache)
    st->occ_cache_on = !(opts && opts->occluder_cache < 0);
    st->pass_cache_on = opts && opts->occluder_cache > 0;
    // the bounce-0 shadow stage is two kernels when it uses the occluder cache
    // (scenes with pass-through materials: with the pass tree, outside the
    // adjoint's replay pass)
    const bool cache_on = st->occ_cache_on && st->occ_cache && st->walk;
    const int cache_pass = cache_on && !S.has_passthrough && !(opts && opts->traversal == MT_TRAVERSAL_DYNAMIC);
    const int pass_cache = cache_on && S.has_passthrough && st->pass_cache_on && S.pass_root != kNoPassTree;
    const int links = S.has_passthrough && st->link[0] && st->link[1] && st->link_cap ? kWfLinkLaunches : 0;
    const int cp = cache_pass + pass_cache + links;
    int kernels_per_window = adjoint ? n_batches * (((3 + cp) + (3 + cache_pass)) * (depth + 1) + 4)
                                     : n_batches * ((3 + cp + (sort_threshold ? 3 : 0)) * (depth + 1) + 3);
    cudaGraphExec_t &exec = adjoint ? st->adj_exec : st->exec;
    // dynamic fetch reorders rays across lanes: on coherent queues (primary
    // rays, NEE rays grouped by light) the grid-stride kernels are faster, so
    // they are the default and dynamic fetch is a tuning candidate
    const bool dyn = opts && opts->traversal == MT_TRAVERSAL_DYNAMIC;
    std::string &exec_key = adjoint ? st->adj_key : st->key;
    if (use_graph) {
        char key[256];
        // the scene travels by value in the captured kernel parameters, so
        // its identity, counters and parameter version are part of the key
        snprintf(key, sizeof key, "%d:%d:%d:%d:%d:%d:%p:%p:%d:%d:%d:%d:%d:%p:%d:%p", (int)sizeof(R), w, h, batch_spp,
                 n_batches, depth, (const void *)S.nodes, (const void *)S.counters, S.version, (int)dyn, block,
                 sort_threshold, S.bvh_width, (const void *)S.trace_rec,
                 (int)st->occ_cache_on + 2 * (int)st->pass_cache_on, st->link[0]);
        if (!exec || exec_key != key) {
            if (exec) cudaGraphExecDestroy(exec);
            exec = nullptr;
            if (!st->cap_stream) WF_CK(cudaStreamCreateWithFlags(&st->cap_stream, cudaStreamNonBlocking), "stream");
            WF_CK(cudaStreamBeginCapture(st->cap_stream, cudaStreamCaptureModeThreadLocal), "begin capture");
            int erc = wf_enqueue<R>(st, S, w, h, batch_spp, n_batches, depth, st->cap_stream, false, block, adjoint,
                                    dyn, nullptr, sort_threshold);
            cudaGraph_t graph = nullptr;
            cudaError_t ce = cudaStreamEndCapture(st->cap_stream, &graph);
            if (erc) {
                if (graph) cudaGraphDestroy(graph);
                return erc;
            }
            WF_CK(ce, "end capture");
            cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
            cudaGraphDestroy(graph);
            WF_CK(ie, "graph instantiate");
            exec_key = key;
        }
        WF_CK(cudaGraphLaunch(exec, stream), "graph launch");
    } else {
        rc = wf_enqueue<R>(st, S, w, h, batch_spp, n_batches, depth, stream, prof, block, adjoint, dyn, nullptr,
                           sort_threshold);
        if (rc) return rc;
    }
    if (ev1) WF_CK(cudaEventRecord(ev1, stream), "cudaEventRecord");
    if (launches) *launches = kernels_per_window;
    return 0;
}

}  // namespace mt
