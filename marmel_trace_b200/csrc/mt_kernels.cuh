// mt_kernels.cuh - the megakernel renderers and batched query kernels.
//
// Included by mt_kernels_f32.cu / mt_kernels_f64.cu, which instantiate the
// launchers for one arithmetic type each.
#pragma once

#include "mt_integrate.cuh"
#include "mt_launch.h"

namespace mt {

// One thread per pixel; the thread walks the pixel's samples in order and
// sums them exactly as pt_render_pixel / render_region do
// (src/pathtrace.c:1053-1095, src/render.c:929-966). The image is read in
// row-major order, so a warp covers 32 horizontally adjacent pixels whose
// primary rays are coherent.
// EXTRAS: the scene has fog, marched media, clouds or textures
// (DevScene::has_extras); without them those paths are compiled out.
template <typename R, int MODE, bool EXTRAS>
__global__ void __launch_bounds__(128) k_render(const __grid_constant__ DevScene<R> S, const DevCamera<R> cam, int w, int h,
                                                int spp_total, int s0, int s1, int depth, int out_kind, void *out)
{
    int pix = blockIdx.x * blockDim.x + threadIdx.x;
    if (pix >= w * h) return;
    int x = pix % w;
    int y = pix / w;
    V3<R> acc = v3(R(0), R(0), R(0));
    for (int s = s0; s < s1; ++s) {
        if (MODE == RENDER_PT) {
            Ray3<R> ray = pt_primary(S, cam, w, h, x, y, s);
            uint32_t seed_key = hash3((uint32_t)x, (uint32_t)y, (uint32_t)s);
            acc = add(acc, pathtrace_radiance<R, EXTRAS>(S, ray, depth, seed_key));
        } else {
            Ray3<R> ray = wh_primary(cam, w, h, spp_total, x, y, s);
            uint32_t seed_key = hash3((uint32_t)x, (uint32_t)y, (uint32_t)s);
            acc = add(acc, whitted_trace<R, EXTRAS>(S, ray, depth, seed_key));
        }
    }
    if (S.counters && s1 > s0) atomicAdd(&S.counters->primary_rays, (unsigned long long)(s1 - s0));
    size_t o = 3 * (size_t)pix;
    if (out_kind == OUT_RGB8) {
        V3<R> mean = scale(acc, R(1) / R(s1 - s0));
        unsigned char *p = (unsigned char *)out + o;
        p[0] = to_byte(mean.x);
        p[1] = to_byte(mean.y);
        p[2] = to_byte(mean.z);
    } else if (out_kind == OUT_MEAN_F32) {
        V3<R> mean = scale(acc, R(1) / R(s1 - s0));
        float *p = (float *)out + o;
        p[0] = (float)mean.x;
        p[1] = (float)mean.y;
        p[2] = (float)mean.z;
    } else if (out_kind == OUT_SUM_F32) {
        float *p = (float *)out + o;
        p[0] = (float)acc.x;
        p[1] = (float)acc.y;
        p[2] = (float)acc.z;
    } else {
        float *p = (float *)out + o;
        p[0] += (float)acc.x;
        p[1] += (float)acc.y;
        p[2] += (float)acc.z;
    }
}

template <typename R>
__global__ void k_intersect(const __grid_constant__ DevScene<R> S, int n, const double *o, const double *d, double tmin, double tmax,
                            int *prim, double *t, double *normal, int *front, int *mat)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    V3<R> ro = v3<R>((R)o[3 * i], (R)o[3 * i + 1], (R)o[3 * i + 2]);
    V3<R> rd = v3<R>((R)d[3 * i], (R)d[3 * i + 1], (R)d[3 * i + 2]);
    SurfaceHit<R> h;
    if (scene_intersect(S, ro, rd, (R)tmin, (R)tmax, &h)) {
        prim[i] = h.prim;
        if (t) t[i] = (double)h.t;
        if (normal) {
            normal[3 * i] = (double)h.normal.x;
            normal[3 * i + 1] = (double)h.normal.y;
            normal[3 * i + 2] = (double)h.normal.z;
        }
        if (front) front[i] = h.front_face;
        if (mat) mat[i] = h.material;
    } else {
        prim[i] = -1;
        if (t) t[i] = 0.0;
        if (front) front[i] = 0;
        if (mat) mat[i] = -1;
    }
}

template <typename R>
__global__ void k_occluded(const __grid_constant__ DevScene<R> S, int n, const double *o, const double *d, double tmin, double tmax,
                           int *occ)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    V3<R> ro = v3<R>((R)o[3 * i], (R)o[3 * i + 1], (R)o[3 * i + 2]);
    V3<R> rd = v3<R>((R)d[3 * i], (R)d[3 * i + 1], (R)d[3 * i + 2]);
    occ[i] = scene_occluded(S, ro, rd, (R)tmin, (R)tmax) ? 1 : 0;
}

template <typename R>
__global__ void k_radiance(const __grid_constant__ DevScene<R> S, int n, const double *o, const double *d, int depth,
                           const unsigned *seeds, double *out, int mode)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    Ray3<R> r;
    r.o = v3<R>((R)o[3 * i], (R)o[3 * i + 1], (R)o[3 * i + 2]);
    r.d = v3<R>((R)d[3 * i], (R)d[3 * i + 1], (R)d[3 * i + 2]);
    V3<R> L = mode == RENDER_PT ? pathtrace_radiance(S, r, depth, seeds[i]) : whitted_trace(S, r, depth, seeds[i]);
    out[3 * i] = (double)L.x;
    out[3 * i + 1] = (double)L.y;
    out[3 * i + 2] = (double)L.z;
}

template <typename R>
__global__ void k_primary(const __grid_constant__ DevScene<R> S, const DevCamera<R> cam, int w, int h, int spp, int mode, double *out)
{
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    long long n = (long long)w * h * spp;
    if (i >= n) return;
    int s = (int)(i % spp);
    long long pix = i / spp;
    int x = (int)(pix % w), y = (int)(pix / w);
    Ray3<R> r = mode == RENDER_PT ? pt_primary(S, cam, w, h, x, y, s) : wh_primary(cam, w, h, spp, x, y, s);
    double *p = out + 6 * i;
    p[0] = (double)r.o.x;
    p[1] = (double)r.o.y;
    p[2] = (double)r.o.z;
    p[3] = (double)r.d.x;
    p[4] = (double)r.d.y;
    p[5] = (double)r.d.z;
}

static inline int grid_for(long long n, int block) { return (int)((n + block - 1) / block); }

// Dynamic shared memory of a traversing kernel: one stack per thread.
template <typename R> static inline size_t stack_smem(const DevScene<R> &S, int block)
{
    return (size_t)(S.stack_depth > 0 ? S.stack_depth : 1) * block * sizeof(int);
}

template <typename R>
cudaError_t launch_render(const DevScene<R> &S, const DevCamera<R> &cam, int w, int h, int spp_total, int s0,
                          int s1, int depth, int mode, int out_kind, void *out, int block, cudaStream_t stream)
{
    if (block <= 0) block = 128;
    if (block > 128) block = 128;  // __launch_bounds__(128)
    long long n = (long long)w * h;
    const int g = grid_for(n, block);
    const size_t sm = stack_smem(S, block);
    if (mode == RENDER_PT && S.has_extras)
        k_render<R, RENDER_PT, true><<<g, block, sm, stream>>>(S, cam, w, h, spp_total, s0, s1, depth, out_kind, out);
    else if (mode == RENDER_PT)
        k_render<R, RENDER_PT, false><<<g, block, sm, stream>>>(S, cam, w, h, spp_total, s0, s1, depth, out_kind, out);
    else if (S.has_extras)
        k_render<R, RENDER_WHITTED, true><<<g, block, sm, stream>>>(S, cam, w, h, spp_total, s0, s1, depth, out_kind, out);
    else
        k_render<R, RENDER_WHITTED, false><<<g, block, sm, stream>>>(S, cam, w, h, spp_total, s0, s1, depth, out_kind, out);
    return cudaGetLastError();
}

template <typename R>
cudaError_t launch_intersect(const DevScene<R> &S, int n, const double *o, const double *d, double tmin, double tmax,
                             int *prim, double *t, double *normal, int *front, int *mat, cudaStream_t stream)
{
    k_intersect<R><<<grid_for(n, 128), 128, stack_smem(S, 128), stream>>>(S, n, o, d, tmin, tmax, prim, t, normal, front, mat);
    return cudaGetLastError();
}

template <typename R>
cudaError_t launch_occluded(const DevScene<R> &S, int n, const double *o, const double *d, double tmin, double tmax,
                            int *occ, cudaStream_t stream)
{
    k_occluded<R><<<grid_for(n, 128), 128, stack_smem(S, 128), stream>>>(S, n, o, d, tmin, tmax, occ);
    return cudaGetLastError();
}

template <typename R>
cudaError_t launch_radiance(const DevScene<R> &S, int n, const double *o, const double *d, int depth,
                            const unsigned *seeds, double *out, int mode, cudaStream_t stream)
{
    k_radiance<R><<<grid_for(n, 64), 64, stack_smem(S, 64), stream>>>(S, n, o, d, depth, seeds, out, mode);
    return cudaGetLastError();
}

template <typename R>
cudaError_t launch_primary(const DevScene<R> &S, const DevCamera<R> &cam, int w, int h, int spp, int mode,
                           double *out, cudaStream_t stream)
{
    long long n = (long long)w * h * spp;
    k_primary<R><<<grid_for(n, 128), 128, 0, stream>>>(S, cam, w, h, spp, mode, out);
    return cudaGetLastError();
}

// ------------------------------------------------------------------
// Adaptive Whitted refinement (render_image_adaptive, src/render.c:1128-1500).
// Per pixel: double sums of R, G, B, luminance Y and Y^2, and the sample count.
// Pass 0 takes samples 0..n0-1 of every pixel; each later pass takes up to
// `batch` more samples of the pixels the active-set kernel flagged. Sample
// index s is global per pixel, so a pixel's k-th sample is the same ray in
// any pass, and each pass sums its samples serially before folding them in,
// as adaptive_region does.
// ------------------------------------------------------------------

// adaptive_sample_offset (src/render.c:1156-1165): the fixed path's offsets
// for s < n0, uniform jitter beyond; lens channels 2s+2 / 2s+3.
template <typename R>
MT_D Ray3<R> adaptive_primary(const DevCamera<R> &cam, int w, int h, int n0, int x, int y, int s)
{
    if (s < n0) return wh_primary(cam, w, h, n0, x, y, s);
    R du = rand01<R>((uint32_t)x, (uint32_t)y, (uint32_t)(s * 2 + 0));
    R dv = rand01<R>((uint32_t)x, (uint32_t)y, (uint32_t)(s * 2 + 1));
    R uu = (R(x) + du) / R(w);
    R vv = R(1) - (R(y) + dv) / R(h);
    R lr1 = rand01<R>((uint32_t)x, (uint32_t)y, (uint32_t)(s * 2 + 2));
    R lr2 = rand01<R>((uint32_t)x, (uint32_t)y, (uint32_t)(s * 2 + 3));
    return camera_ray_dof(cam, uu, vv, lr1, lr2);
}

// One pass (adaptive_region, src/render.c:1174-1240). `list` holds the active
// pixels (count on the device); NULL means every pixel (pass 0).
template <typename R, bool EXTRAS>
__global__ void __launch_bounds__(128) k_adaptive_pass(const __grid_constant__ DevScene<R> S, const DevCamera<R> cam, int w, int h,
                                                       int n0, int nmax, int batch, int depth, const int *list,
                                                       const int *count, double *sums, int *nsamp)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int n_active = list ? *count : w * h;
    if (i >= n_active) return;
    const int p = list ? list[i] : i;
    const int x = p % w, y = p / w;
    const int n = nsamp[p];
    int b = batch;
    if (b > nmax - n) b = nmax - n;
    if (b <= 0) return;
    double sr = 0.0, sg = 0.0, sb = 0.0, sy = 0.0, sy2 = 0.0;
    for (int k = 0; k < b; ++k) {
        const int s = n + k;
        Ray3<R> ray = adaptive_primary(cam, w, h, n0, x, y, s);
        uint32_t seed_key = hash3((uint32_t)x, (uint32_t)y, (uint32_t)s);
        V3<R> c = whitted_trace<R, EXTRAS>(S, ray, depth, seed_key);
        const double cx = (double)c.x, cy = (double)c.y, cz = (double)c.z;
        sr += cx;
        sg += cy;
        sb += cz;
        const double Y = 0.2126 * cx + 0.7152 * cy + 0.0722 * cz;
        sy += Y;
        sy2 += Y * Y;
    }
    double *q = sums + 5 * (size_t)p;
    q[0] += sr;
    q[1] += sg;
    q[2] += sb;
    q[3] += sy;
    q[4] += sy2;
    nsamp[p] = n + b;
    if (S.counters) atomicAdd(&S.counters->primary_rays, (unsigned long long)b);
}

// adaptive_compute_active (src/render.c:1330-1363): refine while the relative
// standard error of the mean luminance exceeds tau and n < nmax. Flagged
// pixels are appended to `list`; *count is their number.
template <int Unused = 0>
__global__ void k_adaptive_active(int wh, int nmax, double tau, const double *sums, const int *nsamp, int *list,
                                  int *count)
{
    const int stride = gridDim.x * blockDim.x;
    const int n_round = (wh + stride - 1) / stride * stride;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n_round; p += stride) {
        bool flag = false;
        if (p < wh) {
            const int n = nsamp[p];
            if (n < nmax) {
                if (n < 2) {
                    flag = true;
                } else {
                    const double nf = (double)n;
                    const double *q = sums + 5 * (size_t)p;
                    const double ybar = q[3] / nf;
                    double var = (q[4] - q[3] * ybar) / (nf - 1.0);
                    if (var < 0.0) var = 0.0;
                    const double se = sqrt(var / nf);
                    const double e = se / (ybar + 1e-4);
                    flag = e > tau;
                }
            }
        }
        const unsigned m = __ballot_sync(0xffffffffu, flag);
        int base = 0;
        const int lane = threadIdx.x & 31;
        if (m && lane == __ffs(m) - 1) base = atomicAdd(count, __popc(m));
        base = __shfl_sync(0xffffffffu, base, __ffs(m ? m : 1u) - 1);
        if (flag) list[base + __popc(m & ((1u << lane) - 1u))] = p;
    }
}

// adaptive_resolve (src/render.c:1365-1375): mean, then quantise once.
template <int Unused = 0>
__global__ void k_adaptive_resolve(int wh, const double *sums, const int *nsamp, unsigned char *rgb)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= wh) return;
    const double inv = 1.0 / (double)nsamp[p];
    const double *q = sums + 5 * (size_t)p;
    rgb[3 * (size_t)p] = to_byte<double>(q[0] * inv);
    rgb[3 * (size_t)p + 1] = to_byte<double>(q[1] * inv);
    rgb[3 * (size_t)p + 2] = to_byte<double>(q[2] * inv);
}

template <typename R>
cudaError_t launch_adaptive_pass(const DevScene<R> &S, const DevCamera<R> &cam, int w, int h, int n0, int nmax,
                                 int batch, int depth, const int *list, const int *count, double *sums, int *nsamp,
                                 cudaStream_t stream)
{
    long long n = (long long)w * h;
    if (S.has_extras)
        k_adaptive_pass<R, true><<<grid_for(n, 128), 128, stack_smem(S, 128), stream>>>(S, cam, w, h, n0, nmax, batch,
                                                                                        depth, list, count, sums, nsamp);
    else
        k_adaptive_pass<R, false><<<grid_for(n, 128), 128, stack_smem(S, 128), stream>>>(S, cam, w, h, n0, nmax, batch,
                                                                                         depth, list, count, sums, nsamp);
    return cudaGetLastError();
}

#define MT_INSTANTIATE(R)                                                                                        \
    template cudaError_t launch_adaptive_pass<R>(const DevScene<R> &, const DevCamera<R> &, int, int, int, int,   \
                                                 int, int, const int *, const int *, double *, int *,            \
                                                 cudaStream_t);                                                   \
    template cudaError_t launch_render<R>(const DevScene<R> &, const DevCamera<R> &, int, int, int, int, int, int, \
                                          int, int, void *, int, cudaStream_t);                                  \
    template cudaError_t launch_intersect<R>(const DevScene<R> &, int, const double *, const double *, double,    \
                                             double, int *, double *, double *, int *, int *, cudaStream_t);      \
    template cudaError_t launch_occluded<R>(const DevScene<R> &, int, const double *, const double *, double,     \
                                            double, int *, cudaStream_t);                                         \
    template cudaError_t launch_radiance<R>(const DevScene<R> &, int, const double *, const double *, int,        \
                                            const unsigned *, double *, int, cudaStream_t);                       \
    template cudaError_t launch_primary<R>(const DevScene<R> &, const DevCamera<R> &, int, int, int, int,         \
                                           double *, cudaStream_t);

}  // namespace mt
