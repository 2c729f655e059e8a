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
template <typename R, int MODE>
__global__ void __launch_bounds__(128) k_render(const DevScene<R> S, const DevCamera<R> cam, int w, int h,
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
            acc = add(acc, pathtrace_radiance(S, ray, depth, seed_key));
        } else {
            Ray3<R> ray = wh_primary(cam, w, h, spp_total, x, y, s);
            uint32_t seed_key = hash3((uint32_t)x, (uint32_t)y, (uint32_t)s);
            acc = add(acc, whitted_trace(S, ray, depth, seed_key));
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
__global__ void k_intersect(const DevScene<R> S, int n, const double *o, const double *d, double tmin, double tmax,
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
__global__ void k_occluded(const DevScene<R> S, int n, const double *o, const double *d, double tmin, double tmax,
                           int *occ)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    V3<R> ro = v3<R>((R)o[3 * i], (R)o[3 * i + 1], (R)o[3 * i + 2]);
    V3<R> rd = v3<R>((R)d[3 * i], (R)d[3 * i + 1], (R)d[3 * i + 2]);
    occ[i] = scene_occluded(S, ro, rd, (R)tmin, (R)tmax) ? 1 : 0;
}

template <typename R>
__global__ void k_radiance(const DevScene<R> S, int n, const double *o, const double *d, int depth,
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
__global__ void k_primary(const DevScene<R> S, const DevCamera<R> cam, int w, int h, int spp, int mode, double *out)
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
    if (mode == RENDER_PT)
        k_render<R, RENDER_PT><<<grid_for(n, block), block, stack_smem(S, block), stream>>>(S, cam, w, h, spp_total, s0, s1, depth,
                                                                         out_kind, out);
    else
        k_render<R, RENDER_WHITTED><<<grid_for(n, block), block, stack_smem(S, block), stream>>>(S, cam, w, h, spp_total, s0, s1,
                                                                              depth, out_kind, out);
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

#define MT_INSTANTIATE(R)                                                                                        \
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
