// mt_launch.h - host-side launchers of the device kernels.
//
// Each launcher is a template defined in mt_kernels.cuh and explicitly
// instantiated once per arithmetic type: float in mt_kernels_f32.cu (FMA
// contraction on) and double in mt_kernels_f64.cu (--fmad=false, so every
// double add and multiply rounds as in the reference's C build).
#pragma once

#include <cuda_runtime.h>

#include "mt_layout.h"

namespace mt {

// Output forms of the per-pixel render kernels.
enum : int {
    OUT_RGB8 = 0,       // mean -> to_byte, top-down RGB8
    OUT_MEAN_F32 = 1,   // mean as float RGB
    OUT_SUM_F32 = 2,    // window sum as float RGB (overwrite)
    OUT_ADD_F32 = 3,    // window sum added to the float RGB buffer
};

enum : int { RENDER_PT = 0, RENDER_WHITTED = 1 };

template <typename R>
cudaError_t launch_render(const DevScene<R> &S, const DevCamera<R> &cam, int w, int h, int spp_total, int s0,
                          int s1, int depth, int mode, int out_kind, void *out, int block, cudaStream_t stream);

template <typename R>
cudaError_t launch_intersect(const DevScene<R> &S, int n, const double *o, const double *d, double tmin, double tmax,
                             int *prim, double *t, double *normal, int *front, int *mat, cudaStream_t stream);

template <typename R>
cudaError_t launch_occluded(const DevScene<R> &S, int n, const double *o, const double *d, double tmin, double tmax,
                            int *occ, cudaStream_t stream);

template <typename R>
cudaError_t launch_radiance(const DevScene<R> &S, int n, const double *o, const double *d, int depth,
                            const unsigned *seeds, double *out, int mode, cudaStream_t stream);

template <typename R>
cudaError_t launch_primary(const DevScene<R> &S, const DevCamera<R> &cam, int w, int h, int spp, int mode,
                           double *out, cudaStream_t stream);

// Adaptive Whitted refinement (render_image_adaptive, src/render.c:1128-1500):
// one pass over the active pixels (list == NULL: every pixel), the active-set
// update and the final resolve. sums: 5 doubles per pixel (R, G, B, Y, Y^2).
template <typename R>
cudaError_t launch_adaptive_pass(const DevScene<R> &S, const DevCamera<R> &cam, int w, int h, int n0, int nmax,
                                 int batch, int depth, const int *list, const int *count, double *sums, int *nsamp,
                                 cudaStream_t stream);
cudaError_t launch_adaptive_active(int wh, int nmax, double tau, const double *sums, const int *nsamp, int *list,
                                   int *count, cudaStream_t stream);
cudaError_t launch_adaptive_resolve(int wh, const double *sums, const int *nsamp, unsigned char *rgb,
                                    cudaStream_t stream);

// Path-replay adjoint over samples [s0, s1): grad += adj_scale * sum over
// pixels and samples of adj_img[pixel] . dL_sample/dtheta (mt_adjoint.cuh).
template <typename R>
cudaError_t launch_adjoint(const DevScene<R> &S, const DevCamera<R> &cam, int w, int h, int s0, int s1, int depth,
                           const float *adj_img, double adj_scale, double *grad, int n_params, cudaStream_t stream);

}  // namespace mt
