// mt_adjoint_launch.cuh - launcher of the adjoint kernel (one arithmetic type
// per translation unit: mt_adjoint.cu FP32, mt_adjoint_f64.cu FP64).
#pragma once

#include "mt_adjoint.cuh"
#include "mt_launch.h"

namespace mt {

template <typename R>
cudaError_t launch_adjoint(const DevScene<R> &S, const DevCamera<R> &cam, int w, int h, int s0, int s1, int depth,
                           const float *adj_img, double adj_scale, double *grad, int n_params, cudaStream_t stream)
{
    const int block = 128;
    long long n = (long long)w * h;
    size_t smem = (size_t)(S.stack_depth > 0 ? S.stack_depth : 1) * block * sizeof(int);
    k_adjoint<R><<<(int)((n + block - 1) / block), block, smem, stream>>>(S, cam, w, h, s0, s1, depth, adj_img,
                                                                          adj_scale, grad, n_params);
    return cudaGetLastError();
}

}  // namespace mt
