// mt_kernels_f64.cu - FP64 instantiation of the device kernels (the exact-
// parity path; compiled with --fmad=false so double arithmetic rounds as the
// reference's C build does).
#include "mt_kernels.cuh"

namespace mt {
MT_INSTANTIATE(double)

// Type-independent adaptive kernels: here, so their double arithmetic rounds
// as the reference's (no FMA contraction).
cudaError_t launch_adaptive_active(int wh, int nmax, double tau, const double *sums, const int *nsamp, int *list,
                                   int *count, cudaStream_t stream)
{
    int blocks = grid_for(wh, 256);
    if (blocks > 4096) blocks = 4096;
    k_adaptive_active<><<<blocks, 256, 0, stream>>>(wh, nmax, tau, sums, nsamp, list, count);
    return cudaGetLastError();
}

cudaError_t launch_adaptive_resolve(int wh, const double *sums, const int *nsamp, unsigned char *rgb,
                                    cudaStream_t stream)
{
    k_adaptive_resolve<><<<grid_for(wh, 256), 256, 0, stream>>>(wh, sums, nsamp, rgb);
    return cudaGetLastError();
}
}
