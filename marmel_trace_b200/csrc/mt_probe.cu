// mt_probe.cu - measured L2 read bandwidth: the roof the traversal kernels
// meet first, since the tree and the triangles of the benchmark scene stay
// resident in the 126 MB L2.
//
// One launch reads a buffer that fits in L2 `reps` times through ld.global.cg
// (cached in L2 only, so L1 hits cannot inflate the figure), 16-byte loads,
// every thread of a persistent grid striding over the whole buffer. Each pass
// starts at another offset, so an SM meets other lines than in its previous
// pass. The launch lasts long enough (hundreds of microseconds) that launch
// latency does not enter the figure, which a short copy of a small buffer
// would be bound by.
#include <cuda_runtime.h>

#include <cstdio>

#include "mtgpu.h"

void mt_set_last_error_text(const char *msg);

namespace {

__global__ void k_l2_read(const float4 *__restrict__ buf, size_t n4, int reps, float *sink)
{
    float acc = 0.0f;
    const size_t tid = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const size_t nt = (size_t)gridDim.x * blockDim.x;
    for (int r = 0; r < reps; ++r) {
        const size_t off = ((size_t)r * 8191u * 64u) % n4;  // < n4
        for (size_t i = tid; i < n4; i += nt) {
            size_t j = i + off;
            if (j >= n4) j -= n4;
            const float4 v = __ldcg(buf + j);
            acc += (v.x + v.y) + (v.z + v.w);
        }
    }
    if (acc == -1.0f) *sink = acc;  // the buffer holds zeros: keeps the loads, never stores
}

int fail(int code, const char *what, cudaError_t e)
{
    static thread_local char msg[256];
    std::snprintf(msg, sizeof msg, "%s: %s", what, cudaGetErrorString(e));
    mt_set_last_error_text(msg);
    return code;
}

}  // namespace

extern "C" int mt_measure_l2_read_gbs(int device, size_t bytes, int reps, double *gbs)
{
    if (!gbs) return MT_ERR_NULL;
    if (bytes < (1u << 20) || bytes > ((size_t)96 << 20) || bytes % 16 || reps < 1) {
        mt_set_last_error_text("mt_measure_l2_read_gbs: bytes must be a multiple of 16 in [1 MiB, 96 MiB], reps >= 1");
        return MT_ERR_INVALID;
    }
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return fail(MT_ERR_NO_DEVICE, "cudaSetDevice", e);
    int sms = 0;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device)) != cudaSuccess)
        return fail(MT_ERR_NO_DEVICE, "cudaDeviceGetAttribute", e);
    float4 *buf = nullptr;
    float *sink = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int rc = MT_OK;
    const size_t n4 = bytes / 16;
    const int block = 512, grid = 4 * sms;  // 2048 threads per SM
    float best_ms = 0.0f;
    if ((e = cudaMalloc(&buf, bytes)) != cudaSuccess || (e = cudaMalloc(&sink, sizeof(float))) != cudaSuccess) {
        rc = fail(MT_ERR_OOM, "cudaMalloc", e);
        goto done;
    }
    if ((e = cudaMemset(buf, 0, bytes)) != cudaSuccess || (e = cudaEventCreate(&e0)) != cudaSuccess ||
        (e = cudaEventCreate(&e1)) != cudaSuccess) {
        rc = fail(MT_ERR_LAUNCH, "set-up", e);
        goto done;
    }
    // one warm-up launch brings the buffer into L2, then the best of three
    for (int k = 0; k < 4; ++k) {
        cudaEventRecord(e0, 0);
        k_l2_read<<<grid, block>>>(buf, n4, reps, sink);
        cudaEventRecord(e1, 0);
        if ((e = cudaEventSynchronize(e1)) != cudaSuccess) {
            rc = fail(MT_ERR_LAUNCH, "k_l2_read", e);
            goto done;
        }
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (k > 0 && (best_ms == 0.0f || ms < best_ms)) best_ms = ms;
    }
    *gbs = (double)bytes * reps / (best_ms * 1e-3) / 1e9;
done:
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaFree(buf);
    cudaFree(sink);
    return rc;
}
