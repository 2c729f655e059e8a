// mt_wavefront.h - the wavefront path-tracing integrator (host interface).
#pragma once

#include <cuda_runtime.h>

#include "../../include/mtgpu.h"
#include "mt_layout.h"

struct mt_scene;

namespace mt {

struct WavefrontState;

// Arguments of the wavefront adjoint: dL/dimage (device, h x w x 3 floats),
// the factor applied to it (1 / samples for a mean image) and the float64
// gradient it accumulates into.
struct WfAdjointCall {
    const float *adj_img;
    double scale;
    double *grad;
    int n_params;
};

// Render samples [s0, s1) of every pixel with the wavefront integrator:
// per-bounce stage kernels over compacted path queues, the window captured in
// a CUDA graph (opts->use_graph > 0), launched without a graph (== 0), or
// launched kernel by kernel with CUDA-event timing per stage (< 0). Same
// output forms as the megakernel (OUT_* in mt_launch.h). One overload per
// arithmetic type (FP32 in mt_wavefront.cu, FP64 in mt_wavefront_f64.cu).
int wavefront_render(WavefrontState *&st, const DevScene<float> &S, const DevCamera<float> &cam, int w, int h,
                     int s0, int s1, int depth, int out_kind, void *out, cudaStream_t stream, const mt_options *opts,
                     cudaEvent_t ev0, cudaEvent_t ev1, int32_t *launches);
int wavefront_render(WavefrontState *&st, const DevScene<double> &S, const DevCamera<double> &cam, int w, int h,
                     int s0, int s1, int depth, int out_kind, void *out, cudaStream_t stream, const mt_options *opts,
                     cudaEvent_t ev0, cudaEvent_t ev1, int32_t *launches);

// Path-replay adjoint over samples [s0, s1) with the wavefront stages: per
// batch a primal pass records every sample's radiance, then a replay pass
// re-traces the same paths from their seeds and accumulates the gradient.
int wavefront_adjoint(WavefrontState *&st, const DevScene<float> &S, const DevCamera<float> &cam, int w, int h,
                      int s0, int s1, int depth, const WfAdjointCall &a, cudaStream_t stream, const mt_options *opts);
int wavefront_adjoint(WavefrontState *&st, const DevScene<double> &S, const DevCamera<double> &cam, int w, int h,
                      int s0, int s1, int depth, const WfAdjointCall &a, cudaStream_t stream, const mt_options *opts);

// Per-stage device time accumulated in profiling mode: extend, shade,
// shadow, other (generate / finalize / reduce); and launch counts.
void wavefront_stage_times(const WavefrontState *st, double ms[4], long long launches[4]);
void wavefront_reset_stage_times(WavefrontState *st);

void wavefront_destroy(WavefrontState *st);
const char *wavefront_last_error();

}  // namespace mt


