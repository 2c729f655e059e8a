// mt_wavefront.h - the wavefront path-tracing integrator (host interface).
#pragma once

#include <cuda_runtime.h>

#include "../../include/mtgpu.h"
#include "mt_layout.h"

struct mt_scene;

namespace mt {

struct WavefrontState;

// Render samples [s0, s1) of every pixel with the wavefront integrator:
// per-bounce stage kernels over compacted path queues. Same output forms as
// the megakernel (OUT_* in mt_launch.h). Returns 0 or an MT_ERR_* code.
template <typename R>
int wavefront_render(WavefrontState *&st, const DevScene<R> &S, const DevCamera<R> &cam, int w, int h, int s0,
                     int s1, int depth, int out_kind, void *out, cudaStream_t stream, const mt_options *opts,
                     cudaEvent_t ev0, cudaEvent_t ev1, int32_t *launches);

void wavefront_destroy(WavefrontState *st);
const char *wavefront_last_error();

}  // namespace mt

// Adaptive Whitted refinement (render_image_adaptive, src/render.c:1128-1500).
int mt_render_image_adaptive(mt_scene *sc, const mt_camera *cam, int w, int h, const mt_render_params *p,
                             unsigned char *rgb);
