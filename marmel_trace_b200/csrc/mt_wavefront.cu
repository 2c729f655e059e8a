// mt_wavefront.cu - wavefront integrator (placeholder until the stage kernels land).
#include "mt_wavefront.h"

namespace mt {

struct WavefrontState {
    int dummy;
};

template <typename R>
int wavefront_render(WavefrontState *&, const DevScene<R> &, const DevCamera<R> &, int, int, int, int, int, int,
                     void *, cudaStream_t, const mt_options *, cudaEvent_t, cudaEvent_t, int32_t *)
{
    return MT_ERR_UNSUPPORTED;
}

template int wavefront_render<float>(WavefrontState *&, const DevScene<float> &, const DevCamera<float> &, int, int,
                                     int, int, int, int, void *, cudaStream_t, const mt_options *, cudaEvent_t,
                                     cudaEvent_t, int32_t *);
template int wavefront_render<double>(WavefrontState *&, const DevScene<double> &, const DevCamera<double> &, int,
                                      int, int, int, int, int, void *, cudaStream_t, const mt_options *, cudaEvent_t,
                                      cudaEvent_t, int32_t *);

void wavefront_destroy(WavefrontState *st) { delete st; }
const char *wavefront_last_error() { return "wavefront integrator not built"; }

}  // namespace mt

int mt_render_image_adaptive(mt_scene *, const mt_camera *, int, int, const mt_render_params *, unsigned char *)
{
    return MT_ERR_UNSUPPORTED;
}
