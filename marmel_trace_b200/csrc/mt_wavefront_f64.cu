// mt_wavefront_f64.cu - FP64 instantiation of the wavefront integrator
// (compiled with --fmad=false like the FP64 megakernel).
#include "mt_wavefront_host.cuh"

namespace mt {

int wavefront_render(WavefrontState *&st, const DevScene<double> &S, const DevCamera<double> &cam, int w, int h,
                     int s0, int s1, int depth, int out_kind, void *out, cudaStream_t stream, const mt_options *opts,
                     cudaEvent_t ev0, cudaEvent_t ev1, int32_t *launches)
{
    return wavefront_render_impl<double>(st, S, cam, w, h, s0, s1, depth, out_kind, out, stream, opts, ev0, ev1,
                                         launches);
}

int wavefront_adjoint(WavefrontState *&st, const DevScene<double> &S, const DevCamera<double> &cam, int w, int h,
                      int s0, int s1, int depth, const WfAdjointCall &a, cudaStream_t stream, const mt_options *opts)
{
    return wavefront_render_impl<double>(st, S, cam, w, h, s0, s1, depth, OUT_SUM_F32, nullptr, stream, opts,
                                         nullptr, nullptr, nullptr, &a);
}

}  // namespace mt
