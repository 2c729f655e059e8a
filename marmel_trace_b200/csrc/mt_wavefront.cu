// mt_wavefront.cu - FP32 instantiation of the wavefront integrator and its
// type-independent host helpers.
#include "mt_wavefront_host.cuh"

namespace mt {

int wavefront_render(WavefrontState *&st, const DevScene<float> &S, const DevCamera<float> &cam, int w, int h,
                     int s0, int s1, int depth, int out_kind, void *out, cudaStream_t stream, const mt_options *opts,
                     cudaEvent_t ev0, cudaEvent_t ev1, int32_t *launches)
{
    return wavefront_render_impl<float>(st, S, cam, w, h, s0, s1, depth, out_kind, out, stream, opts, ev0, ev1,
                                        launches);
}

int wavefront_adjoint(WavefrontState *&st, const DevScene<float> &S, const DevCamera<float> &cam, int w, int h,
                      int s0, int s1, int depth, const WfAdjointCall &a, cudaStream_t stream, const mt_options *opts)
{
    return wavefront_render_impl<float>(st, S, cam, w, h, s0, s1, depth, OUT_SUM_F32, nullptr, stream, opts, nullptr,
                                        nullptr, nullptr, &a);
}

void wavefront_stage_times(const WavefrontState *st, double ms[4], long long launches[4])
{
    for (int i = 0; i < 4; ++i) {
        ms[i] = st ? st->kernel_ms[i] : 0.0;
        launches[i] = st ? st->kernel_launches[i] : 0;
    }
}

void wavefront_reset_stage_times(WavefrontState *st)
{
    if (!st) return;
    for (int i = 0; i < 4; ++i) {
        st->kernel_ms[i] = 0.0;
        st->kernel_launches[i] = 0;
    }
}

void wavefront_destroy(WavefrontState *st)
{
    if (!st) return;
    wf_free(st);
    if (st->h_params) cudaFreeHost(st->h_params);
    if (st->cap_stream) cudaStreamDestroy(st->cap_stream);
    if (st->kev_init)
        for (int i = 0; i < 64; ++i) cudaEventDestroy(st->kev[i]);
    delete st;
}

const char *wavefront_last_error() { return wfdetail::last_error().c_str(); }

}  // namespace mt
