// mt_kernels_f32.cu - FP32 instantiation of the device kernels (the
// production path; compiled with FMA contraction).
#include "mt_kernels.cuh"

namespace mt {
MT_INSTANTIATE(float)
}
