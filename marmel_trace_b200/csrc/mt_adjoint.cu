// mt_adjoint.cu - FP32 instantiation of the path-replay adjoint.
#include "mt_adjoint_launch.cuh"

namespace mt {
template cudaError_t launch_adjoint<float>(const DevScene<float> &, const DevCamera<float> &, int, int, int, int, int,
                                           const float *, double, double *, int, cudaStream_t);
}
