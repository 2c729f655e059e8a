// mt_adjoint_f64.cu - FP64 instantiation of the path-replay adjoint
// (compiled with --fmad=false like the other FP64 units).
#include "mt_adjoint_launch.cuh"

namespace mt {
template cudaError_t launch_adjoint<double>(const DevScene<double> &, const DevCamera<double> &, int, int, int, int,
                                            int, const float *, double, double *, int, cudaStream_t);
}
