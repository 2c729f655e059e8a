// mt_kernels_f64.cu - FP64 instantiation of the device kernels (the exact-
// parity path; compiled with --fmad=false so double arithmetic rounds as the
// reference's C build does).
#include "mt_kernels.cuh"

namespace mt {
MT_INSTANTIATE(double)
}
