// FP64 instantiation of the persistent iteration kernel (persist.cuh).
// Compiled with --fmad=false, as the split kernels of kernels.cu, so that
// every expression rounds the same way.
#define CTBFM_COHERENT_LOADS 1
#include "kernels_impl.cuh"
#include "persist.cuh"

namespace ctbfm {
template struct Persistent<double>;
}  // namespace ctbfm
