// FP32 instantiation of the persistent iteration kernel (persist.cuh), with
// the float compile flags of kernels_f32.cu.
#define CTBFM_COHERENT_LOADS 1
#include "kernels_impl.cuh"
#include "persist.cuh"

namespace ctbfm {
template struct Persistent<float>;
}  // namespace ctbfm
