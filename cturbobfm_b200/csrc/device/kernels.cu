// FP64 instantiation of the loop kernels. Compiled with --fmad=false: no
// multiply-add contraction, so each expression rounds as the reference's does.
#include "kernels_impl.cuh"

namespace ctbfm {
template struct Launcher<double>;
}  // namespace ctbfm
