// FP32 instantiation of the loop kernels: fluxes, dissipation, limiters and
// body forces in float, the state in float plus a Kahan compensation term;
// norms, boundary integrals, profiles, the plenum and real-gas table
// inversions stay in double. Compiled with multiply-add contraction and
// approximate float division and square root (build.py).
#include "kernels_impl.cuh"

namespace ctbfm {
template struct Launcher<float>;
}  // namespace ctbfm
