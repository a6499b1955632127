// FP32 instantiation of the loop kernels: fluxes, dissipation, limiters and
// body forces in float, the state in float plus a Kahan compensation term;
// norms, boundary integrals, profiles and the plenum stay in double.
#include "kernels_impl.cuh"

namespace ctbfm {
template struct Launcher<float>;
}  // namespace ctbfm
