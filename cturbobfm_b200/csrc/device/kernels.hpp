// Host-side launchers of the FP64 loop kernels (kernels.cu).
#pragma once

#include <cuda_runtime.h>

#include "case.cuh"

namespace ctbfm {

// Five state / residual arrays passed by value to a kernel.
struct P5 {
    double* p[5];
};

int nodeBlocks(long long n);
int periodicBlocks(long long np);

cudaError_t launchBoundaryIntegrals(const DevCase& c, P5 Uin, bool turbo, cudaStream_t s);
cudaError_t launchTimeStep(const DevCase& c, P5 Uin, cudaStream_t s);
cudaError_t launchPre(const DevCase& c, P5 Uin, bool turbo, bool profiles, bool dtpart, cudaStream_t s);
cudaError_t launchSetLimits(const DevCase& c, long long itStop, long long histBase, cudaStream_t s);
// mode 0: Runge-Kutta stage update into Uout; mode 1: residual into Rout.
cudaError_t launchStage(const DevCase& c, P5 Uin, P5 Uout, double alpha, bool last, int mode, P5 Rout,
                        cudaStream_t s);
cudaError_t launchFinalize(const DevCase& c, cudaStream_t s);
// single kernels of a stage (profiling)
cudaError_t launchPrim(const DevCase& c, P5 Uin, cudaStream_t s);
cudaError_t launchFaces(const DevCase& c, int dir, P5 Uin, cudaStream_t s);
cudaError_t launchNodes(const DevCase& c, P5 Uin, P5 Uout, double alpha, bool last, int mode, P5 Rout, cudaStream_t s);
cudaError_t launchPeriodic(const DevCase& c, P5 Uout, double alpha, bool last, int mode, P5 Rout, cudaStream_t s);

constexpr int kKernelKinds = 10;

// Static device scratch of ctbfm_compute_residual_noalloc (noalloc.cu): its
// device address on the current device (looked up once per device) and size.
constexpr size_t kNoAllocScratchBytes = size_t(16) << 20;
cudaError_t noallocScratch(double** ptr, size_t* bytes);

}  // namespace ctbfm
