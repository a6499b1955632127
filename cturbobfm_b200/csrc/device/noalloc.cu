// Face-flux scratch for ctbfm_compute_residual_noalloc (include/ctbfm.h).
//
// Some callers cannot call cudaMalloc when they need a residual: processes
// whose device memory is owned up front by another allocator (a framework's
// caching allocator or a fixed pool reserved at start-up, so a fresh
// cudaMalloc can fail or fragment that pool), and control loops that must not
// block in the driver's allocator in the middle of a time step. For them the
// residual evaluation keeps its per-face flux contributions in the
// file-scope array below instead of in memory the solver allocates.
//
// Limits and sharing rules:
//   * the array holds kNoAllocScratchBytes (16 MiB), i.e. 5 words per face for
//     at most 419430 faces summed over the swept directions in FP64 and
//     838860 in fp32_kahan; larger cases are rejected;
//   * every GPU on which a solver is created holds the array until the
//     process exits: with lazy module loading (CUDA_MODULE_LOADING=LAZY, the
//     CUDA 12 default) the driver backs the array when its address is first
//     looked up, so the solver constructor does that look-up, and the
//     no-allocation entry point itself never triggers the reservation;
//   * all calls on a device share the one array, which keeps the last call's
//     contents; nothing in it has to start at zero, because each call writes
//     every slot it later reads;
//   * calls that overlap on the GPU (different streams, or different solvers
//     on the same device without ordering) race on the array.
//
// The array's name in host code is a host-side stand-in, not a device address:
// host code obtains the device address once per device with
// cudaGetSymbolAddress (with that device current) and passes it to the kernels.
// Creating a solver performs that set-up for the solver's device, before any
// stream capture the caller may start.

#include <cuda_runtime.h>

#include <mutex>

#include "kernels.hpp"

namespace ctbfm {

static __device__ __align__(256) double g_noallocScratch[kNoAllocScratchBytes / sizeof(double)];

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_scratchMutex;
double* g_scratchAddress[kMaxDevices] = {};
}  // namespace

cudaError_t noallocScratch(int dev, double** ptr, size_t* bytes) {
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    int cur = -1;
    cudaError_t e = cudaGetDevice(&cur);
    if (e != cudaSuccess) return e;
    if (cur != dev) return cudaErrorInvalidDevice;  // the look-up must run with dev current
    std::lock_guard<std::mutex> lock(g_scratchMutex);
    if (!g_scratchAddress[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noallocScratch);
        if (e != cudaSuccess) return e;
        g_scratchAddress[dev] = static_cast<double*>(p);
    }
    *ptr = g_scratchAddress[dev];
    *bytes = kNoAllocScratchBytes;
    return cudaSuccess;
}

}  // namespace ctbfm
