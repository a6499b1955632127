// Host-side launchers of the loop kernels (kernels_impl.cuh), instantiated for
// double (kernels.cu, --fmad=false) and float (kernels_f32.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>

#include "case.cuh"

namespace ctbfm {

// Device array of tiles for one kernel family.
struct TileList {
    const Tile* tiles = nullptr;
    int n = 0;
};

// Tile lists of the split stage (k_prim, k_faces, k_nodes) for one set of
// members.
struct SplitLists {
    TileList node;  // nodes (k_prim, k_nodes)
    // faces per direction, scheme (0 JST, 1 Roe) and face set: 0 every face
    // of the direction; for K lines of at least 3 nodes, and J lines of at
    // least 3 nodes whose rows of nk faces do not fall on whole warps, 1 the
    // faces two or more faces from both ends of each line (plain interior
    // stencils) and 2 the four faces at the ends (boundary and next-to-
    // boundary stencils), so that no warp mixes the two code paths
    TileList face[3][2][3];
};

// Everything a batched launch needs: the instances' descriptions on the
// device and the tile lists of each kernel family.
template <typename R>
struct BatchView {
    const DevCaseT<R>* cases = nullptr;  // m device-resident instance descriptions
    int m = 0;
    bool ideal = true;  // some member uses the ideal gas
    bool real = false;  // some member uses the real-gas look-up tables
    bool bfmCommon = true;  // some member uses no BFM or Hall / Hall-Thollet / Lift-Drag / blockage
    bool bfmRare = false;   // some member uses the Chima or Correlations body force
    TileList node;        // nodes of every instance (k_dt)
    // stage kernels: fusedMode 0 runs every member through the split stage
    // (split[0]); fusedMode 1 runs the members that can (fuse_ok) through the
    // fused stage kernel k_stage (one tile per box of nodes, by scheme, in
    // fbox) and the others through the split stage (split[1])
    int fusedMode = 0;
    SplitLists split[2];
    TileList fbox[2];
    size_t fusedSmem = 0;  // dynamic shared memory of a k_stage block (largest member box)
    TileList per;         // periodic (i, j) pairs of periodic instances
    bool viscous = false;  // some member is viscous (VISCOSITY_ACTIVE)
    TileList vnode;        // nodes of the viscous instances (k_grad)
    TileList vface[3];     // every face of each swept direction of the viscous instances (k_vfaces)
    bool sa = false;       // some member runs the Spalart-Allmaras model
    TileList sanode;       // nodes of the SA instances (k_prim, k_grad, k_sa_prep, k_sa_res, k_sa_update)
    TileList sainst;       // one tile per SA instance (k_sa_bc, k_sa_sweep)
    TileList inst;        // one tile per instance (k_pre, k_finalize)
    TileList bint;        // 8 plane tiles per instance that needs turbo performance
    TileList bintAll;     // 8 plane tiles for every instance
};

template <typename R>
struct Launcher {
    static cudaError_t setLimits(const BatchView<R>& b, long long n, cudaStream_t s);
    // copies the m control blocks into out[0..m) (device memory)
    static cudaError_t gatherControl(const BatchView<R>& b, Control* out, cudaStream_t s);
    static cudaError_t boundaryIntegrals(const BatchView<R>& b, bool all, int force, cudaStream_t s);
    static cudaError_t timeStep(const BatchView<R>& b, int force, cudaStream_t s);
    static cudaError_t pre(const BatchView<R>& b, bool forceTurbo, bool dtpart, bool profiles, int force,
                           cudaStream_t s);
    static cudaError_t prim(const BatchView<R>& b, int stage, int force, cudaStream_t s);
    static cudaError_t faces(const BatchView<R>& b, int dir, int stage, int force, cudaStream_t s);
    // k_grad and k_vfaces of the viscous members
    static cudaError_t viscous(const BatchView<R>& b, int stage, int force, cudaStream_t s);
    static cudaError_t nodes(const BatchView<R>& b, int stage, int force, cudaStream_t s);
    static cudaError_t periodic(const BatchView<R>& b, int stage, int force, cudaStream_t s);
    // TurbulenceModelSA::solve of the SA members, once per iteration before
    // the stages: primitives and solution gradient of U^n, boundary values,
    // nu hat gradient, residual, the two sweeps, update, boundary values
    static cudaError_t turbulence(const BatchView<R>& b, cudaStream_t s);
    // k_stage over the fused members' boxes (fusedMode 1)
    static cudaError_t fused(const BatchView<R>& b, int stage, int force, cudaStream_t s);
    // dynamic shared memory of a k_stage block of an instance with box
    // (bi, bj, bk) in topology topo and scheme (0 JST, 1 Roe)
    static size_t fusedSmemBytes(int bi, int bj, int bk, int topo, int scheme);
    static cudaError_t finalize(const BatchView<R>& b, int force, cudaStream_t s);
    // k_prim, k_faces, (k_grad, k_vfaces), k_nodes, k_stage, k_periodic of one
    // stage (stage -1: residual only)
    static cudaError_t stage(const BatchView<R>& b, int stage, int force, cudaStream_t s);
    // one whole iteration of every instance in the batch
    static cudaError_t iteration(const BatchView<R>& b, int nstages, cudaStream_t s);
};

extern template struct Launcher<double>;
extern template struct Launcher<float>;

// State of the persistent kernel's grid barrier (device memory, zeroed when
// allocated; every launch leaves count at 0).
struct GridSync {
    unsigned count;  // blocks arrived at the current barrier
    unsigned gen;    // barrier generation
    int error;       // 1: a barrier wait ran out and the kernel stopped
    int active[2];   // instances still running after a finalize phase (alternate iterations)
    int pad;
};

// The persistent iteration kernel k_run (persist.cuh): one cooperative
// launch runs whole iterations of a batch, its phases (time step, pre-stage,
// and per stage faces, nodes, periodic planes, then finalize) separated by a
// grid barrier instead of kernel boundaries. For batches of ideal-gas,
// inviscid members without the SA model and with one advection scheme.
template <typename R>
struct Persistent {
    // n iterations (fewer if every member stops); scheme 0 JST, 1 Roe
    static cudaError_t run(const BatchView<R>& b, int scheme, int nstages, long long n, GridSync* gs,
                           cudaStream_t s);
    // `reps` forced stage-0 evaluations, as the autotuner times the other
    // stage kernels
    static cudaError_t tuneStage(const BatchView<R>& b, int scheme, int reps, GridSync* gs, cudaStream_t s);
    // blocks of one launch for this batch (co-resident blocks, at most the
    // largest phase's tiles)
    static int gridBlocks(const BatchView<R>& b, int scheme);
};

extern template struct Persistent<double>;
extern template struct Persistent<float>;

constexpr int kKernelKinds = 11;
constexpr int kTileSize = 256;  // elements per tile (one per thread)
// fused stage kernel: nodes per box (one per thread) and the faces (all
// directions) a box may hold in shared memory
constexpr int kFusedBoxNodes = 256;
constexpr int kFusedFaceCap = 1024;
// periodic (i, j) pairs per tile, one block of as many threads each: the
// periodic planes hold few pairs with much work each (7 680 on the bench
// workload: 120 blocks instead of 30)
constexpr int kPeriodicTile = 64;

// Static device scratch of ctbfm_compute_residual_noalloc (noalloc.cu): its
// device address on device dev, which must be current (looked up once per
// device), and its size.
constexpr size_t kNoAllocScratchBytes = size_t(16) << 20;
cudaError_t noallocScratch(int dev, double** ptr, size_t* bytes);

}  // namespace ctbfm
