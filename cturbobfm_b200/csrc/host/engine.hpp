// Device-side engine: InstanceT<R> owns one operating point's device arrays
// (working precision R); GroupT<R> advances any set of instances together —
// it uploads their descriptions, builds the tile lists every kernel family
// launches over (a packed index of all instances' nodes, faces and planes) and
// captures CUDA graphs of whole iterations.
#pragma once

#include <cuda_runtime.h>

#include <stdexcept>
#include <string>
#include <vector>

#include "../device/case.cuh"
#include "../device/kernels.hpp"

namespace ctbfm {

class CudaError : public std::runtime_error {
public:
    using std::runtime_error::runtime_error;
};

inline void cudaCheck(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw CudaError(std::string(what) + ": " + cudaGetErrorString(e));
}

// Device memory of instances, groups and batches: a library-owned
// stream-ordered pool per device that keeps released blocks for reuse, so
// creating, promoting and releasing solves costs no driver mapping or
// unmapping. A block is ready when deviceAlloc returns; deviceFree first
// waits for the device's outstanding work (as cudaFree does), then returns
// the block to the pool.
void* deviceAlloc(size_t bytes);
void deviceFree(void* p) noexcept;
// bytes the current device's pool holds that no user holds (free for reuse)
size_t devicePoolIdle();
// Pinned host blocks (control-block copies), recycled by size class.
void* pinnedAlloc(size_t bytes);
void pinnedFree(void* p, size_t bytes) noexcept;

template <typename R>
class InstanceT {
public:
    InstanceT() = default;
    ~InstanceT();
    InstanceT(const InstanceT&) = delete;
    InstanceT& operator=(const InstanceT&) = delete;

    R* allocR(size_t n);
    double* allocD(size_t n);
    const R* uploadR(const std::vector<double>& v);
    const double* uploadD(const std::vector<double>& v);
    // Device arrays are carved (256-byte aligned) from a few large
    // allocations: the first of `reserve` bytes (when set before the first
    // array), each further one at least double the previous. One cudaMalloc
    // and one cudaFree per slab instead of one per array keeps creating and
    // promoting solves cheap.
    void reserve(size_t bytes) { hint_ = bytes; }
    void* allocBytes(size_t n);
    size_t deviceBytes() const { return bytes_; }
    size_t usedBytes() const { return used_; }

    DevCaseT<R> c{};  // host copy of the description, pointers into this instance's device arrays

private:
    std::vector<void*> allocs_;
    size_t bytes_ = 0;   // held: the slabs
    size_t used_ = 0;    // carved
    char* slab_ = nullptr;
    size_t slabUsed_ = 0, slabCap_ = 0;
    size_t hint_ = 0;
};

// What a group's autotuner chose (face tiles, stage fusion) and on how many
// nodes, so that a later group of similar size can adopt it instead of
// timing again.
struct GroupTuning {
    bool valid = false;
    int faceTile[3] = {kTileSize, kTileSize, kTileSize};
    int fusedMode = 0;
    bool persistent = false;
    float stageMs[3] = {0.f, 0.f, 0.f};
    long long nodes = 0;
};

template <typename R>
class GroupT {
public:
    explicit GroupT(std::vector<InstanceT<R>*> members);
    ~GroupT();
    GroupT(const GroupT&) = delete;
    GroupT& operator=(const GroupT&) = delete;

    // n iterations of every member (fewer for members that converge or
    // diverge), enqueued on s without host synchronisation.
    void enqueue(long long n, cudaStream_t s);
    const BatchView<R>& view() const { return view_; }
    int stages() const { return nstages_; }
    int size() const { return static_cast<int>(members_.size()); }
    // Re-uploads the members' descriptions (after a member's host copy
    // changed), ordered on stream s; allocates nothing.
    void refresh(cudaStream_t s);
    // Chooses the face-tile size per direction by timing (done once, at the
    // first enqueue of at least kTuneMinIterations iterations, when enabled).
    void tune(cudaStream_t s);
    void setAutotune(bool on) { autotune_ = on; }
    // Stage kernels: 0 the split stage for every member, 1 the fused stage
    // kernel for the members that can run it (the others split), 3 the
    // persistent iteration kernel k_run (split when the group cannot run it),
    // 2 chosen by the autotuner (until it has run: fused in float, split in
    // double, the faster ones on the workloads measured). FP64 results are
    // the same either way; the captured graphs are rebuilt.
    void setFusedMode(int mode);
    bool tuned() const { return tuned_; }
    int fusedMode() const { return view_.fusedMode; }
    // iterations run as k_run launches
    bool persistent() const { return persist_; }
    // every member can run in k_run: ideal gas, inviscid, no SA model, one
    // advection scheme
    bool persistentOk() const { return persistOk_; }
    int faceTile(int d) const { return faceTile_[d]; }
    // the autotuner's stage timings (ms per stage: split, fused, persistent;
    // 0 untimed)
    float stageMs(int mode) const { return stageMs_[mode]; }
    long long nodes() const;
    // the autotuner's choices (valid once this group's own autotuner has run)
    GroupTuning tuning() const;
    // takes another group's tuning (face tiles; stage fusion when this group
    // has GPU_STAGE_FUSION = auto) and marks this group tuned
    void adopt(const GroupTuning& t);
    static constexpr long long kTuneMinIterations = 64;

private:
    cudaGraphExec_t captureIterations(int iters);
    void buildTiles();

    std::vector<InstanceT<R>*> members_;
    int nstages_ = 0;
    DevCaseT<R>* dCases_ = nullptr;
    Tile* dTiles_ = nullptr;
    BatchView<R> view_;
    cudaStream_t captureStream_ = nullptr;
    cudaGraphExec_t graph_ = nullptr;   // graphIters_ iterations
    cudaGraphExec_t graph1_ = nullptr;  // one iteration
    int graphIters_ = 8;
    int faceTile_[3] = {kTileSize, kTileSize, kTileSize};
    float stageMs_[3] = {0.f, 0.f, 0.f};
    bool persistOk_ = false;
    bool persist_ = false;
    int scheme_ = 0;
    GridSync* dSync_ = nullptr;
    // iterations per k_run launch: keeps a launch short (a few to tens of
    // milliseconds), so that a cooperative launch waiting for room next to
    // another group's kernels never waits long
    static constexpr long long kRunIterations = 32;
    float timeStage(int mode, cudaStream_t s, cudaEvent_t e0, cudaEvent_t e1);
    bool tuned_ = false;
    bool autotune_ = true;
    bool fusionAuto_ = false;
    bool selfTuned_ = false;  // this group's own autotuner ran (not adopted)
};

extern template class InstanceT<double>;
extern template class InstanceT<float>;
extern template class GroupT<double>;
extern template class GroupT<float>;

}  // namespace ctbfm
