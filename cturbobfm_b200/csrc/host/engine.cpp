// Device-side engine: see engine.hpp.
#include "engine.hpp"

#include <cstdint>
#include <map>
#include <mutex>

#include <algorithm>

namespace ctbfm {

// ---------------------------------------------------------------- InstanceT

namespace {

constexpr int kMaxDevices = 64;
std::mutex gPoolMu;
cudaMemPool_t gPools[kMaxDevices] = {};

cudaMemPool_t poolOf(int dev) {
    if (dev < 0 || dev >= kMaxDevices) throw CudaError("device index out of range");
    std::lock_guard<std::mutex> lock(gPoolMu);
    if (!gPools[dev]) {
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        cudaMemPool_t pool = nullptr;
        cudaCheck(cudaMemPoolCreate(&pool, &props), "cudaMemPoolCreate");
        uint64_t keep = UINT64_MAX;  // released blocks stay in the pool
        cudaCheck(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep), "cudaMemPoolSetAttribute");
        gPools[dev] = pool;
    }
    return gPools[dev];
}

std::mutex gPinnedMu;
std::map<size_t, std::vector<void*>> gPinned;  // free pinned blocks by size class

size_t pinnedClass(size_t bytes) {
    size_t c = 256;
    while (c < bytes) c *= 2;
    return c;
}

}  // namespace

void* deviceAlloc(size_t bytes) {
    int dev = 0;
    cudaCheck(cudaGetDevice(&dev), "cudaGetDevice");
    void* p = nullptr;
    cudaMemPool_t pool = poolOf(dev);
    cudaError_t e = cudaMallocFromPoolAsync(&p, std::max<size_t>(bytes, 16), pool, cudaStreamLegacy);
    if (e == cudaErrorMemoryAllocation) {  // hand the pool's idle blocks back to the device and try again
        (void)cudaGetLastError();
        cudaCheck(cudaDeviceSynchronize(), "cudaDeviceSynchronize");
        cudaCheck(cudaMemPoolTrimTo(pool, 0), "cudaMemPoolTrimTo");
        e = cudaMallocFromPoolAsync(&p, std::max<size_t>(bytes, 16), pool, cudaStreamLegacy);
    }
    cudaCheck(e, "cudaMallocFromPoolAsync");
    cudaCheck(cudaStreamSynchronize(cudaStreamLegacy), "cudaStreamSynchronize");
    return p;
}

void deviceFree(void* p) noexcept {
    if (!p) return;
    cudaDeviceSynchronize();
    cudaFreeAsync(p, cudaStreamLegacy);
}

size_t devicePoolIdle() {
    int dev = 0;
    cudaCheck(cudaGetDevice(&dev), "cudaGetDevice");
    cudaMemPool_t pool = poolOf(dev);
    uint64_t reserved = 0, used = 0;
    cudaCheck(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &reserved), "cudaMemPoolGetAttribute");
    cudaCheck(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &used), "cudaMemPoolGetAttribute");
    return reserved > used ? static_cast<size_t>(reserved - used) : 0;
}

void* pinnedAlloc(size_t bytes) {
    const size_t c = pinnedClass(bytes);
    {
        std::lock_guard<std::mutex> lock(gPinnedMu);
        auto& v = gPinned[c];
        if (!v.empty()) {
            void* p = v.back();
            v.pop_back();
            return p;
        }
    }
    void* p = nullptr;
    cudaCheck(cudaMallocHost(&p, c), "cudaMallocHost");
    return p;
}

void pinnedFree(void* p, size_t bytes) noexcept {
    if (!p) return;
    try {
        std::lock_guard<std::mutex> lock(gPinnedMu);
        gPinned[pinnedClass(bytes)].push_back(p);
    } catch (...) {
        cudaFreeHost(p);
    }
}

template <typename R>
InstanceT<R>::~InstanceT() {
    for (void* p : allocs_) deviceFree(p);
}

template <typename R>
void* InstanceT<R>::allocBytes(size_t n) {
    const size_t a = (std::max<size_t>(n, 16) + 255) & ~size_t(255);
    if (!slab_ || slabUsed_ + a > slabCap_) {
        constexpr size_t kMinSlab = size_t(1) << 20;
        size_t cap = std::max(a, hint_ ? hint_ : kMinSlab);
        if (slab_) cap = std::max(cap, 2 * slabCap_);
        hint_ = 0;
        void* p = deviceAlloc(cap);
        allocs_.push_back(p);
        slab_ = static_cast<char*>(p);
        slabCap_ = cap;
        slabUsed_ = 0;
        bytes_ += cap;
    }
    void* p = slab_ + slabUsed_;
    slabUsed_ += a;
    used_ += a;
    return p;
}

template <typename R>
R* InstanceT<R>::allocR(size_t n) {
    return static_cast<R*>(allocBytes(n * sizeof(R)));
}

template <typename R>
double* InstanceT<R>::allocD(size_t n) {
    return static_cast<double*>(allocBytes(n * sizeof(double)));
}

template <typename R>
const R* InstanceT<R>::uploadR(const std::vector<double>& v) {
    R* d = allocR(v.size());
    if (sizeof(R) == sizeof(double)) {
        cudaCheck(cudaMemcpy(d, v.data(), v.size() * sizeof(double), cudaMemcpyHostToDevice), "cudaMemcpy");
    } else {
        std::vector<R> tmp(v.begin(), v.end());
        cudaCheck(cudaMemcpy(d, tmp.data(), tmp.size() * sizeof(R), cudaMemcpyHostToDevice), "cudaMemcpy");
    }
    return d;
}

template <typename R>
const double* InstanceT<R>::uploadD(const std::vector<double>& v) {
    double* d = allocD(v.size());
    cudaCheck(cudaMemcpy(d, v.data(), v.size() * sizeof(double), cudaMemcpyHostToDevice), "cudaMemcpy");
    return d;
}

// ------------------------------------------------------------------- GroupT

template <typename R>
GroupT<R>::GroupT(std::vector<InstanceT<R>*> members) : members_(std::move(members)) {
    if (members_.empty()) throw std::invalid_argument("empty group");
    // stage kernels run the largest stage count; members with fewer stages
    // skip the extra launches on the device
    nstages_ = 0;
    for (auto* m : members_) nstages_ = std::max(nstages_, m->c.nstages);
    const int M = static_cast<int>(members_.size());
    buildTiles();
    dCases_ = static_cast<DevCaseT<R>*>(deviceAlloc(M * sizeof(DevCaseT<R>)));
    view_.cases = dCases_;
    view_.m = M;
    view_.ideal = view_.real = false;
    for (auto* m : members_) (m->c.lut ? view_.real : view_.ideal) = true;
    view_.bfmCommon = view_.bfmRare = false;
    for (auto* m : members_) (bfmRareModel(m->c) ? view_.bfmRare : view_.bfmCommon) = true;
    view_.viscous = false;
    for (auto* m : members_) view_.viscous = view_.viscous || m->c.viscous;
    view_.sa = false;
    for (auto* m : members_) view_.sa = view_.sa || m->c.sa;
    view_.fusedMode = 1;
    scheme_ = members_[0]->c.scheme;
    persistOk_ = !view_.real && !view_.viscous && !view_.sa;
    for (auto* m : members_) persistOk_ = persistOk_ && m->c.scheme == scheme_;
    if (persistOk_) {
        dSync_ = static_cast<GridSync*>(deviceAlloc(sizeof(GridSync)));
        cudaCheck(cudaMemset(dSync_, 0, sizeof(GridSync)), "cudaMemset");
    }
    refresh(nullptr);
    cudaCheck(cudaStreamSynchronize(nullptr), "cudaStreamSynchronize");
    cudaCheck(cudaStreamCreateWithFlags(&captureStream_, cudaStreamNonBlocking), "cudaStreamCreate");
}

// Tile lists over the packed index of all members. Node tiles are kTileSize
// elements (the per-tile reduction partials depend on it); face tiles take the
// per-direction size the autotuner chose (any multiple of the block size: a
// block loops over its tile).
template <typename R>
void GroupT<R>::buildTiles() {
    const int M = static_cast<int>(members_.size());
    std::vector<Tile> node, snode[2], face[2][3][2][3], fbox[2], per, inst, bint, bintAll, vnode, vface[3], sanode,
        sainst;
    auto cover = [](std::vector<Tile>& out, int m, long long count, long long size) {
        int local = 0;
        for (long long s = 0; s < count; s += size) out.push_back({m, local++, s, std::min<long long>(size, count - s)});
        return local;
    };
    size_t smem = 0;
    for (int m = 0; m < M; m++) {
        const DevCaseT<R>& c = members_[m]->c;
        const int nt = cover(node, m, c.n, kTileSize);
        if (nt != c.node_tiles) throw std::logic_error("node tile count mismatch");
        // split-stage lists: [0] every member, [1] the members outside the
        // fused stage kernel
        for (int mode = 0; mode < 2; mode++) {
            if (mode == 1 && c.fuse_ok) continue;
            cover(snode[mode], m, c.n, kTileSize);
            for (int d = 0; d < (c.topo == 1 ? 3 : 2); d++) {
                const long long nf =
                    static_cast<long long>(c.ni + (d == 0)) * (c.nj + (d == 1)) * (c.nk + (d == 2));
                const int nline = d == 0 ? c.ni : (d == 1 ? c.nj : c.nk);  // nodes along a line of direction d
                // K lines (J lines whose rows of nk faces do not fill whole
                // warps, and the I lines of 2-D grids) run as two launches,
                // plain faces 2 .. n-2 and the four end faces of every line, so
                // the plain launch carries no boundary or extrapolation code; 3-D
                // I faces and warp-aligned J rows run as one launch (splitting
                // them measured slower: the four end planes of 3-D I make a large
                // launch of boundary code, 0.807 against 0.750 ms per iteration
                // on the 160 x 48 x 64 annulus; 2-D map batch 2 % faster split)
                const bool split = nline >= 3 && (d == 2 || (d == 1 && c.nk % 32 != 0) || (d == 0 && c.nk == 1));
                if (!split) {
                    cover(face[mode][d][c.scheme][0], m, nf, faceTile_[d]);
                } else {
                    const long long lines = d == 0 ? static_cast<long long>(c.nj) * c.nk
                                                   : (d == 1 ? static_cast<long long>(c.ni) * c.nk
                                                             : static_cast<long long>(c.ni) * c.nj);
                    cover(face[mode][d][c.scheme][1], m, lines * (nline - 3), faceTile_[d]);
                    // the end faces are few and carry the boundary code:
                    // one per thread, whatever the plain faces' tile
                    cover(face[mode][d][c.scheme][2], m, lines * 4, kTileSize);
                }
            }
        }
        if (c.fuse_ok) {  // one tile per box; Tile.local and Tile.start are the box index
            for (int bx = 0; bx < c.nboxes; bx++) fbox[c.scheme].push_back({m, bx, bx, 1});
            smem = std::max(smem, Launcher<R>::fusedSmemBytes(c.fbox[0], c.fbox[1], c.fbox[2], c.topo, c.scheme));
        }
        if (c.viscous) {
            cover(vnode, m, c.n, kTileSize);
            for (int d = 0; d < (c.topo == 1 ? 3 : 2); d++)
                cover(vface[d], m, static_cast<long long>(c.ni + (d == 0)) * (c.nj + (d == 1)) * (c.nk + (d == 2)),
                      kTileSize);
        }
        if (c.sa) {
            cover(sanode, m, c.n, kTileSize);
            sainst.push_back({m, 0, 0, 1});
        }
        if (c.periodic && cover(per, m, static_cast<long long>(c.ni) * c.nj, kPeriodicTile) != c.per_tiles)
            throw std::logic_error("periodic tile count mismatch");
        inst.push_back({m, 0, 0, 1});
        for (int b = 0; b < 8; b++)
            for (int k = c.bint_off[b]; k < c.bint_off[b + 1]; k++) {
                const Tile t{m, b, static_cast<long long>(k - c.bint_off[b]) * kBintChunk, kBintChunk};
                bintAll.push_back(t);
                if (c.need_turbo) bint.push_back(t);
            }
    }
    view_.fusedSmem = smem;
    std::vector<Tile> all;
    std::vector<std::pair<TileList*, size_t>> offs;
    auto add = [&](TileList& tl, const std::vector<Tile>& v) {
        offs.push_back({&tl, all.size()});
        tl.n = static_cast<int>(v.size());
        all.insert(all.end(), v.begin(), v.end());
    };
    add(view_.node, node);
    for (int mode = 0; mode < 2; mode++) {
        add(view_.split[mode].node, snode[mode]);
        for (int d = 0; d < 3; d++)
            for (int s = 0; s < 2; s++)
                for (int k = 0; k < 3; k++) add(view_.split[mode].face[d][s][k], face[mode][d][s][k]);
    }
    for (int s = 0; s < 2; s++) add(view_.fbox[s], fbox[s]);
    add(view_.per, per);
    add(view_.vnode, vnode);
    add(view_.sanode, sanode);
    add(view_.sainst, sainst);
    for (int d = 0; d < 3; d++) add(view_.vface[d], vface[d]);
    add(view_.inst, inst);
    add(view_.bint, bint);
    add(view_.bintAll, bintAll);
    deviceFree(dTiles_);
    dTiles_ = nullptr;
    dTiles_ = static_cast<Tile*>(deviceAlloc(std::max<size_t>(all.size(), 1) * sizeof(Tile)));
    cudaCheck(cudaMemcpy(dTiles_, all.data(), all.size() * sizeof(Tile), cudaMemcpyHostToDevice), "cudaMemcpy");
    // a copy from pageable memory may still be in flight when cudaMemcpy
    // returns, and the kernels run on non-blocking streams: wait for it (the
    // legacy default stream holds the copy and does not wait for the
    // non-blocking streams, so other groups' work on the device runs on)
    cudaCheck(cudaStreamSynchronize(cudaStreamLegacy), "cudaStreamSynchronize");
    for (auto& [tl, off] : offs) tl->tiles = dTiles_ + off;
    if (graph_) {  // launches captured with the old lists
        cudaGraphExecDestroy(graph_);
        graph_ = nullptr;
    }
    if (graph1_) {
        cudaGraphExecDestroy(graph1_);
        graph1_ = nullptr;
    }
}

// Autotuner of the face tiles: per direction, times the face kernels of the
// current state (stage 0, forced; they only rewrite the face contributions,
// which the next stage recomputes) with tiles of 256 to 2048 faces and keeps
// the fastest, a larger tile only when it is at least 2 % faster. Results do
// not depend on the tiling (every face is computed on its own).
template <typename R>
void GroupT<R>::tune(cudaStream_t s) {
    tuned_ = true;
    selfTuned_ = true;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaCheck(cudaEventCreate(&e0), "cudaEventCreate");
    cudaCheck(cudaEventCreate(&e1), "cudaEventCreate");
    const int sizes[] = {256, 512, 1024, 2048};
    const int mode = view_.fusedMode;
    view_.fusedMode = 0;  // the face tiles of every member
    for (int d = 0; d < 3; d++) {
        int nt = 0;
        for (int sc = 0; sc < 2; sc++)
            for (int k = 0; k < 3; k++) nt += view_.split[0].face[d][sc][k].n;
        if (!nt) continue;
        float best = 0.f;
        int bestSize = kTileSize;
        for (int sz : sizes) {
            faceTile_[d] = sz;
            buildTiles();
            cudaCheck(Launcher<R>::faces(view_, d, 0, 1, s), "launch k_faces (tuning)");
            cudaCheck(cudaEventRecord(e0, s), "cudaEventRecord");
            for (int r = 0; r < 3; r++) cudaCheck(Launcher<R>::faces(view_, d, 0, 1, s), "launch k_faces (tuning)");
            cudaCheck(cudaEventRecord(e1, s), "cudaEventRecord");
            cudaCheck(cudaEventSynchronize(e1), "cudaEventSynchronize");
            float ms = 0.f;
            cudaCheck(cudaEventElapsedTime(&ms, e0, e1), "cudaEventElapsedTime");
            if (sz == sizes[0] || ms < 0.98f * best) {
                best = ms;
                bestSize = sz;
            }
        }
        faceTile_[d] = bestSize;
    }
    view_.fusedMode = mode;
    buildTiles();
    // stage kernels: forced stage-0 evaluations (they rewrite only the first
    // stage buffer, the primitives and the periodic residuals, which the next
    // stage 0 recomputes) with the split stage, the fused stage kernel and
    // the persistent kernel, each as it runs; another than the split stage is
    // kept when at least 2 % faster than the best so far
    bool anyFused = false;
    for (auto* m : members_) anyFused = anyFused || m->c.fuse_ok;
    if (fusionAuto_ && (anyFused || persistOk_)) {
        stageMs_[0] = timeStage(0, s, e0, e1);
        stageMs_[1] = anyFused ? timeStage(1, s, e0, e1) : 0.f;
        stageMs_[2] = persistOk_ ? timeStage(2, s, e0, e1) : 0.f;
        int best = 0;
        float bestMs = stageMs_[0];
        if (anyFused && stageMs_[1] < 0.98f * bestMs) {
            best = 1;
            bestMs = stageMs_[1];
        }
        if (persistOk_ && stageMs_[2] < 0.98f * bestMs) best = 2;
        view_.fusedMode = best == 1 ? 1 : 0;
        persist_ = best == 2;
        if (graph_) {
            cudaGraphExecDestroy(graph_);
            graph_ = nullptr;
        }
        if (graph1_) {
            cudaGraphExecDestroy(graph1_);
            graph1_ = nullptr;
        }
    }
    // the iteration graphs of the chosen stage, captured now (capturing runs
    // nothing), so that no later enqueue pays for the capture
    if (!persist_) {
        if (!graph_) graph_ = captureIterations(graphIters_);
        if (!graph1_) graph1_ = captureIterations(1);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
}

// Time of one forced stage-0 evaluation in stage mode `mode` (0 split,
// 1 fused, 2 persistent) as it runs in the loop: the split and fused stages
// from a captured graph of `reps` evaluations, the persistent kernel as a
// k_run of `reps` evaluations; each timed after one untimed run.
template <typename R>
float GroupT<R>::timeStage(int mode, cudaStream_t s, cudaEvent_t e0, cudaEvent_t e1) {
    constexpr int reps = 4;
    struct ExecGuard {
        cudaGraphExec_t g = nullptr;
        ~ExecGuard() {
            if (g) cudaGraphExecDestroy(g);
        }
    } exec;
    view_.fusedMode = mode == 1 ? 1 : 0;
    if (mode < 2) {
        cudaGraph_t g = nullptr;
        cudaCheck(cudaStreamBeginCapture(captureStream_, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture");
        cudaError_t e = cudaSuccess;
        for (int r = 0; r < reps && e == cudaSuccess; r++) e = Launcher<R>::stage(view_, 0, 1, captureStream_);
        const cudaError_t e2 = cudaStreamEndCapture(captureStream_, &g);
        cudaCheck(e, "launch stage (tuning)");
        cudaCheck(e2, "cudaStreamEndCapture");
        const cudaError_t e3 = cudaGraphInstantiate(&exec.g, g, 0);
        cudaGraphDestroy(g);
        cudaCheck(e3, "cudaGraphInstantiate");
    }
    auto run = [&] {
        if (mode < 2) cudaCheck(cudaGraphLaunch(exec.g, s), "cudaGraphLaunch");
        else cudaCheck(Persistent<R>::tuneStage(view_, scheme_, reps, dSync_, s), "launch k_run (tuning)");
    };
    run();
    cudaCheck(cudaEventRecord(e0, s), "cudaEventRecord");
    run();
    cudaCheck(cudaEventRecord(e1, s), "cudaEventRecord");
    cudaCheck(cudaEventSynchronize(e1), "cudaEventSynchronize");
    float ms = 0.f;
    cudaCheck(cudaEventElapsedTime(&ms, e0, e1), "cudaEventElapsedTime");
    return ms / reps;
}

template <typename R>
long long GroupT<R>::nodes() const {
    long long n = 0;
    for (auto* m : members_) n += m->c.n;
    return n;
}

template <typename R>
GroupTuning GroupT<R>::tuning() const {
    GroupTuning t;
    t.valid = selfTuned_;
    for (int d = 0; d < 3; d++) t.faceTile[d] = faceTile_[d];
    t.fusedMode = view_.fusedMode;
    t.persistent = persist_;
    for (int k = 0; k < 3; k++) t.stageMs[k] = stageMs_[k];
    t.nodes = nodes();
    return t;
}

template <typename R>
void GroupT<R>::adopt(const GroupTuning& t) {
    if (!t.valid) return;
    for (int k = 0; k < 3; k++) stageMs_[k] = t.stageMs[k];
    bool same = true;
    for (int d = 0; d < 3; d++) same = same && faceTile_[d] == t.faceTile[d];
    for (int d = 0; d < 3; d++) faceTile_[d] = t.faceTile[d];
    if (!same) buildTiles();  // also drops captured graphs
    if (fusionAuto_) {
        view_.fusedMode = t.fusedMode;
        persist_ = t.persistent && persistOk_;
    }
    tuned_ = true;
}

template <typename R>
void GroupT<R>::setFusedMode(int mode) {
    fusionAuto_ = mode == 2;
    if (mode == 2) mode = sizeof(R) == sizeof(float) ? 1 : 0;  // until the autotuner has timed them
    persist_ = mode == 3 && persistOk_;
    const int fused = mode == 1 ? 1 : 0;
    if (fused == view_.fusedMode) return;
    view_.fusedMode = fused;
    if (graph_) {
        cudaGraphExecDestroy(graph_);
        graph_ = nullptr;
    }
    if (graph1_) {
        cudaGraphExecDestroy(graph1_);
        graph1_ = nullptr;
    }
}

template <typename R>
GroupT<R>::~GroupT() {
    if (graph_) cudaGraphExecDestroy(graph_);
    if (graph1_) cudaGraphExecDestroy(graph1_);
    if (captureStream_) {
        cudaStreamSynchronize(captureStream_);
        cudaStreamDestroy(captureStream_);
    }
    deviceFree(dCases_);
    deviceFree(dTiles_);
    deviceFree(dSync_);
}

// The members' descriptions gathered on the host and sent in one pageable
// host-to-device copy, ordered on s: the call returns once its source is
// staged, so the host copies may change right after.
template <typename R>
void GroupT<R>::refresh(cudaStream_t s) {
    std::vector<DevCaseT<R>> all(members_.size());
    for (size_t i = 0; i < members_.size(); i++) all[i] = members_[i]->c;
    cudaCheck(cudaMemcpyAsync(dCases_, all.data(), all.size() * sizeof(DevCaseT<R>), cudaMemcpyHostToDevice, s),
              "cudaMemcpyAsync");
}

// Captures `iters` whole iterations into one executable graph.
template <typename R>
cudaGraphExec_t GroupT<R>::captureIterations(int iters) {
    cudaGraph_t g = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaCheck(cudaStreamBeginCapture(captureStream_, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture");
    cudaError_t e = cudaSuccess;
    for (int i = 0; i < iters && e == cudaSuccess; i++) e = Launcher<R>::iteration(view_, nstages_, captureStream_);
    const cudaError_t e2 = cudaStreamEndCapture(captureStream_, &g);
    cudaCheck(e, "launch during graph capture");
    cudaCheck(e2, "cudaStreamEndCapture");
    const cudaError_t e3 = cudaGraphInstantiate(&exec, g, 0);
    cudaGraphDestroy(g);
    cudaCheck(e3, "cudaGraphInstantiate");
    return exec;
}

// n iterations as graphs of graphIters_ iterations plus single-iteration
// graphs for the rest (one graph launch instead of 20-30 kernel launches).
template <typename R>
void GroupT<R>::enqueue(long long n, cudaStream_t s) {
    if (n <= 0) return;
    if (!tuned_ && autotune_ && n >= kTuneMinIterations) tune(s);
    cudaCheck(Launcher<R>::setLimits(view_, n, s), "launch k_set_limits");
    if (persist_) {
        for (long long left = n; left > 0; left -= kRunIterations)
            cudaCheck(Persistent<R>::run(view_, scheme_, nstages_, std::min(left, kRunIterations), dSync_, s),
                      "launch k_run");
        return;
    }
    long long left = n;
    if (left >= graphIters_) {
        if (!graph_) graph_ = captureIterations(graphIters_);
        while (left >= graphIters_) {
            cudaCheck(cudaGraphLaunch(graph_, s), "cudaGraphLaunch");
            left -= graphIters_;
        }
    }
    if (left > 0 && !graph1_) graph1_ = captureIterations(1);
    for (long long i = 0; i < left; i++) cudaCheck(cudaGraphLaunch(graph1_, s), "cudaGraphLaunch");
}

template class InstanceT<double>;
template class InstanceT<float>;
template class GroupT<double>;
template class GroupT<float>;

}  // namespace ctbfm
