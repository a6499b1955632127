// Persistent iteration kernel k_run: one cooperative launch runs whole
// pseudo-time iterations of a batch. The phases of an iteration are the
// bodies of the split kernels (kernels_impl.cuh) over the same tile lists,
// each walked with a grid-stride loop, separated by a grid barrier instead
// of kernel boundaries:
//
//   boundary integrals + time step + stage-0 primitives   (all read U^n only)
//   pre-stage (global dt, turbo performance, outlet profiles)
//   per Runge-Kutta stage: faces (every direction and face set) | nodes
//                          (which store the next stage's primitives) |
//                          periodic planes (periodic members only)
//   finalize (norms, convergence), and the count of members still running;
//   the launch ends early when none is.
//
// The work and its order per element are those of the split kernels, so the
// results are bit for bit theirs; what goes away is the per-kernel launch and
// drain, which dominates small batches (a 2-D instance of a few thousand
// nodes runs 20+ launches of a few microseconds each per iteration).
//
// Included by kernels_persist.cu / kernels_persist_f32.cu after
// kernels_impl.cuh, with CTBFM_COHERENT_LOADS defined: later phases read
// what earlier phases of the same launch wrote, which the read-only data
// path does not guarantee.
//
// Grid barrier: thread 0 of each block arrives on a counter and waits for the
// generation to change, with a spin limit; a wait that runs out sets the
// error word, and every block then stops and marks its share of the members
// with status 3 (device error), which the host reports. The launch is
// cooperative, so all blocks are co-resident and the barrier cannot wait on
// a block that is not running.

#include <mutex>

namespace ctbfm {

namespace {

template <typename R>
struct RunArgs {
    const DevCaseT<R>* cases;
    int m;
    TileList bint, dt, inst, node, per;
    TileList face[9];  // direction d, face set k at 3*d + k
    int faceOff[10];   // prefix sums of the face tile counts
    int nstages;
    long long n;       // iterations
    int tuneReps;      // > 0: forced stage-0 evaluations only
    long long spinLimit;
    GridSync* gs;
};

// Tile entry inside the persistent kernel: the enter() checks, with the tile
// taken from a grid-stride index; the instance description is copied into
// shared memory only when the instance changes (descriptions do not change
// while the kernel runs). Block-uniform: every thread reads the same words.
template <typename R>
__device__ __forceinline__ bool enterTile(const DevCaseT<R>* cases, const Tile* tiles, int idx, DevCaseT<R>& sc,
                                          int& cur, int stage, int force, Tile& t) {
    __syncthreads();  // the previous tile's users of the description are done
    t = tiles[idx];
    const DevCaseT<R>* g = cases + t.inst;
    if (!force) {
        const Control* ctl = g->ctl;
        if (ctl->status != 0 || ctl->it >= ctl->it_stop) return false;
    }
    if (stage >= g->nstages) return false;
    if (cur != t.inst) {
        const int4* src = reinterpret_cast<const int4*>(g);
        int4* dst = reinterpret_cast<int4*>(&sc);
        constexpr int n16 = static_cast<int>(sizeof(DevCaseT<R>) / 16);
        for (int i = threadIdx.x; i < n16; i += blockDim.x) dst[i] = __ldg(src + i);
        cur = t.inst;
        __syncthreads();
    }
    return true;
}

// Sense-counting grid barrier with a bounded wait (see the file comment).
// The fences order each block's writes before its arrival and its later
// reads after the release; returns false once any block's wait ran out.
__device__ __forceinline__ bool gridBarrier(GridSync* gs, long long spinLimit) {
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned* gen = &gs->gen;
        const unsigned g0 = *gen;
        __threadfence();
        if (atomicAdd(&gs->count, 1u) == gridDim.x - 1) {
            atomicExch(&gs->count, 0u);
            __threadfence();
            atomicAdd(&gs->gen, 1u);
        } else {
            long long spins = 0;
            while (*gen == g0) {
                if (++spins > spinLimit) {
                    atomicExch(&gs->error, 1);
                    break;
                }
                __nanosleep(32);
            }
        }
        __threadfence();
    }
    __syncthreads();
    return *reinterpret_cast<volatile int*>(&gs->error) == 0;
}

// After a barrier wait ran out: each block marks its share of the members.
template <typename R>
__device__ __forceinline__ void runFailed(const RunArgs<R>& a) {
    if (threadIdx.x == 0)
        for (int i = blockIdx.x; i < a.m; i += gridDim.x) a.cases[i].ctl->status = 3;
}

// The phase bodies as separate (not inlined) functions: each is register-
// allocated on its own, as in its split kernel, instead of all of them
// sharing the allocation of one very large function.
template <int DIR, int SCHEME, typename R, int SET>
__device__ __noinline__ void n_faces(const DevCaseT<R>& c, const Tile& tl, int stage) {
    b_faces<DIR, SCHEME, R, 0, SET>(c, tl, stage);
}
template <typename R, int BX>
__device__ __noinline__ void n_nodes(const DevCaseT<R>& c, const Tile& tl, int stage) {
    b_nodes<R, 0, BX>(c, tl, stage);
}
template <typename R>
__device__ __noinline__ void n_prim(const DevCaseT<R>& c, const Tile& tl, int stage) {
    b_prim<R>(c, tl, stage);
}
template <typename R>
__device__ __noinline__ void n_periodic(const DevCaseT<R>& c, const Tile& tl, int stage) {
    b_periodic<R>(c, tl, stage);
}
template <typename R>
__device__ __noinline__ void n_dt(const DevCaseT<R>& c, const Tile& tl) {
    b_dt<R, 0>(c, tl);
}
template <typename R>
__device__ __noinline__ void n_bint(const DevCaseT<R>& c, const Tile& tl) {
    b_bint<R, 0>(c, tl);
}
template <typename R>
__device__ __noinline__ void n_pre(const DevCaseT<R>& c, const Tile& tl) {
    b_pre<R>(c, tl, 0, 1, 1);
}
template <typename R>
__device__ __noinline__ void n_finalize(const DevCaseT<R>& c, const Tile& tl) {
    b_finalize<R>(c, tl, 0);
}

template <typename R, typename F>
__device__ __forceinline__ void forTiles(const RunArgs<R>& a, const TileList& L, DevCaseT<R>& c, int& cur, int stage,
                                         int force, F&& body) {
    for (int t = blockIdx.x; t < L.n; t += gridDim.x) {
        Tile tl;
        if (enterTile(a.cases, L.tiles, t, c, cur, stage, force, tl)) body(tl);
    }
}

// Face tile t of the face phase if it falls in list J (direction J / 3, face
// set J % 3).
template <int J, typename R, int SCHEME>
__device__ __forceinline__ bool faceJob(const RunArgs<R>& a, DevCaseT<R>& c, int& cur, int t, int stage, int force) {
    if (t < a.faceOff[J] || t >= a.faceOff[J + 1]) return false;
    Tile tl;
    if (enterTile(a.cases, a.face[J].tiles, t - a.faceOff[J], c, cur, stage, force, tl))
        n_faces<J / 3, SCHEME, R, J % 3>(c, tl, stage);
    return true;
}

template <typename R, int SCHEME>
__device__ __forceinline__ void facePhase(const RunArgs<R>& a, DevCaseT<R>& c, int& cur, int stage, int force) {
    for (int t = blockIdx.x; t < a.faceOff[9]; t += gridDim.x) {
        faceJob<0, R, SCHEME>(a, c, cur, t, stage, force) || faceJob<1, R, SCHEME>(a, c, cur, t, stage, force) ||
            faceJob<2, R, SCHEME>(a, c, cur, t, stage, force) || faceJob<3, R, SCHEME>(a, c, cur, t, stage, force) ||
            faceJob<4, R, SCHEME>(a, c, cur, t, stage, force) || faceJob<5, R, SCHEME>(a, c, cur, t, stage, force) ||
            faceJob<6, R, SCHEME>(a, c, cur, t, stage, force) || faceJob<7, R, SCHEME>(a, c, cur, t, stage, force) ||
            faceJob<8, R, SCHEME>(a, c, cur, t, stage, force);
    }
}

template <typename R>
__device__ __forceinline__ void nodePhase(const RunArgs<R>& a, DevCaseT<R>& c, int& cur, int stage, int force) {
    forTiles(a, a.node, c, cur, stage, force, [&](const Tile& tl) {
        if (bfmRareModel(c)) n_nodes<R, 1>(c, tl, stage);
        else n_nodes<R, 0>(c, tl, stage);
    });
}

#define CTBFM_RUN_SYNC()                      \
    do {                                      \
        if (!gridBarrier(a.gs, a.spinLimit)) { \
            runFailed(a);                     \
            return;                           \
        }                                     \
    } while (0)

template <typename R, int SCHEME>
__global__ void __launch_bounds__(256, (facesMinBlocks<SCHEME, R>())) k_run(const RunArgs<R> a) {
    __shared__ DevCaseT<R> c;
    int cur = -1;
    if (a.tuneReps > 0) {  // forced stage-0 evaluations (autotuner)
        for (int r = 0; r < a.tuneReps; r++) {
            forTiles(a, a.node, c, cur, 0, 1, [&](const Tile& tl) { n_prim<R>(c, tl, 0); });
            CTBFM_RUN_SYNC();
            facePhase<R, SCHEME>(a, c, cur, 0, 1);
            CTBFM_RUN_SYNC();
            nodePhase<R>(a, c, cur, 0, 1);
            CTBFM_RUN_SYNC();
            if (a.per.n) {
                forTiles(a, a.per, c, cur, 0, 1, [&](const Tile& tl) { n_periodic<R>(c, tl, 0); });
                CTBFM_RUN_SYNC();
            }
        }
        return;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        a.gs->active[0] = 0;
        a.gs->active[1] = 0;
    }
    for (long long itn = 0; itn < a.n; itn++) {
        // Launcher::iteration: k_bint, k_dt, k_pre, then the stages and k_finalize
        forTiles(a, a.bint, c, cur, 0, 0, [&](const Tile& tl) { n_bint<R>(c, tl); });
        forTiles(a, a.dt, c, cur, 0, 0, [&](const Tile& tl) { n_dt<R>(c, tl); });
        forTiles(a, a.node, c, cur, 0, 0, [&](const Tile& tl) { n_prim<R>(c, tl, 0); });
        CTBFM_RUN_SYNC();
        forTiles(a, a.inst, c, cur, 0, 0, [&](const Tile& tl) { n_pre<R>(c, tl); });
        CTBFM_RUN_SYNC();
        for (int st = 0; st < a.nstages; st++) {
            facePhase<R, SCHEME>(a, c, cur, st, 0);
            CTBFM_RUN_SYNC();
            nodePhase<R>(a, c, cur, st, 0);
            CTBFM_RUN_SYNC();
            if (a.per.n) {
                forTiles(a, a.per, c, cur, st, 0, [&](const Tile& tl) { n_periodic<R>(c, tl, st); });
                CTBFM_RUN_SYNC();
            }
        }
        const int slot = static_cast<int>(itn & 1);
        if (blockIdx.x == 0 && threadIdx.x == 0) a.gs->active[slot ^ 1] = 0;  // the next iteration's count
        forTiles(a, a.inst, c, cur, 0, 0, [&](const Tile& tl) {
            n_finalize<R>(c, tl);
            if (threadIdx.x == 0) {
                const Control* ctl = c.ctl;
                if (ctl->status == 0 && ctl->it < ctl->it_stop) atomicAdd(&a.gs->active[slot], 1);
            }
        });
        CTBFM_RUN_SYNC();
        if (*reinterpret_cast<volatile int*>(&a.gs->active[slot]) == 0) return;  // every member has stopped
    }
}

#undef CTBFM_RUN_SYNC

// A barrier wait limit of 2^25 polls of at least 32 ns each: over a second,
// several hundred times the longest phase of the largest batches.
constexpr long long kBarrierSpins = 1LL << 25;

template <typename R>
RunArgs<R> runArgs(const BatchView<R>& b, int scheme) {
    RunArgs<R> a{};
    a.cases = b.cases;
    a.m = b.m;
    a.bint = b.bint;
    a.dt = b.node;
    a.inst = b.inst;
    a.node = b.split[0].node;
    a.per = b.per;
    a.faceOff[0] = 0;
    for (int d = 0; d < 3; d++)
        for (int k = 0; k < 3; k++) {
            a.face[3 * d + k] = b.split[0].face[d][scheme][k];
            a.faceOff[3 * d + k + 1] = a.faceOff[3 * d + k] + a.face[3 * d + k].n;
        }
    a.spinLimit = kBarrierSpins;
    return a;
}

// Co-resident blocks of k_run<R, SCHEME> on the current device (queried once
// per device).
template <typename R, int SCHEME>
cudaError_t residentBlocks(int* out) {
    constexpr int kDevices = 64;
    static std::mutex mu;
    static int cache[kDevices] = {};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(mu);
    if (!cache[dev]) {
        int perSM = 0, sms = 0;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, k_run<R, SCHEME>, 256, 0);
        if (e != cudaSuccess) return e;
        e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (e != cudaSuccess) return e;
        if (perSM < 1) return cudaErrorLaunchOutOfResources;
        cache[dev] = perSM * sms;
    }
    *out = cache[dev];
    return cudaSuccess;
}

template <typename R>
int largestPhase(const RunArgs<R>& a) {
    int n = a.faceOff[9];
    for (int t : {a.bint.n + a.dt.n + a.node.n, a.inst.n, a.node.n, a.per.n}) n = t > n ? t : n;
    return n > 0 ? n : 1;
}

template <typename R, int SCHEME>
cudaError_t launchRun(const RunArgs<R>& a, cudaStream_t s) {
    int resident = 0;
    cudaError_t e = residentBlocks<R, SCHEME>(&resident);
    if (e != cudaSuccess) return e;
    const int want = largestPhase(a);
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(static_cast<unsigned>(want < resident ? want : resident));
    cfg.blockDim = dim3(256);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeCooperative;
    at[0].val.cooperative = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, k_run<R, SCHEME>, a);
}

}  // namespace

template <typename R>
cudaError_t Persistent<R>::run(const BatchView<R>& b, int scheme, int nstages, long long n, GridSync* gs,
                               cudaStream_t s) {
    if (n <= 0 || !b.m) return cudaSuccess;
    RunArgs<R> a = runArgs(b, scheme);
    a.nstages = nstages;
    a.n = n;
    a.tuneReps = 0;
    a.gs = gs;
    return scheme ? launchRun<R, 1>(a, s) : launchRun<R, 0>(a, s);
}

template <typename R>
cudaError_t Persistent<R>::tuneStage(const BatchView<R>& b, int scheme, int reps, GridSync* gs, cudaStream_t s) {
    if (reps <= 0 || !b.m) return cudaSuccess;
    RunArgs<R> a = runArgs(b, scheme);
    a.nstages = 1;
    a.n = 0;
    a.tuneReps = reps;
    a.gs = gs;
    return scheme ? launchRun<R, 1>(a, s) : launchRun<R, 0>(a, s);
}

template <typename R>
int Persistent<R>::gridBlocks(const BatchView<R>& b, int scheme) {
    int resident = 0;
    const cudaError_t e = scheme ? residentBlocks<R, 1>(&resident) : residentBlocks<R, 0>(&resident);
    if (e != cudaSuccess) return 0;
    const int want = largestPhase(runArgs(b, scheme));
    return want < resident ? want : resident;
}

}  // namespace ctbfm
