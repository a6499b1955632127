// Kernels of the explicit residual-and-update loop (sm_100a), templated on the
// working precision R and driven by tiles, so that one launch advances any set
// of operating points (one, or a whole batch of uneven grids).
//
// A launch's grid has one block per Tile; a tile is a contiguous range of one
// instance's elements (nodes, faces of one direction, periodic (i,j) pairs,
// boundary planes or the instance itself). Each block returns at once when
// its instance has converged, diverged or reached its iteration limit, so
// finished instances cost next to nothing while the rest of the batch runs,
// and otherwise copies the instance's DevCaseT into shared memory.
//
// One pseudo-time iteration, with no host synchronisation:
//   k_set_limits (once per enqueue), k_bint (boundary integrals, when turbo
//   performance is needed), k_dt, k_pre, then per Runge-Kutta stage k_prim,
//   k_faces<I|J|K>, k_nodes, k_periodic, and finally k_finalize.
//
// The double instantiation (kernels.cu) is compiled with --fmad=false so that
// each expression rounds as the reference's does; the float instantiation
// (kernels_f32.cu) keeps a Kahan compensation term of the state.

#include <cuda_runtime.h>

#include <mutex>

#include "kernels.hpp"
#include "sources.cuh"
#include "viscous.cuh"

namespace ctbfm {

namespace {

// Resident blocks of 256 threads per SM asked of the face and node kernels,
// i.e. their register budget (65536 / (256 * blocks) per thread), measured on
// B200 (bench workload and a 768 x 256 JST bump): double Roe faces 3 blocks
// (85 registers, 69.6 us for the K faces against 76.3 us at 2 blocks and
// 124 us unbounded), double JST faces 2 (3 spills more than it gains), nodes
// 3 in double (63.6 us against 71.8 us at 2) and 4 in float (the batched
// compressor map 5 % faster than at 3).
template <int SCHEME, typename R>
constexpr int facesMinBlocks() {
    return (sizeof(R) == 8 && SCHEME == 0) ? 2 : 3;
}
template <typename R>
constexpr int nodesMinBlocks() {
    return sizeof(R) == 8 ? 3 : 4;
}

// Block entry: reads the block's tile, returns false (the whole block leaves
// before touching anything else) when its instance has converged, diverged,
// reached its iteration limit, has no such stage or another fluid model than
// the kernel was compiled for, and otherwise copies the
// instance description into shared memory. Every thread reads the same
// control words, which no kernel writes while others read them.
// Programmatic dependent launch: kernels are launched with programmatic
// stream serialization, so a grid's launch is processed while its
// predecessor's blocks drain, and each kernel waits here, before touching any
// memory, until the previous grid on its stream has completed and its writes
// are visible. The predecessor signals only by exiting (an explicit early
// launch_dependents measured 1.5-4 % slower per iteration on the
// 160 x 48 x 64 annulus). Without the launch attribute the wait does
// nothing.
__device__ __forceinline__ void gridDependency() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

template <typename R>
__device__ __forceinline__ bool enter(const DevCaseT<R>* cases, const Tile* tiles, DevCaseT<R>& sc, int stage,
                                      int force, Tile& t, int fluid = -1, int bfmx = -1) {
    gridDependency();
    t = tiles[blockIdx.x];
    const DevCaseT<R>* g = cases + t.inst;
    // kernels compiled for one fluid model (0 ideal, 1 look-up table) take
    // only the instances of that model
    if (fluid >= 0 && (g->lut != nullptr) != (fluid != 0)) return false;
    // node kernels compiled with (1) or without (0) the Chima / Correlations forces
    if (bfmx >= 0 && bfmRareModel(*g) != (bfmx != 0)) return false;
    if (!force) {
        const Control* ctl = g->ctl;
        if (ctl->status != 0 || ctl->it >= ctl->it_stop) return false;
    }
    if (stage >= g->nstages) return false;
    const int4* src = reinterpret_cast<const int4*>(g);
    int4* dst = reinterpret_cast<int4*>(&sc);
    constexpr int n16 = static_cast<int>(sizeof(DevCaseT<R>) / 16);
    for (int i = threadIdx.x; i < n16; i += blockDim.x) dst[i] = __ldg(src + i);
    __syncthreads();
    return true;
}

// Stage buffers: RK4 U -> S1 -> S2 -> S1 -> U, RK3 U -> S1 -> S2 -> U (the
// last stage updates U^n in place); stage -1 is a residual-only evaluation of
// U^n into S2.
template <typename R>
__device__ __forceinline__ R* const* stageIn(const DevCaseT<R>& c, int s) {
    if (s <= 0) return c.U;
    if (s == 1) return c.S1;
    if (s == 2) return c.S2;
    return c.S1;
}
template <typename R>
__device__ __forceinline__ R* const* stageOut(const DevCaseT<R>& c, int s) {
    if (s < 0) return c.S2;
    if (s == c.nstages - 1) return c.U;
    if (s == 0) return c.S1;
    if (s == 1) return c.S2;
    return c.S1;
}

// Not inlined: the boundary faces are few, and keeping their many flux
// variants out of the face kernels' bodies halves the kernels' spills.
// onWall: the face's own (i, j, k), read as a node, lies on a no-slip wall of
// a viscous instance (BoundaryBase::isNodeOnNoSlipWall,
// include/boundary_base.hpp:44-49): inlet faces there take the stagnation
// flux (src/boundary_inlet.cpp:16-19, src/boundary_inlet_supersonic.cpp:15-18).
template <int SCHEME, typename R>
__device__ __noinline__ S5<R> boundaryFlux(const DevCaseT<R>& c, Gas<R> gs, int pidx, const S5<R>& Uint, V3<R> n,
                                              long long qtheta, int fj, long long it, bool onWall) {
    const DevPatch& p = c.patch[pidx];
    if (onWall && (p.type == kBcInlet || p.type == kBcInletSupersonic)) return stagnationWallFlux(R(p.v[0]), n);
    switch (p.type) {
        case kBcInlet: return bcInlet(c, gs, p, Uint, n, c.cost[qtheta], c.sint[qtheta]);
        case kBcOutlet: return bcOutlet(c, gs, Uint, n, R(p.v[0]), it);
        case kBcInletSupersonic: return bcInletSupersonic(gs, p, n);
        case kBcOutletSupersonic: return bcOutletSupersonic(gs, Uint, n);
        case kBcFarfield: return bcFarfield(gs, p, Uint, n);
        case kBcTransparent:
            // BoundaryTransparent (src/boundary_transparent.cpp:5-16): the
            // scheme's own flux with the interior state on both sides
            if (SCHEME == 0) return fluxJst(gs, Uint, Uint, Uint, Uint, n);
            return fluxRoe(gs, c.muscl, c.limiter, Uint, Uint, Uint, Uint, n);
        case kBcMassFlow:  // BoundaryOutletMassFlow (src/boundary_outlet_mass_flow.cpp:4-19)
        case kBcRadialEq:
        case kBcThrottle: {
            // BoundaryOutletThrottle / RadialEquilibrium index the profile by the
            // face's j (src/boundary_outlet_throttle.cpp:14).
            const int m = p.profile;
            const int jj = fj < c.prof_n[m] ? fj : c.prof_n[m] - 1;
            return bcOutlet(c, gs, Uint, n, R(c.prof_p[c.prof_off[m] + jj]), it);
        }
        case kBcInviscidWall:
        case kBcNoSlipWall: return bcWall(gs, Uint, n);  // BoundaryInviscidWall for both (src/solver.cpp:393-398)
        default: return zero5<R>();  // periodic / wedge faces: BoundaryFake, zero flux
    }
}

// linearInterpolation (src/math_utils.cpp:487-514): constant beyond the ends,
// otherwise linear in the interval [x_i, x_i+1) that holds xp (x ascending).
__device__ __forceinline__ double linearInterpolation(const double* x, const double* y, int n, double xp) {
    if (xp <= x[0]) return y[0];
    if (xp >= x[n - 1]) return y[n - 1];
    int i = 0;
    while (i + 1 < n && x[i + 1] <= xp) i++;  // last x_i <= xp: std::upper_bound - 1
    const double t = (xp - x[i]) / (x[i + 1] - x[i]);
    return (1.0 - t) * y[i] + t * y[i + 1];
}

// Deterministic block sum of NV doubles per thread; result valid in thread 0.
template <int NV>
__device__ __forceinline__ void blockSum(double (&v)[NV]) {
    __shared__ double sh[NV][32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int c = 0; c < NV; c++)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[c] += __shfl_down_sync(0xffffffffu, v[c], o);
    if (lane == 0)
#pragma unroll
        for (int c = 0; c < NV; c++) sh[c][warp] = v[c];
    __syncthreads();
    if (warp == 0) {
        const int nw = (blockDim.x + 31) >> 5;
#pragma unroll
        for (int c = 0; c < NV; c++) {
            v[c] = lane < nw ? sh[c][lane] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v[c] += __shfl_down_sync(0xffffffffu, v[c], o);
        }
    }
    __syncthreads();
}

__device__ __forceinline__ double blockMin(double v) {
    __shared__ double sh[32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_down_sync(0xffffffffu, v, o));
    if (lane == 0) sh[warp] = v;
    __syncthreads();
    if (warp == 0) {
        const int nw = (blockDim.x + 31) >> 5;
        v = lane < nw ? sh[lane] : INFINITY;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_down_sync(0xffffffffu, v, o));
    }
    __syncthreads();
    return v;
}

// The state in double, including the compensation term of the float path.
template <typename R>
__device__ __forceinline__ S5<double> state64(const DevCaseT<R>& c, R* const* U, long long q) {
    S5<double> s;
#pragma unroll
    for (int v = 0; v < 5; v++) s.v[v] = static_cast<double>(U[v][q]);
    if (c.compensated && U == c.U)
#pragma unroll
        for (int v = 0; v < 5; v++) s.v[v] -= static_cast<double>(c.Uc[v][q]);
    return s;
}

// Viscous face contributions of node (i, j, k) (Solver::computeViscousFluxResiduals,
// src/solver.cpp:2060-2171): interior faces only; the reference adds
// -flux*|S| to the left node and subtracts it from the right one, so a node
// takes +V of its start face, then -V of its end face, direction by direction
// (K only in 3-D). The mass residual receives zeros, which change nothing.
template <typename R>
__device__ __forceinline__ void addViscousResidual(const DevCaseT<R>& c, int i, int j, int k, S5<R>& Res) {
    const int nj = c.nj, nk = c.nk;
    {
        const long long f0 = (static_cast<long long>(i) * nj + j) * nk + k;
        const long long f1 = f0 + static_cast<long long>(nj) * nk;
#pragma unroll
        for (int v = 0; v < 4; v++) {
            if (i >= 1) Res.v[v + 1] = Res.v[v + 1] + c.V[0][v][f0];
            if (i + 1 <= c.ni - 1) Res.v[v + 1] = Res.v[v + 1] - c.V[0][v][f1];
        }
    }
    {
        const long long f0 = (static_cast<long long>(i) * (nj + 1) + j) * nk + k;
        const long long f1 = f0 + nk;
#pragma unroll
        for (int v = 0; v < 4; v++) {
            if (j >= 1) Res.v[v + 1] = Res.v[v + 1] + c.V[1][v][f0];
            if (j + 1 <= nj - 1) Res.v[v + 1] = Res.v[v + 1] - c.V[1][v][f1];
        }
    }
    if (c.topo == 1) {
        const long long f0 = (static_cast<long long>(i) * nj + j) * (nk + 1) + k;
        const long long f1 = f0 + 1;
#pragma unroll
        for (int v = 0; v < 4; v++) {
            if (k >= 1) Res.v[v + 1] = Res.v[v + 1] + c.V[2][v][f0];
            if (k + 1 <= nk - 1) Res.v[v + 1] = Res.v[v + 1] - c.V[2][v][f1];
        }
    }
}

// Solver::setMomentumSolutionOnViscousWalls (src/solver.cpp:3147-3186) on the
// residual of a wall node (enforceNoSlipWallsOnResiduals, :1856-1863): the
// momentum residual becomes the mass residual times the zero wall velocity.
template <typename R>
__device__ __forceinline__ void noSlipResidual(S5<R>& Res) {
    Res.v[1] = Res.v[0] * R(0);
    Res.v[2] = Res.v[0] * R(0);
    Res.v[3] = Res.v[0] * R(0);
}

// ----------------------------------------------------------- viscous terms
// Solver::computeSolutionGradient (src/solver.cpp:3033-3058) with
// computeGradientsGreenGauss4 (src/math_utils.cpp:237-392): per node the
// gradients of u, v, w and T over the six dual faces, W E N S B T, each face
// value interpolated between the node and its neighbour with the face
// centre's distance weights (the node's own value on boundary faces), summed
// in that order and multiplied by 1/V. Reads the primitives of k_prim.
template <typename R, int FL>
__global__ void __launch_bounds__(256) k_grad(const DevCaseT<R>* cases, const Tile* tiles, int stage, int force) {
    __shared__ DevCaseT<R> c;
    Tile tl;
    if (!enter(cases, tiles, c, stage, force, tl, FL)) return;
    const Gas<R> gs{R(c.gamma), R(c.rgas), FL ? c.lut : nullptr};
    const int ni = c.ni, nj = c.nj, nk = c.nk;
    const long long sI = static_cast<long long>(nj) * nk;
    for (long long q = tl.start + threadIdx.x; q < tl.start + tl.count; q += blockDim.x) {
        const int k = static_cast<int>(q % nk);
        const long long tq = q / nk;
        const int j = static_cast<int>(tq % nj);
        const int i = static_cast<int>(tq / nj);
        auto fields = [&](long long n, R (&f)[4]) {
            const S5<R> W = load5(c.W, n);
            f[0] = W.v[1];
            f[1] = W.v[2];
            f[2] = W.v[3];
            f[3] = gradientTemperature(c, gs, W);
        };
        R fc[4];
        fields(q, fc);
        R g[4][3];
#pragma unroll
        for (int v = 0; v < 4; v++) g[v][0] = g[v][1] = g[v][2] = R(0);
        // face f of the node: neighbour (or -1), face index in its direction's
        // grid, sign of S, and whether the node is the face's left node
        auto face = [&](int d, long long fidx, long long nb, bool neg, bool left) {
            R sv[4];
            if (nb >= 0) {
                const R w = left ? __ldg(c.gwL[d] + fidx) : __ldg(c.gwR[d] + fidx);
                R fn[4];
                fields(nb, fn);
#pragma unroll
                for (int v = 0; v < 4; v++) sv[v] = fc[v] + (fn[v] - fc[v]) * w;
            } else {
#pragma unroll
                for (int v = 0; v < 4; v++) sv[v] = fc[v];
            }
            R S[3] = {__ldg(c.sraw[d][0] + fidx), __ldg(c.sraw[d][1] + fidx), __ldg(c.sraw[d][2] + fidx)};
            if (neg) S[0] = -S[0], S[1] = -S[1], S[2] = -S[2];
#pragma unroll
            for (int v = 0; v < 4; v++)
#pragma unroll
                for (int x = 0; x < 3; x++) g[v][x] = addRn(g[v][x], mulRn(S[x], sv[v]));
        };
        const long long fI = (static_cast<long long>(i) * nj + j) * nk + k;        // I face i
        const long long fJ = (static_cast<long long>(i) * (nj + 1) + j) * nk + k;  // J face j
        const long long fK = (static_cast<long long>(i) * nj + j) * (nk + 1) + k;  // K face k
        face(0, fI, i > 0 ? q - sI : -1, true, false);             // west: face i, node on its right
        face(0, fI + sI, i < ni - 1 ? q + sI : -1, false, true);   // east: face i+1, node on its left
        face(1, fJ + nk, j < nj - 1 ? q + nk : -1, false, true);   // north: face j+1
        face(1, fJ, j > 0 ? q - nk : -1, true, false);             // south: face j
        face(2, fK, k > 0 ? q - 1 : -1, true, false);              // bottom: face k
        face(2, fK + 1, k < nk - 1 ? q + 1 : -1, false, true);     // top: face k+1
        const R inv = R(1) / c.vol[q];
#pragma unroll
        for (int v = 0; v < 4; v++)
#pragma unroll
            for (int x = 0; x < 3; x++) c.G[3 * v + x][q] = g[v][x] * inv;
    }
}

// Solver::computeViscousFluxResiduals (src/solver.cpp:2060-2171): one thread
// per face of direction DIR in storage order (3 blocks of 256 per SM: 80
// registers with a few spills, 3 % faster in FP64 and 12 % in float than 90
// registers at 2 blocks on the viscous duct); interior faces write
// flux * |S| of the momentum and energy equations from the averaged node
// states and gradients (boundary faces carry no viscous flux and are not
// read).
template <int DIR, typename R, int FL>
__global__ void __launch_bounds__(256, 3) k_vfaces(const DevCaseT<R>* cases, const Tile* tiles, int stage, int force) {
    __shared__ DevCaseT<R> c;
    Tile tl;
    if (!enter(cases, tiles, c, stage, force, tl, FL)) return;
    const Gas<R> gs{R(c.gamma), R(c.rgas), FL ? c.lut : nullptr};
    const int nfj = c.nj + (DIR == 1), nfk = c.nk + (DIR == 2);
    const int nlast = DIR == 0 ? c.ni : (DIR == 1 ? c.nj : c.nk);
    const long long st = DIR == 0 ? static_cast<long long>(c.nj) * c.nk : (DIR == 1 ? c.nk : 1);
    const DevFacesT<R>& F = c.f[DIR];
    R* const* U = stageIn(c, stage);
    for (long long f = tl.start + threadIdx.x; f < tl.start + tl.count; f += blockDim.x) {
        const int fk = static_cast<int>(f % nfk);
        const long long t = f / nfk;
        const int fj = static_cast<int>(t % nfj);
        const int fi = static_cast<int>(t / nfj);
        const int dface = DIR == 0 ? fi : (DIR == 1 ? fj : fk);
        if (dface == 0 || dface == nlast) continue;
        const long long qR = nodeIdx(c, fi, fj, fk);
        const long long qL = qR - st;
        const S5<R> Ua = (load5(U, qL) + load5(U, qR)) * R(0.5);
        V3<R> gr[4];
#pragma unroll
        for (int v = 0; v < 4; v++)
            gr[v] = v3((c.G[3 * v][qL] + c.G[3 * v][qR]) * R(0.5), (c.G[3 * v + 1][qL] + c.G[3 * v + 1][qR]) * R(0.5),
                       (c.G[3 * v + 2][qL] + c.G[3 * v + 2][qR]) * R(0.5));
        const R muEddy = (saEddy(c, U[0][qL], qL) + saEddy(c, U[0][qR], qR)) * R(0.5);
        const V3<R> n = v3(__ldg(F.nx + f), __ldg(F.ny + f), __ldg(F.nz + f));
        const R area = __ldg(F.area + f);
        R flux[4];
        viscousFlux(c, gs, Ua, gr[0], gr[1], gr[2], gr[3], n, muEddy, flux);
#pragma unroll
        for (int v = 0; v < 4; v++) c.V[DIR][v][f] = flux[v] * area;
    }
}

// ------------------------------------------------------------------ faces
// Solver::computeAdvectionFluxResidualsImpl (src/solver.cpp:1865-2040): one
// thread per face of direction DIR; writes flux * |S|. SET 0 enumerates every
// face of the direction in storage order; for J and K, SET 1 enumerates the
// faces at positions 2 .. n-2 along each line and SET 2 the faces at 0, 1,
// n-1 and n (n = nj or nk, at least 3), the k index fastest where the line
// is not along k, so that warps of one launch take one code path.
template <int DIR, int SCHEME, typename R, int FL, int SET>
__device__ __forceinline__ void b_faces(const DevCaseT<R>& c, const Tile& tl, int stage) {
    const long long it = c.ctl->it + 1;
    const Gas<R> gs{R(c.gamma), R(c.rgas), FL ? c.lut : nullptr};
    const int nfj = c.nj + (DIR == 1), nfk = c.nk + (DIR == 2);
    const long long st = DIR == 0 ? static_cast<long long>(c.nj) * c.nk : (DIR == 1 ? c.nk : 1);
    const int nlast = DIR == 0 ? c.ni : (DIR == 1 ? c.nj : c.nk);
    const DevFacesT<R>& F = c.f[DIR];
    R* const* U = stageIn(c, stage);
    for (long long p = tl.start + threadIdx.x; p < tl.start + tl.count; p += blockDim.x) {
        long long f;
        int fi, fj, fk;
        if (SET == 0 || DIR == 0) {
            if (SET == 0) {
                f = p;
            } else {  // I faces: the planes fi = 2 .. ni-2 are contiguous, the end planes 0, 1, ni-1, ni
                const long long plane = static_cast<long long>(c.nj) * c.nk;
                if (SET == 1) {
                    f = 2 * plane + p;
                } else {
                    const int s4 = static_cast<int>(p / plane);
                    f = static_cast<long long>(s4 < 2 ? s4 : c.ni - 3 + s4) * plane + p % plane;
                }
            }
            fk = static_cast<int>(f % nfk);
            const long long t = f / nfk;
            fj = static_cast<int>(t % nfj);
            fi = static_cast<int>(t / nfj);
        } else if (DIR == 1) {
            fk = static_cast<int>(p % c.nk);
            const long long t = p / c.nk;
            if (SET == 1) {
                const int m = c.nj - 3;
                fj = 2 + static_cast<int>(t % m);
                fi = static_cast<int>(t / m);
            } else {
                const int s4 = static_cast<int>(t % 4);
                fj = s4 < 2 ? s4 : c.nj - 3 + s4;
                fi = static_cast<int>(t / 4);
            }
            f = (static_cast<long long>(fi) * nfj + fj) * c.nk + fk;
        } else {
            long long t;
            if (SET == 1) {
                const int m = c.nk - 3;
                fk = 2 + static_cast<int>(p % m);
                t = p / m;
            } else {
                const int s4 = static_cast<int>(p % 4);
                fk = s4 < 2 ? s4 : c.nk - 3 + s4;
                t = p / 4;
            }
            fj = static_cast<int>(t % c.nj);
            fi = static_cast<int>(t / c.nj);
            f = (static_cast<long long>(fi) * c.nj + fj) * nfk + fk;
        }
        const int dface = DIR == 0 ? fi : (DIR == 1 ? fj : fk);
        if (DIR == 2 && c.bfm && c.bpresent[nodeIdx(c, fi, fj, 0)] > R(0)) continue;  // blade rows: no K flux
        V3<R> n = v3(__ldg(F.nx + f), __ldg(F.ny + f), __ldg(F.nz + f));
        const R area = __ldg(F.area + f);
        S5<R> flux;
        // SET 1 holds plain interior faces only, SET 2 only the four end faces
        // of a line: each launch compiles only the paths it can take
        if (SET != 1 && (dface == 0 || dface == nlast)) {
            const int side = dface == 0 ? 0 : 1;
            const int ni_ = DIR == 0 ? (side ? c.ni - 1 : 0) : fi;
            const int nj_ = DIR == 1 ? (side ? c.nj - 1 : 0) : fj;
            const int nk_ = DIR == 2 ? (side ? c.nk - 1 : 0) : fk;
            const long long q = nodeIdx(c, ni_, nj_, nk_);
            if (side == 0) n = -n;  // outward normal of the start face
            int pidx;
            if (DIR == 0) pidx = c.mapI[(static_cast<long long>(side) * c.nj + fj) * c.nk + fk];
            else if (DIR == 1) pidx = c.mapJ[(static_cast<long long>(fi) * 2 + side) * c.nk + fk];
            else pidx = c.mapK[(static_cast<long long>(fi) * c.nj + fj) * 2 + side];
            // theta of the face's (i, j, k) node for the cylindrical inlet frame
            const long long qth =
                nodeIdx(c, fi < c.ni ? fi : c.ni - 1, fj < c.nj ? fj : c.nj - 1, fk < c.nk ? fk : c.nk - 1);
            const bool onWall = c.viscous && fi < c.ni && fj < c.nj && fk < c.nk && c.wall[nodeIdx(c, fi, fj, fk)];
            flux = boundaryFlux<SCHEME>(c, gs, pidx, load5(U, q), n, qth, fj, it, onWall);
        } else {
            const long long qR = nodeIdx(c, fi, fj, fk);
            const long long qL = qR - st;
            // faces whose four stencil nodes are plain interior nodes read the
            // primitives k_prim computed once per node (bitwise the same values
            // as converting here); faces next to a boundary or a periodic seam
            // extrapolate or rotate conservative states first
            const bool plain = SET == 1 || (SET == 0 && dface >= 2 && dface <= nlast - 2);
            if (plain) {
                if (SCHEME == 0) {
                    flux = fluxJstPR(gs, load5(U, qL - st), load5(U, qL), load5(U, qR), load5(U, qR + st),
                                     load5(c.W, qL), load5(c.W, qR), CTBFM_LDS(c.Wp + qL - st), CTBFM_LDS(c.Wp + qL),
                                     CTBFM_LDS(c.Wp + qR), CTBFM_LDS(c.Wp + qR + st), CTBFM_LDS(c.Wr + qL),
                                     CTBFM_LDS(c.Wr + qR), n);
                } else {
                    flux = fluxRoeW(gs, c.muscl, c.limiter, c.muscl ? load5(c.W, qL - st) : zero5<R>(),
                                    load5(c.W, qL), load5(c.W, qR), c.muscl ? load5(c.W, qR + st) : zero5<R>(), n,
                                    v3(__ldg(F.n2x + f), __ldg(F.n2y + f), R(0)));
                }
            } else {
                // the three real stencil nodes take the primitives (and, for
                // JST, pressures and spectral radii) stored per node, the same
                // values as converting their states here; only the ghost state
                // (extrapolated, or rotated across the periodic seam) is
                // converted
                const S5<R> Ul = load5(U, qL), Ur = load5(U, qR);
                S5<R> Ull, Urr;
                long long qReal;  // the real outer node: qL - st (ghost on the right) or qR + st
                const bool ghostLeft = dface == 1;
                if (DIR == 2 && c.periodic) {
                    if (ghostLeft) {
                        Ull = rotState(load5(U, nodeIdx(c, fi, fj, c.nk - 2)), R(c.per_cos_m), R(c.per_sin_m));
                        qReal = qR + 1;
                        Urr = load5(U, qReal);
                    } else {  // dface == nlast - 1
                        qReal = qR - 2;
                        Ull = load5(U, qReal);
                        Urr = rotState(load5(U, nodeIdx(c, fi, fj, 1)), R(c.per_cos_p), R(c.per_sin_p));
                    }
                } else {
                    if (ghostLeft) {
                        Ull = Ul - (Ur - Ul);
                        qReal = qR + st;
                        Urr = load5(U, qReal);
                    } else {  // dface == nlast - 1
                        qReal = qL - st;
                        Ull = load5(U, qReal);
                        Urr = Ur + (Ur - Ul);
                    }
                }
                const S5<R> Wl = load5(c.W, qL), Wr = load5(c.W, qR);
                if (SCHEME == 0) {
                    const S5<R> Wg = primOf(ghostLeft ? Ull : Urr);
                    const R pg = pressurePrim(gs, Wg), pReal = CTBFM_LDS(c.Wp + qReal);
                    flux = fluxJstPR(gs, Ull, Ul, Ur, Urr, Wl, Wr, ghostLeft ? pg : pReal, CTBFM_LDS(c.Wp + qL),
                                     CTBFM_LDS(c.Wp + qR), ghostLeft ? pReal : pg, CTBFM_LDS(c.Wr + qL),
                                     CTBFM_LDS(c.Wr + qR), n);
                } else {
                    const V3<R> n2 = v3(__ldg(F.n2x + f), __ldg(F.n2y + f), R(0));
                    if (c.muscl) {
                        const S5<R> Wg = primOf(ghostLeft ? Ull : Urr), Wreal = load5(c.W, qReal);
                        flux = fluxRoeW(gs, 1, c.limiter, ghostLeft ? Wg : Wreal, Wl, Wr, ghostLeft ? Wreal : Wg, n,
                                        n2);
                    } else {
                        flux = fluxRoeW(gs, 0, c.limiter, zero5<R>(), Wl, Wr, zero5<R>(), n, n2);
                    }
                }
            }
        }
#pragma unroll
        for (int v = 0; v < 5; v++) F.c[v][f] = flux.v[v] * area;
    }
}

template <int DIR, int SCHEME, typename R, int FL, int SET>
__global__ void __launch_bounds__(256, (facesMinBlocks<SCHEME, R>())) k_faces(const DevCaseT<R>* cases, const Tile* tiles, int stage, int force) {
    __shared__ DevCaseT<R> c;
    Tile tl;
    if (!enter(cases, tiles, c, stage, force, tl, FL)) return;
    b_faces<DIR, SCHEME, R, FL, SET>(c, tl, stage);
}

// Primitives of the stage input (getPrimitiveVariablesFromConservative,
// src/math_utils.cpp:49-57), once per node for the face kernels; for JST
// also each node's pressure and spectral radius |u| + a, which the JST flux
// of every face reads at its four (pressure) and two (radius) stencil nodes
// (the same values the flux computed per face before).
// The node kernels of stages 0 .. nstages-2 store the primitives of the
// state they write, which the next stage's faces read, so k_prim runs only
// for stage 0 (and residual-only evaluations).
template <typename R>
__device__ __forceinline__ void storePrim(const DevCaseT<R>& c, long long q, const S5<R>& U) {
    const Gas<R> gs{R(c.gamma), R(c.rgas), c.lut};
    const S5<R> W = primOf(U);
    store5(c.W, q, W);
    if (c.Wp) {
        c.Wp[q] = pressurePrim(gs, W);
        c.Wr[q] = jstR(gs, W);
    }
}

template <typename R>
__device__ __forceinline__ void b_prim(const DevCaseT<R>& c, const Tile& tl, int stage) {
    R* const* U = stageIn(c, stage);
    for (long long q = tl.start + threadIdx.x; q < tl.start + tl.count; q += blockDim.x) storePrim(c, q, load5(U, q));
}

template <typename R>
__global__ void __launch_bounds__(256) k_prim(const DevCaseT<R>* cases, const Tile* tiles, int stage, int force) {
    __shared__ DevCaseT<R> c;
    Tile tl;
    if (!enter(cases, tiles, c, stage, force, tl)) return;
    b_prim<R>(c, tl, stage);
}

// ------------------------------------------------------------------ nodes
// Residual assembly in the reference's accumulation order (I faces, J faces,
// K faces, viscous I, J, K faces, then sources; no-slip wall nodes lose their
// momentum residual last), then Solver::updateSolution (src/solver.cpp:2230-2249)
// U(k) = U^n - R * (alpha*dt/V); with the compensated state the update is a
// Kahan sum carrying the rounding error of U^n. stage -1 writes R to S2.
template <typename R, int FL, int BX>
__device__ __forceinline__ void b_nodes(const DevCaseT<R>& c, const Tile& tl, int stage) {
    const Gas<R> gs{R(c.gamma), R(c.rgas), FL ? c.lut : nullptr};
    const double t = c.ctl->t;
    const R dtg = R(c.ctl->dt_min);
    const bool resOnly = stage < 0;
    const bool last = !resOnly && stage == c.nstages - 1;
    const R alpha = resOnly ? R(0) : R(c.coeffs[stage]);
    R* const* Uin = stageIn(c, stage);
    R* const* Uout = stageOut(c, stage);
    double acc[5] = {0, 0, 0, 0, 0};
    const int nj = c.nj, nk = c.nk;
    for (long long q = tl.start + threadIdx.x; q < tl.start + tl.count; q += blockDim.x) {
        const int k = static_cast<int>(q % nk);
        const long long tq = q / nk;
        const int j = static_cast<int>(tq % nj);
        const int i = static_cast<int>(tq / nj);
        S5<R> Res = zero5<R>();
        {  // I faces: face i (node is right, or the start boundary) then face i+1
            const long long f0 = (static_cast<long long>(i) * nj + j) * nk + k;
            const long long f1 = f0 + static_cast<long long>(nj) * nk;
#pragma unroll
            for (int v = 0; v < 5; v++) {
                const R a = c.f[0].c[v][f0];
                Res.v[v] = (i == 0) ? Res.v[v] + a : Res.v[v] - a;
                Res.v[v] = Res.v[v] + c.f[0].c[v][f1];
            }
        }
        {  // J faces
            const long long f0 = (static_cast<long long>(i) * (nj + 1) + j) * nk + k;
            const long long f1 = f0 + nk;
#pragma unroll
            for (int v = 0; v < 5; v++) {
                const R a = c.f[1].c[v][f0];
                Res.v[v] = (j == 0) ? Res.v[v] + a : Res.v[v] - a;
                Res.v[v] = Res.v[v] + c.f[1].c[v][f1];
            }
        }
        if (c.topo == 1 && !(c.bfm && c.bpresent[nodeIdx(c, i, j, 0)] > R(0))) {  // K faces
            const long long f0 = (static_cast<long long>(i) * nj + j) * (nk + 1) + k;
            const long long f1 = f0 + 1;
#pragma unroll
            for (int v = 0; v < 5; v++) {
                const R a = c.f[2].c[v][f0];
                Res.v[v] = (k == 0) ? Res.v[v] + a : Res.v[v] - a;
                Res.v[v] = Res.v[v] + c.f[2].c[v][f1];
            }
        }
        if (c.viscous) addViscousResidual(c, i, j, k, Res);
        if (hasSources(c)) {  // the stage input's primitives (and JST pressure) stored per node
            const S5<R> Wn = load5(c.W, q);
            const R pn = c.Wp ? CTBFM_LDS(c.Wp + q) : pressure_rho_u_et(gs, Wn.v[0], velOf(Wn), Wn.v[4]);
            applySourcesW<BX>(c, gs, Uin, i, j, k, q, Wn, pn, t, Res);
        }
        if (c.periodic && (k == 0 || k == nk - 1)) {
            const long long pq = (k == 0 ? 0 : c.n / nk) + static_cast<long long>(i) * nj + j;
            store5(c.Rp, pq, Res);
            continue;
        }
        if (c.viscous && c.wall[q]) noSlipResidual(Res);
        if (resOnly) {
            store5(Uout, q, Res);
            continue;
        }
        const R dt = c.dt_method == 1 ? dtg : (c.dt_method == 2 ? R(c.fixed_dt) : c.dt[q]);
        const R fac = alpha * dt / c.vol[q];
        const S5<R> Un = load5(c.U, q);
        S5<R> Un1;
        if (c.compensated) {
            const S5<R> Cn = load5(c.Uc, q);
            S5<R> Cn1;
#pragma unroll
            for (int v = 0; v < 5; v++) {
                const R y = -(Res.v[v] * fac) - Cn.v[v];
                const R s = Un.v[v] + y;
                Cn1.v[v] = (s - Un.v[v]) - y;
                Un1.v[v] = s;
            }
            if (last) store5(c.Uc, q, Cn1);
        } else {
#pragma unroll
            for (int v = 0; v < 5; v++) Un1.v[v] = Un.v[v] - Res.v[v] * fac;
        }
        store5(Uout, q, Un1);
        if (stage < c.nstages - 1) storePrim(c, q, Un1);
        if (last)
#pragma unroll
            for (int v = 0; v < 5; v++) acc[v] += static_cast<double>(Res.v[v]) * static_cast<double>(Res.v[v]);
    }
    if (last) {
        blockSum<5>(acc);
        if (threadIdx.x == 0)
#pragma unroll
            for (int v = 0; v < 5; v++) c.partial[tl.local * 5 + v] = acc[v];
    }
}

template <typename R, int FL, int BX>
__global__ void __launch_bounds__(256, (nodesMinBlocks<R>())) k_nodes(const DevCaseT<R>* cases, const Tile* tiles, int stage, int force) {
    __shared__ DevCaseT<R> c;
    Tile tl;
    if (!enter(cases, tiles, c, stage, force, tl, FL, BX)) return;
    b_nodes<R, FL, BX>(c, tl, stage);
}

// Solver::enforcePeriodicityOnResiduals (src/solver.cpp:1836-1853), the
// no-slip walls on the averaged residuals (:1856-1863), the update
// of the two periodic planes and Solver::enforcePeriodicityOnSolution
// (src/solver.cpp:2308-2327). One thread per (i, j) pair.
template <typename R>
__device__ __forceinline__ void b_periodic(const DevCaseT<R>& c, const Tile& tl, int stage) {
    const R dtg = R(c.ctl->dt_min);
    const bool resOnly = stage < 0;
    const bool last = !resOnly && stage == c.nstages - 1;
    const R alpha = resOnly ? R(0) : R(c.coeffs[stage]);
    R* const* Uout = stageOut(c, stage);
    const R cm = R(c.per_cos_m), sm = R(c.per_sin_m), cp = R(c.per_cos_p), sp = R(c.per_sin_p);
    const long long np = static_cast<long long>(c.ni) * c.nj;
    double acc[5] = {0, 0, 0, 0, 0};
    for (long long p = tl.start + threadIdx.x; p < tl.start + tl.count; p += blockDim.x) {
        const S5<R> R1 = load5(c.Rp, p), R2 = load5(c.Rp, np + p);
        S5<R> Ra = (R1 + rotState(R2, cm, sm)) * R(0.5);
        S5<R> Rb = rotState(Ra, cp, sp);
        const long long q0 = p * c.nk, q1 = p * c.nk + c.nk - 1;
        if (c.viscous) {  // Solver::enforceNoSlipWallsOnResiduals after the periodic average
            if (c.wall[q0]) noSlipResidual(Ra);
            if (c.wall[q1]) noSlipResidual(Rb);
        }
        if (resOnly) {
            store5(Uout, q0, Ra);
            store5(Uout, q1, Rb);
            continue;
        }
        const R dt0 = c.dt_method == 1 ? dtg : (c.dt_method == 2 ? R(c.fixed_dt) : c.dt[q0]);
        const R dt1 = c.dt_method == 1 ? dtg : (c.dt_method == 2 ? R(c.fixed_dt) : c.dt[q1]);
        const R f0 = alpha * dt0 / c.vol[q0];
        const R f1 = alpha * dt1 / c.vol[q1];
        S5<R> U0, U1;
        if (c.compensated) {
            const S5<R> A0 = load5(c.U, q0), A1 = load5(c.U, q1);
            const S5<R> C0 = load5(c.Uc, q0), C1 = load5(c.Uc, q1);
            S5<R> D0, D1;
#pragma unroll
            for (int v = 0; v < 5; v++) {
                const R y0 = -(Ra.v[v] * f0) - C0.v[v];
                U0.v[v] = A0.v[v] + y0;
                D0.v[v] = (U0.v[v] - A0.v[v]) - y0;
                const R y1 = -(Rb.v[v] * f1) - C1.v[v];
                U1.v[v] = A1.v[v] + y1;
                D1.v[v] = (U1.v[v] - A1.v[v]) - y1;
            }
            if (last) {
                const S5<R> Da = (D0 + rotState(D1, cm, sm)) * R(0.5);
                store5(c.Uc, q0, Da);
                store5(c.Uc, q1, rotState(Da, cp, sp));
            }
        } else {
            U0 = load5(c.U, q0) - Ra * f0;
            U1 = load5(c.U, q1) - Rb * f1;
        }
        const S5<R> Ua = (U0 + rotState(U1, cm, sm)) * R(0.5);
        const S5<R> Ub = rotState(Ua, cp, sp);
        store5(Uout, q0, Ua);
        store5(Uout, q1, Ub);
        if (stage < c.nstages - 1) {
            storePrim(c, q0, Ua);
            storePrim(c, q1, Ub);
        }
        if (last)
#pragma unroll
            for (int v = 0; v < 5; v++)
                acc[v] += static_cast<double>(Ra.v[v]) * static_cast<double>(Ra.v[v]) +
                          static_cast<double>(Rb.v[v]) * static_cast<double>(Rb.v[v]);
    }
    if (last) {
        blockSum<5>(acc);
        if (threadIdx.x == 0)
#pragma unroll
            for (int v = 0; v < 5; v++) c.partial[(c.node_tiles + tl.local) * 5 + v] = acc[v];
    }
}

template <typename R>
__global__ void __launch_bounds__(256) k_periodic(const DevCaseT<R>* cases, const Tile* tiles, int stage, int force) {
    __shared__ DevCaseT<R> c;
    Tile tl;
    if (!enter(cases, tiles, c, stage, force, tl)) return;
    b_periodic<R>(c, tl, stage);
}

// ------------------------------------------------------------ fused stage
#include "stage_fused.cuh"

// ------------------------------------------------------- Spalart-Allmaras
#include "sa.cuh"

// ------------------------------------------------------------- time step
// Solver::computeTimestepArray (src/solver.cpp:1531-1630):
// dt = CFL / (sum_d (|u . e_d| + a) / |e_d| + 4 nu sum_d 1 / |e_d|^2) over the
// dual-node edges, the viscous term only for viscous instances.
template <typename R, int FL>
__device__ __forceinline__ void b_dt(const DevCaseT<R>& c, const Tile& tl) {
    if (c.dt_method == 2) return;
    const Gas<R> gs{R(c.gamma), R(c.rgas), FL ? c.lut : nullptr};
    const R cfl = R(c.cfl);
    double mn = INFINITY;
    for (long long q = tl.start + threadIdx.x; q < tl.start + tl.count; q += blockDim.x) {
        const S5<R> W = primOf(load5(c.U, q));
        const V3<R> u = velOf(W);
        const R a = soundSpeed_rho_u_et(gs, W.v[0], u, W.v[4]);
        const V3<R> dI = v3(c.edge[0][q], c.edge[1][q], c.edge[2][q]);
        const V3<R> dJ = v3(c.edge[4][q], c.edge[5][q], c.edge[6][q]);
        const R ui = fabs(dot(u, dI)), uj = fabs(dot(u, dJ));
        R lc = (ui + a) / c.edge[3][q];
        lc += (uj + a) / c.edge[7][q];
        if (c.topo == 1) {
            const V3<R> dK = v3(c.edge[8][q], c.edge[9][q], c.edge[10][q]);
            lc += (fabs(dot(u, dK)) + a) / c.edge[11][q];
        }
        R dt;
        if (c.viscous) {  // 4 (nu + nu_t) sum_d 1/|e_d|^2, nu_t = 0
            const R mu = molecularViscosity(c, temperature_rho_u_et(gs, W.v[0], u, W.v[4]));
            const R nu = mu / W.v[0], nut = saEddy(c, W.v[0], q) / W.v[0];
            const R dsI = c.edge[3][q], dsJ = c.edge[7][q];
            R ih2 = R(1) / (dsI * dsI);
            ih2 += R(1) / (dsJ * dsJ);
            if (c.topo == 1) ih2 += R(1) / (c.edge[11][q] * c.edge[11][q]);
            dt = cfl / (lc + R(4) * (nu + nut) * ih2);
        } else {
            dt = cfl / lc;
        }
        c.dt[q] = dt;
        mn = fmin(mn, static_cast<double>(dt));
    }
    mn = blockMin(mn);
    if (threadIdx.x == 0) c.partial[(c.node_tiles + c.per_tiles) * 5 + tl.local] = mn;
}

template <typename R, int FL>
__global__ void __launch_bounds__(256) k_dt(const DevCaseT<R>* cases, const Tile* tiles, int force) {
    __shared__ DevCaseT<R> c;
    Tile tl;
    if (!enter(cases, tiles, c, 0, force, tl, FL)) return;
    b_dt<R, FL>(c, tl);
}

// ------------------------------------------------------ boundary integrals
// Solver::updateMassFlows (src/solver.cpp:1633-1649) and the mass-weighted
// total pressure / temperature integrals of Solver::updateTurboPerformance
// (src/solver.cpp:1652-1781), in double. Tile.local = 0..5: mass flow through
// plane `local`; 6, 7: Pt and Tt integrals over the inlet / outlet planes.
template <typename R>
__device__ __forceinline__ void planeExtent(const DevCaseT<R>& c, int b, int& na, int& nb) {
    if (b <= 1) { na = c.nj; nb = c.nk; }
    else if (b <= 3) { na = c.ni; nb = c.nk; }
    else { na = c.ni; nb = c.nj; }
}
template <typename R>
__device__ __forceinline__ long long planeNode(const DevCaseT<R>& c, int b, int a, int bb) {
    switch (b) {
        case 0: return nodeIdx(c, 0, a, bb);
        case 1: return nodeIdx(c, c.ni - 1, a, bb);
        case 2: return nodeIdx(c, a, 0, bb);
        case 3: return nodeIdx(c, a, c.nj - 1, bb);
        case 4: return nodeIdx(c, a, bb, 0);
        default: return nodeIdx(c, a, bb, c.nk - 1);
    }
}
template <typename R>
__device__ __forceinline__ int turboPlane(const DevCaseT<R>& c, int m) {
    switch (c.turbo_dir) {
        case 1: return m == 0 ? 1 : 0;
        case 2: return m == 0 ? 2 : 3;
        case 3: return m == 0 ? 3 : 2;
        default: return m == 0 ? 0 : 1;
    }
}

template <typename R, int FL>
__device__ __forceinline__ void b_bint(const DevCaseT<R>& c, const Tile& tl) {
    const Gas<double> gs{c.gamma, c.rgas, FL ? c.lut : nullptr};
    const int blk = tl.local;
    // in 2-D the K_START and K_END planes are the same nodes (with other
    // surface vectors): the plane-4 blocks sum both, K_END's mass flow in
    // their second sum, and the plane-5 blocks have nothing to do
    const bool pairK = blk == 4 && c.nk == 1;
    if (blk == 5 && c.nk == 1) return;
    const int plane = blk < 6 ? blk : turboPlane(c, blk - 6);
    int na, nb;
    planeExtent(c, plane, na, nb);
    const long long cnt = static_cast<long long>(na) * nb;
    const long long end = tl.start + tl.count < cnt ? tl.start + tl.count : cnt;
    double s[4] = {0.0, 0.0, 0.0, 0.0};
    for (long long e = tl.start + threadIdx.x; e < end; e += blockDim.x) {
        const int a = static_cast<int>(e / nb), bb = static_cast<int>(e % nb);
        const long long q = planeNode(c, plane, a, bb);
        const double sx = c.bsx[plane][e], sy = c.bsy[plane][e], sz = c.bsz[plane][e];
        const S5<double> Uq = state64(c, c.U, q);
        if (blk < 6) {
            s[0] += sx * Uq.v[1] + sy * Uq.v[2] + sz * Uq.v[3];
            if (pairK) s[1] += c.bsx[5][e] * Uq.v[1] + c.bsy[5][e] * Uq.v[2] + c.bsz[5][e] * Uq.v[3];
        } else {
            const S5<double> W = primOf(Uq);
            const double rho = W.v[0];
            const V3<double> u = velOf(W);
            const double P = totalPressure_rho_u_et(gs, rho, u, W.v[4]);
            const double T = totalTemperature_rho_u_et(gs, rho, u, W.v[4]);
            s[0] += sx * (rho * u.x * P) + sy * (rho * u.y * P) + sz * (rho * u.z * P);
            s[1] += sx * (rho * u.x * T) + sy * (rho * u.y * T) + sz * (rho * u.z * T);
            if (FL) {  // total enthalpy and entropy (src/solver.cpp:1732-1749)
                const double H = totalEnthalpy_rho_u_et(gs, rho, u, W.v[4]);
                const double S = entropy_rho_u_et(gs, rho, u, W.v[4]);
                s[2] += sx * (rho * u.x * H) + sy * (rho * u.y * H) + sz * (rho * u.z * H);
                s[3] += sx * (rho * u.x * S) + sy * (rho * u.y * S) + sz * (rho * u.z * S);
            }
        }
    }
    blockSum<4>(s);
    if (threadIdx.x == 0) {
        double* part = c.bint_part + (c.bint_off[blk] + tl.start / kBintChunk) * 4;
#pragma unroll
        for (int v = 0; v < 4; v++) part[v] = s[v];
    }
}

// The boundary integrals from their chunk partials, added in chunk order
// (one thread; k_pre after k_bint).
template <typename R>
__device__ __forceinline__ void combineBoundaryIntegrals(const DevCaseT<R>& c) {
    Control* ctl = c.ctl;
    for (int b = 0; b < 8; b++) {
        double s[4] = {0.0, 0.0, 0.0, 0.0};
        const bool pairK = b == 5 && c.nk == 1;  // K_END summed by the K_START blocks (second sum)
        const int src = pairK ? 4 : b;
        for (int k = c.bint_off[src]; k < c.bint_off[src + 1]; k++)
#pragma unroll
            for (int v = 0; v < 4; v++) s[v] += c.bint_part[k * 4 + v];
        if (pairK) {
            ctl->massflow[5] = s[1];
        } else if (b < 6) {
            ctl->massflow[b] = s[0];
        } else {
            ctl->pt_int[b - 6] = s[0];
            ctl->tt_int[b - 6] = s[1];
            ctl->ht_int[b - 6] = s[2];
            ctl->s_int[b - 6] = s[3];
        }
    }
}

template <typename R, int FL>
__global__ void __launch_bounds__(256) k_bint(const DevCaseT<R>* cases, const Tile* tiles, int force) {
    __shared__ DevCaseT<R> c;
    Tile tl;
    if (!enter(cases, tiles, c, 0, force, tl, FL)) return;
    b_bint<R, FL>(c, tl);
}

// ------------------------------------------------------------ pre-stage
// Global min(dt); turbo performance with FluidIdeal::computeTotalEfficiency_PRtt_TRt
// (src/fluid_ideal.cpp:179-191); GreitzerModel::computePlenumPressure
// (src/greitzer_model.cpp:36-56); Solver::updateRadialProfiles
// (src/solver.cpp:2688-2787) with integrateRadialEquilibrium
// (src/math_utils.cpp:141-170). All double. One block per instance.
template <typename R>
__device__ __forceinline__ void b_pre(const DevCaseT<R>& c, const Tile& tl, int forceTurbo, int dtpart,
                                      int profiles) {
    Control* ctl = c.ctl;
    if (!dtpart) {
    } else if (c.dt_method == 2) {
        if (threadIdx.x == 0) ctl->dt_min = c.fixed_dt;
    } else {
        double mn = INFINITY;
        const double* part = c.partial + (c.node_tiles + c.per_tiles) * 5;
        for (int b = threadIdx.x; b < c.node_tiles; b += blockDim.x) mn = fmin(mn, part[b]);
        mn = blockMin(mn);
        if (threadIdx.x == 0) ctl->dt_min = mn;
    }
    if (threadIdx.x != 0) return;
    if (c.need_turbo || forceTurbo) {
        combineBoundaryIntegrals(c);
        const int p0 = turboPlane(c, 0), p1 = turboPlane(c, 1);
        double mflow = 0.5 * (fabs(ctl->massflow[p0]) + fabs(ctl->massflow[p1]));
        if (c.topo == 2) mflow *= 2.0 * M_PI / c.wedge;
        else if (c.per_angle_deg != 0.0) mflow *= 360.0 / c.per_angle_deg;
        double pt[2], tt[2], ht[2], en[2];
        for (int m = 0; m < 2; m++) {
            double mf = ctl->massflow[m == 0 ? p0 : p1];
            if (fabs(mf) < 1e-12) mf = (mf >= 0.0 ? 1e-12 : -1e-12);
            pt[m] = ctl->pt_int[m] / mf;
            tt[m] = ctl->tt_int[m] / mf;
            ht[m] = ctl->ht_int[m] / mf;
            en[m] = ctl->s_int[m] / mf;
        }
        const double pr = (fabs(pt[0]) > 1e-12) ? pt[1] / pt[0] : 1.0;
        const double tr = (fabs(tt[0]) > 1e-12) ? tt[1] / tt[0] : 1.0;
        double eta;
        if (c.lut) {
            // src/solver.cpp:1768-1776 with FluidBase::computeTotalEfficiency_h
            // (include/fluid_base.hpp:145-157)
            const double hOutS = lutEnthalpy_p_s(*c.lut, pt[1], en[0]);
            const double dh = ht[1] - ht[0], dhs = hOutS - ht[0];
            if (fabs(dh) < 1e-12) eta = 1.0;
            else if (dh >= 0.0) eta = dhs / dh;
            else eta = (fabs(dhs) < 1e-12) ? 1.0 : dh / dhs;
        } else {
            const double dT = tr - 1.0;
            const double dTs = pow(pr, (c.gamma - 1.0) / c.gamma) - 1.0;
            if (fabs(dT) < 1e-12) eta = 1.0;
            else if (dT >= 0.0) eta = dTs / dT;
            else eta = (fabs(dTs) < 1e-12) ? 1.0 : dT / dTs;
        }
        ctl->turbo[0] = mflow;
        ctl->turbo[1] = pr;
        ctl->turbo[2] = tr;
        ctl->turbo[3] = eta;
        ctl->has_turbo = 1;
        if (c.bfm_model == 5) {  // SourceBFMChima::computeBodyForceSource (src/source_bfm_chima.cpp:33-41)
            ctl->chima_turn = linearInterpolation(c.chima_mf, c.chima_turn, c.chima_n, mflow);
            ctl->chima_loss = linearInterpolation(c.chima_mf, c.chima_loss, c.chima_n, mflow);
        }
    }
    if (!profiles || (c.nprofiles == 0 && !c.greitzer)) return;
    if (c.greitzer) {
        ctl->gz_min = ctl->turbo[0];
        ctl->gz_t += c.fixed_dt;
        // computeSoundSpeed_p_T: FluidIdeal sqrt(gamma R T), FluidReal the (p, T) table
        const double a = c.lut ? lutInterp(c.lut->pt[kPtA], ctl->gz_p, ctl->gz_T) : sqrt(c.gamma * c.rgas * ctl->gz_T);
        const double np = ctl->gz_p + c.fixed_dt * a * a / c.plenum_volume * (ctl->gz_min - ctl->gz_mout);
        ctl->gz_p = np;
        const double dp = ctl->gz_p - c.ambient_p;
        ctl->gz_mout = (dp > 0.0) ? sqrt(dp / c.throttle_kt) : 0.0;
        ctl->hub_p = ctl->gz_p;
    }
    for (int m = 0; m < c.nprofiles; m++) {
        double* p = c.prof_p + c.prof_off[m];
        const double* r = c.prof_r + c.prof_off[m];
        const int n = c.prof_n[m];
        if (c.greitzer) {
        } else if (c.prof_type[m] == kBcThrottle) {
            ctl->hub_p = c.inlet_pt + c.prof_kt[m] * ctl->turbo[0] * ctl->turbo[0];
        } else if (c.prof_type[m] == kBcMassFlow) {
            // mass-flow controller (src/solver.cpp:2734-2770): relax the hub
            // pressure by the relative mass-flow error, clamped
            double cur = fabs(ctl->massflow[c.prof_plane[m]]);
            if (c.topo == 2) cur *= 2.0 * M_PI / c.wedge;
            else if (c.per_angle_deg != 0.0) cur *= 360.0 / c.per_angle_deg;
            const double err = (cur - c.prof_mf[m]) / c.prof_mf[m];
            double dp = c.prof_relax[m] * err;
            dp = dp < -c.mf_max_change ? -c.mf_max_change : (c.mf_max_change < dp ? c.mf_max_change : dp);
            double p0 = p[0];
            if (p0 <= 0.0) p0 = c.init_p > 0.0 ? c.init_p : 101325.0;
            const double hub = p0 * (1.0 + dp);
            ctl->hub_p = hub < 100.0 ? 100.0 : hub;
        } else if (c.prof_type[m] == kBcRadialEq) {
            ctl->hub_p = p[0];
        }
        if (c.prof_fill[m]) {  // no radial equilibrium: the hub value everywhere
            for (int jj = 0; jj < n; jj++) p[jj] = ctl->hub_p;
            continue;
        }
        // sample density and |u_theta| at (prof_i, j, 0) and integrate dp/dr
        double rho1 = 0, ut1 = 0;
        p[0] = ctl->hub_p;
        for (int jj = 0; jj < n; jj++) {
            const long long q = nodeIdx(c, c.prof_i[m], c.prof_j0[m] + jj, 0);
            const S5<double> W = primOf(state64(c, c.U, q));
            const V3<double> vc = cylOfCart(velOf(W), c.cost64[q], c.sint64[q]);
            const double rho2 = W.v[0], ut2 = fabs(vc.z);
            if (jj > 0) {
                const double r1 = r[jj - 1], r2 = r[jj];
                const double dr = r2 - r1;
                const double d1 = rho1 * ut1 * ut1 / r1;
                const double d2 = rho2 * ut2 * ut2 / r2;
                p[jj] = p[jj - 1] + 0.5 * (d1 + d2) * dr;
            }
            rho1 = rho2;
            ut1 = ut2;
        }
    }
}

template <typename R>
__global__ void __launch_bounds__(256) k_pre(const DevCaseT<R>* cases, const Tile* tiles, int forceTurbo, int dtpart,
                                             int profiles, int force) {
    __shared__ DevCaseT<R> c;
    Tile tl;
    if (!enter(cases, tiles, c, 0, force, tl)) return;
    b_pre<R>(c, tl, forceTurbo, dtpart, profiles);
}

// ------------------------------------------------------------- finalize
// Solver::computeLogResidualNorm (src/solver.cpp:1488-1508),
// printInfoResiduals' initial maximum (src/solver.cpp:1426-1439),
// Solver::checkConvergence (src/solver.cpp:2985-3015) and the time advance
// t += min(dt) (src/solver.cpp:1389). One block per instance.
// fusedMode 1: instances that ran the fused stage kernel have their norm
// partials in its region (one per box) instead of the node tiles'.
template <typename R>
__device__ __forceinline__ void b_finalize(const DevCaseT<R>& c, const Tile& tl, int fusedMode) {
    Control* ctl = c.ctl;
    const bool fz = fusedMode && c.fuse_ok;
    const int na = fz ? c.nboxes : c.node_tiles;
    const double* pa =
        fz ? c.partial + (static_cast<long long>(c.node_tiles) + c.per_tiles) * 5 + c.node_tiles : c.partial;
    const double* pp = c.partial + static_cast<long long>(c.node_tiles) * 5;  // periodic planes
    const int nparts = na + (c.periodic ? c.per_tiles : 0);
    double s[5] = {0, 0, 0, 0, 0};
    for (int b = threadIdx.x; b < nparts; b += blockDim.x) {
        const double* src = b < na ? pa + b * 5 : pp + (b - na) * 5;
#pragma unroll
        for (int v = 0; v < 5; v++) s[v] += src[v];
    }
    blockSum<5>(s);
    if (threadIdx.x != 0) return;
    const long long it = ctl->it + 1;
    ctl->t += ctl->dt_min;
    double lr[5];
    bool diverged = false;
    for (int v = 0; v < 5; v++) {
        const double nrm = sqrt(s[v]);
        if (isnan(nrm) || isinf(nrm)) diverged = true;
        lr[v] = (nrm >= 2.2250738585072014e-308) ? log10(nrm / static_cast<double>(c.n)) : -16.0;
        if (lr[v] < -16.0) lr[v] = -16.0;
        ctl->lognorm[v] = lr[v];
    }
    ctl->it = it;
    if (diverged) {
        ctl->status = 2;
        return;
    }
    if (!ctl->has_init) {
        for (int v = 0; v < 5; v++) ctl->init_log[v] = lr[v];
        ctl->has_init = 1;
    } else if (it <= 5) {
        for (int v = 0; v < 5; v++) ctl->init_log[v] = rmax(ctl->init_log[v], lr[v]);
    }
    const long long row = it - 1 - ctl->hist_base;
    if (c.hist && row >= 0 && row < c.hist_cap) {
        double* h = c.hist + row * kHistWidth;
        for (int v = 0; v < 5; v++) h[v] = lr[v];
        for (int b = 0; b < 6; b++) h[5 + b] = ctl->massflow[b];
        for (int b = 0; b < 4; b++) h[11 + b] = c.need_turbo ? ctl->turbo[b] : 0.0;
        h[15] = ctl->hub_p;
        h[16] = ctl->t;
    }
    if (c.steady) {
        bool conv = true;
        double drop = INFINITY;
        for (int v = 0; v < 5; ++v) {
            if (v == 3 && c.topo != 1 && c.topo != 2) continue;
            if (ctl->init_log[v] <= -15.99) continue;
            if (lr[v] <= -15.0) continue;
            drop = fmin(drop, ctl->init_log[v] - lr[v]);
            if (lr[v] >= ctl->init_log[v] - static_cast<double>(c.drop)) conv = false;
        }
        if (conv) ctl->status = 1;
        if (it <= 5) {
            ctl->best_drop = 0.0;
            ctl->drop_mark = 0.0;
            ctl->it_best = it;
        } else {
            ctl->best_drop = fmax(ctl->best_drop, drop);
            if (drop >= ctl->drop_mark + 0.05) {
                ctl->drop_mark = drop;
                ctl->it_best = it;
            }
        }
    }
}

template <typename R>
__global__ void __launch_bounds__(256) k_finalize(const DevCaseT<R>* cases, const Tile* tiles, int force,
                                                  int fusedMode) {
    __shared__ DevCaseT<R> c;
    Tile tl;
    if (!enter(cases, tiles, c, 0, force, tl)) return;
    b_finalize<R>(c, tl, fusedMode);
}

// Copies every instance's control block into one array (one D2H copy for a
// whole batch).
template <typename R>
__global__ void k_gather_control(const DevCaseT<R>* cases, int m, Control* out) {
    gridDependency();
    const int i = blockIdx.x;
    if (i >= m) return;
    const int* src = reinterpret_cast<const int*>(cases[i].ctl);
    int* dst = reinterpret_cast<int*>(out + i);
    for (int w = threadIdx.x; w < static_cast<int>(sizeof(Control) / 4); w += blockDim.x) dst[w] = src[w];
}

// Sets each instance's iteration limit (n more iterations, at most its
// N_ITERATIONS, like the reference's loop bound) and history origin.
template <typename R>
__global__ void k_set_limits(const DevCaseT<R>* cases, int m, long long n) {
    gridDependency();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    Control* ctl = cases[i].ctl;
    const long long stop = ctl->it + n;
    ctl->it_stop = stop < cases[i].max_it ? stop : cases[i].max_it;
    ctl->hist_base = ctl->it;
}

}  // namespace

// ------------------------------------------------------------- launchers

#ifndef CTBFM_PDL
#define CTBFM_PDL 1
#endif

// Every kernel is launched with programmatic stream serialization (see
// gridDependency); launch errors surface through cudaGetLastError.
template <typename... P, typename... A>
void launchK(void (*k)(P...), unsigned grid, unsigned block, cudaStream_t s, A... a) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = CTBFM_PDL;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    (void)cudaLaunchKernelEx(&cfg, k, static_cast<P>(a)...);
}

template <typename R>
cudaError_t Launcher<R>::setLimits(const BatchView<R>& b, long long n, cudaStream_t s) {
    launchK(k_set_limits<R>, (b.m + 127) / 128, 128, s, b.cases, b.m, n);
    return cudaGetLastError();
}

template <typename R>
cudaError_t Launcher<R>::gatherControl(const BatchView<R>& b, Control* out, cudaStream_t s) {
    if (b.m) launchK(k_gather_control<R>, b.m, 64, s, b.cases, b.m, out);
    return cudaGetLastError();
}

template <typename R>
cudaError_t Launcher<R>::boundaryIntegrals(const BatchView<R>& b, bool all, int force, cudaStream_t s) {
    const TileList& t = all ? b.bintAll : b.bint;
    if (t.n && b.ideal) launchK(k_bint<R, 0>, t.n, 256, s, b.cases, t.tiles, force);
    if (t.n && b.real) launchK(k_bint<R, 1>, t.n, 256, s, b.cases, t.tiles, force);
    return cudaGetLastError();
}

template <typename R>
cudaError_t Launcher<R>::timeStep(const BatchView<R>& b, int force, cudaStream_t s) {
    if (b.node.n && b.ideal) launchK(k_dt<R, 0>, b.node.n, 256, s, b.cases, b.node.tiles, force);
    if (b.node.n && b.real) launchK(k_dt<R, 1>, b.node.n, 256, s, b.cases, b.node.tiles, force);
    return cudaGetLastError();
}

template <typename R>
cudaError_t Launcher<R>::pre(const BatchView<R>& b, bool forceTurbo, bool dtpart, bool profiles, int force,
                             cudaStream_t s) {
    if (b.inst.n)
        launchK(k_pre<R>, b.inst.n, 256, s, b.cases, b.inst.tiles, forceTurbo ? 1 : 0, dtpart ? 1 : 0, profiles ? 1 : 0,
                                          force);
    return cudaGetLastError();
}

template <typename R>
cudaError_t Launcher<R>::prim(const BatchView<R>& b, int stage, int force, cudaStream_t s) {
    const TileList& t = b.split[b.fusedMode].node;
    if (t.n) launchK(k_prim<R>, t.n, 256, s, b.cases, t.tiles, stage, force);
    return cudaGetLastError();
}

namespace {
template <int DIR, int SCHEME, int FL, typename R>
void launchFaceSets(const BatchView<R>& b, int stage, int force, cudaStream_t s) {
    const TileList* t = b.split[b.fusedMode].face[DIR][SCHEME];
    if (t[0].n) launchK(k_faces<DIR, SCHEME, R, FL, 0>, t[0].n, 256, s, b.cases, t[0].tiles, stage, force);
    if (t[1].n) launchK(k_faces<DIR, SCHEME, R, FL, 1>, t[1].n, 256, s, b.cases, t[1].tiles, stage, force);
    if (t[2].n) launchK(k_faces<DIR, SCHEME, R, FL, 2>, t[2].n, 256, s, b.cases, t[2].tiles, stage, force);
}
template <int FL, typename R>
void launchFaces(const BatchView<R>& b, int dir, int stage, int force, cudaStream_t s) {
    if (dir == 0) {
        launchFaceSets<0, 0, FL>(b, stage, force, s);
        launchFaceSets<0, 1, FL>(b, stage, force, s);
    } else if (dir == 1) {
        launchFaceSets<1, 0, FL>(b, stage, force, s);
        launchFaceSets<1, 1, FL>(b, stage, force, s);
    } else {
        launchFaceSets<2, 0, FL>(b, stage, force, s);
        launchFaceSets<2, 1, FL>(b, stage, force, s);
    }
}
}  // namespace

template <typename R>
cudaError_t Launcher<R>::faces(const BatchView<R>& b, int dir, int stage, int force, cudaStream_t s) {
    if (b.ideal) launchFaces<0>(b, dir, stage, force, s);
    if (b.real) launchFaces<1>(b, dir, stage, force, s);
    return cudaGetLastError();
}

template <typename R>
cudaError_t Launcher<R>::viscous(const BatchView<R>& b, int stage, int force, cudaStream_t s) {
    if (!b.viscous) return cudaSuccess;
    if (b.vnode.n && b.ideal) launchK(k_grad<R, 0>, b.vnode.n, 256, s, b.cases, b.vnode.tiles, stage, force);
    if (b.vnode.n && b.real) launchK(k_grad<R, 1>, b.vnode.n, 256, s, b.cases, b.vnode.tiles, stage, force);
    if (b.ideal) {
        if (b.vface[0].n) launchK(k_vfaces<0, R, 0>, b.vface[0].n, 256, s, b.cases, b.vface[0].tiles, stage, force);
        if (b.vface[1].n) launchK(k_vfaces<1, R, 0>, b.vface[1].n, 256, s, b.cases, b.vface[1].tiles, stage, force);
        if (b.vface[2].n) launchK(k_vfaces<2, R, 0>, b.vface[2].n, 256, s, b.cases, b.vface[2].tiles, stage, force);
    }
    if (b.real) {
        if (b.vface[0].n) launchK(k_vfaces<0, R, 1>, b.vface[0].n, 256, s, b.cases, b.vface[0].tiles, stage, force);
        if (b.vface[1].n) launchK(k_vfaces<1, R, 1>, b.vface[1].n, 256, s, b.cases, b.vface[1].tiles, stage, force);
        if (b.vface[2].n) launchK(k_vfaces<2, R, 1>, b.vface[2].n, 256, s, b.cases, b.vface[2].tiles, stage, force);
    }
    return cudaGetLastError();
}

template <typename R>
cudaError_t Launcher<R>::nodes(const BatchView<R>& b, int stage, int force, cudaStream_t s) {
    const TileList& t = b.split[b.fusedMode].node;
    if (t.n && b.ideal && b.bfmCommon) launchK(k_nodes<R, 0, 0>, t.n, 256, s, b.cases, t.tiles, stage, force);
    if (t.n && b.real && b.bfmCommon) launchK(k_nodes<R, 1, 0>, t.n, 256, s, b.cases, t.tiles, stage, force);
    if (t.n && b.ideal && b.bfmRare) launchK(k_nodes<R, 0, 1>, t.n, 256, s, b.cases, t.tiles, stage, force);
    if (t.n && b.real && b.bfmRare) launchK(k_nodes<R, 1, 1>, t.n, 256, s, b.cases, t.tiles, stage, force);
    return cudaGetLastError();
}

template <typename R>
size_t Launcher<R>::fusedSmemBytes(int bi, int bj, int bk, int topo, int scheme) {
    FusedBox b;
    fusedLayout(bi, bj, bk, topo == 1, b);
    return (static_cast<size_t>(fusedNodeFields(scheme)) * b.nW + 5 * static_cast<size_t>(b.nfI + b.nfJ + b.nfK)) *
           sizeof(R);
}

namespace {
// Dynamic shared memory beyond the default 48 KB must be allowed per kernel
// and device (its largest size so far; k_stage blocks of smaller instances
// use less).
template <typename R, int SCHEME, int FL>
cudaError_t launchStage(const BatchView<R>& b, const TileList& t, int stage, int force, cudaStream_t s) {
    constexpr int kDevices = 64;
    static std::mutex mu;
    static size_t allowed[kDevices] = {};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kDevices) return cudaErrorInvalidDevice;
    {
        std::lock_guard<std::mutex> lock(mu);
        if (b.fusedSmem > allowed[dev]) {
            e = cudaFuncSetAttribute(k_stage<R, SCHEME, FL>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     static_cast<int>(b.fusedSmem));
            if (e != cudaSuccess) return e;
            allowed[dev] = b.fusedSmem;
        }
    }
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(t.n);
    cfg.blockDim = dim3(kFusedBoxNodes);
    cfg.dynamicSmemBytes = b.fusedSmem;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = CTBFM_PDL;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, k_stage<R, SCHEME, FL>, b.cases, t.tiles, stage, force);
}
}  // namespace

template <typename R>
cudaError_t Launcher<R>::fused(const BatchView<R>& b, int stage, int force, cudaStream_t s) {
    if (!b.fusedMode) return cudaSuccess;
    cudaError_t e = cudaSuccess;
    for (int sc = 0; sc < 2 && e == cudaSuccess; sc++) {
        const TileList& t = b.fbox[sc];
        if (!t.n) continue;
        if (sc == 0) {
            if (b.ideal && e == cudaSuccess) e = launchStage<R, 0, 0>(b, t, stage, force, s);
            if (b.real && e == cudaSuccess) e = launchStage<R, 0, 1>(b, t, stage, force, s);
        } else {
            if (b.ideal && e == cudaSuccess) e = launchStage<R, 1, 0>(b, t, stage, force, s);
            if (b.real && e == cudaSuccess) e = launchStage<R, 1, 1>(b, t, stage, force, s);
        }
    }
    return e != cudaSuccess ? e : cudaGetLastError();
}

template <typename R>
cudaError_t Launcher<R>::periodic(const BatchView<R>& b, int stage, int force, cudaStream_t s) {
    if (b.per.n) launchK(k_periodic<R>, b.per.n, kPeriodicTile, s, b.cases, b.per.tiles, stage, force);
    return cudaGetLastError();
}

template <typename R>
cudaError_t Launcher<R>::finalize(const BatchView<R>& b, int force, cudaStream_t s) {
    if (b.inst.n) launchK(k_finalize<R>, b.inst.n, 256, s, b.cases, b.inst.tiles, force, b.fusedMode);
    return cudaGetLastError();
}

template <typename R>
cudaError_t Launcher<R>::stage(const BatchView<R>& b, int stage, int force, cudaStream_t s) {
    // later stages read the primitives the previous stage's node kernels stored
    cudaError_t e = stage <= 0 ? prim(b, stage, force, s) : cudaSuccess;
    for (int d = 0; d < 3 && e == cudaSuccess; d++) e = faces(b, d, stage, force, s);
    if (e == cudaSuccess) e = viscous(b, stage, force, s);
    if (e == cudaSuccess) e = nodes(b, stage, force, s);
    if (e == cudaSuccess) e = fused(b, stage, force, s);
    if (e == cudaSuccess) e = periodic(b, stage, force, s);
    return e;
}

template <typename R>
cudaError_t Launcher<R>::turbulence(const BatchView<R>& b, cudaStream_t s) {
    if (!b.sa || !b.sanode.n) return cudaSuccess;
    const TileList& n = b.sanode;
    const TileList& m = b.sainst;
    launchK(k_prim<R>, n.n, 256, s, b.cases, n.tiles, 0, 0);
    launchK(k_grad<R, 0>, n.n, 256, s, b.cases, n.tiles, 0, 0);
    launchK(k_sa_bc<R>, m.n, 256, s, b.cases, m.tiles, 0);
    launchK(k_sa_prep<R, 0>, n.n, 256, s, b.cases, n.tiles, 0);
    launchK(k_sa_res<R>, n.n, 256, s, b.cases, n.tiles, 0);
    launchK(k_sa_sweep<R, 1>, m.n, 1024, s, b.cases, m.tiles, 0);
    launchK(k_sa_sweep<R, 0>, m.n, 1024, s, b.cases, m.tiles, 0);
    launchK(k_sa_update<R>, n.n, 256, s, b.cases, n.tiles, 0);
    launchK(k_sa_bc<R>, m.n, 256, s, b.cases, m.tiles, 0);
    return cudaGetLastError();
}

template <typename R>
cudaError_t Launcher<R>::iteration(const BatchView<R>& b, int nstages, cudaStream_t s) {
    cudaError_t e = boundaryIntegrals(b, false, 0, s);
    if (e == cudaSuccess) e = timeStep(b, 0, s);
    if (e == cudaSuccess) e = pre(b, false, true, true, 0, s);
    if (e == cudaSuccess) e = turbulence(b, s);
    for (int st = 0; st < nstages && e == cudaSuccess; st++) e = stage(b, st, 0, s);
    if (e == cudaSuccess) e = finalize(b, 0, s);
    return e;
}

}  // namespace ctbfm
