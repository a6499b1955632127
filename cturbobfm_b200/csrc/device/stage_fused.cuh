// Fused stage kernel k_stage: one Runge-Kutta stage of an instance's
// interior (face fluxes, residual assembly, sources, update and residual-norm
// partials) in one launch, included by kernels_impl.cuh inside its anonymous
// namespace (it uses enter(), boundaryFlux(), blockSum() and the stage
// buffers defined there).
//
// A block owns a box of nodes (c.fbox: extent along i, j, k; at most 256
// nodes, one per thread). It
//   1. converts the stage input of the box and of a cross-shaped halo of two
//      nodes along each swept direction into primitives in shared memory
//      (plus, for JST, each node's pressure and spectral radius |u| + a),
//      stored compactly: the box, then the I, J and K halo slabs;
//   2. evaluates every face of the box's nodes, I, J and K faces as one pool
//      shared by all threads (faces on the box's edges are evaluated by both
//      neighbouring boxes), into shared memory; one copy of the flux code
//      serves the three directions;
//   3. adds each node's start and end face of each direction to its residual
//      in the order of Solver::computeResiduals (src/solver.cpp:1783-1833),
//      then applies the sources, the update U(k) = U^n - alpha dt/V R (Kahan-
//      compensated in float) and the residual-norm partials, as k_nodes does.
// Faces whose four stencil nodes are interior read the shared-memory
// primitives; boundary faces and faces next to a boundary or a periodic seam
// go through fusedSideFlux, which reads the conservative states from global
// memory exactly as k_faces does. In FP64 every face flux and every residual
// is the same value, bit for bit, as in the split stage (k_prim, k_faces,
// k_nodes): only where the intermediate values live changes (shared memory
// instead of HBM).
#pragma once

// Box geometry of one block: extent, origin, and the compact layout of the
// primitives in shared memory (box nodes, then the halo slabs of two nodes on
// both sides along I, J and, in 3-D, K; halo corners are not stored).
struct FusedBox {
    int bi, bj, bk;               // box extent
    int oi, oj, ok;               // origin (global node indices)
    int baseI, baseJ, baseK, nW;  // offsets of the halo slabs, stored nodes
    int nfI, nfJ, nfK;            // faces per direction
};

CTBFM_HD inline void fusedLayout(int bi, int bj, int bk, bool three, FusedBox& b) {
    b.bi = bi;
    b.bj = bj;
    b.bk = bk;
    b.oi = b.oj = b.ok = 0;
    b.baseI = bi * bj * bk;
    b.baseJ = b.baseI + 4 * bj * bk;
    b.baseK = b.baseJ + bi * 4 * bk;
    b.nW = b.baseK + (three ? bi * bj * 4 : 0);
    b.nfI = (bi + 1) * bj * bk;
    b.nfJ = bi * (bj + 1) * bk;
    b.nfK = three ? bi * bj * (bk + 1) : 0;
}

// Shared-memory fields per stored node: primitives (5), and for JST the
// node's pressure and spectral radius.
CTBFM_HD constexpr int fusedNodeFields(int scheme) { return scheme == 0 ? 7 : 5; }

// Slot of local node (ii, jj, kk) (at most one coordinate outside the box).
__device__ __forceinline__ int fusedSlot(const FusedBox& b, int ii, int jj, int kk) {
    if (ii < 0 || ii >= b.bi) return b.baseI + ((ii < 0 ? ii + 2 : ii - b.bi + 2) * b.bj + jj) * b.bk + kk;
    if (jj < 0 || jj >= b.bj) return b.baseJ + (ii * 4 + (jj < 0 ? jj + 2 : jj - b.bj + 2)) * b.bk + kk;
    if (kk < 0 || kk >= b.bk) return b.baseK + (ii * b.bj + jj) * 4 + (kk < 0 ? kk + 2 : kk - b.bk + 2);
    return (ii * b.bj + jj) * b.bk + kk;
}

// Local node of slot p (the inverse of fusedSlot).
__device__ __forceinline__ void fusedNodeOf(const FusedBox& b, int p, int& ii, int& jj, int& kk) {
    if (p < b.baseI) {
        kk = p % b.bk;
        jj = (p / b.bk) % b.bj;
        ii = p / (b.bk * b.bj);
    } else if (p < b.baseJ) {
        const int q = p - b.baseI;
        kk = q % b.bk;
        const int t = q / b.bk;
        jj = t % b.bj;
        const int h = t / b.bj;
        ii = h < 2 ? h - 2 : b.bi + h - 2;
    } else if (p < b.baseK) {
        const int q = p - b.baseJ;
        kk = q % b.bk;
        const int t = q / b.bk;
        const int h = t % 4;
        ii = t / 4;
        jj = h < 2 ? h - 2 : b.bj + h - 2;
    } else {
        const int q = p - b.baseK;
        const int h = q % 4;
        const int t = q / 4;
        jj = t % b.bj;
        ii = t / b.bj;
        kk = h < 2 ? h - 2 : b.bk + h - 2;
    }
}

// Resident blocks of 256 threads per SM asked of k_stage (its register
// budget), as for the face kernels: double JST 2, otherwise 3.
template <int SCHEME, typename R>
constexpr int fusedMinBlocks() {
    return (sizeof(R) == 8 && SCHEME == 0) ? 2 : 3;
}

// Boundary faces and faces next to a boundary or a periodic seam of
// direction d, exactly as k_faces computes them (conservative states from
// global memory); returns flux * |S|. Not inlined: these faces are few, and
// their code stays out of the fused kernel's registers and instruction cache.
template <int SCHEME, typename R>
__device__ __noinline__ S5<R> fusedSideFlux(const DevCaseT<R>& c, Gas<R> gs, R* const* U, int d, int fi, int fj,
                                            int fk, long long f, long long it) {
    const long long st = d == 0 ? static_cast<long long>(c.nj) * c.nk : (d == 1 ? c.nk : 1);
    const int nlast = d == 0 ? c.ni : (d == 1 ? c.nj : c.nk);
    const int dface = d == 0 ? fi : (d == 1 ? fj : fk);
    const DevFacesT<R>& F = c.f[d];
    V3<R> n = v3(__ldg(F.nx + f), __ldg(F.ny + f), __ldg(F.nz + f));
    const R area = __ldg(F.area + f);
    S5<R> flux;
    if (dface == 0 || dface == nlast) {
        const int side = dface == 0 ? 0 : 1;
        const int ni_ = d == 0 ? (side ? c.ni - 1 : 0) : fi;
        const int nj_ = d == 1 ? (side ? c.nj - 1 : 0) : fj;
        const int nk_ = d == 2 ? (side ? c.nk - 1 : 0) : fk;
        const long long q = nodeIdx(c, ni_, nj_, nk_);
        if (side == 0) n = -n;
        int pidx;
        if (d == 0) pidx = c.mapI[(static_cast<long long>(side) * c.nj + fj) * c.nk + fk];
        else if (d == 1) pidx = c.mapJ[(static_cast<long long>(fi) * 2 + side) * c.nk + fk];
        else pidx = c.mapK[(static_cast<long long>(fi) * c.nj + fj) * 2 + side];
        const long long qth =
            nodeIdx(c, fi < c.ni ? fi : c.ni - 1, fj < c.nj ? fj : c.nj - 1, fk < c.nk ? fk : c.nk - 1);
        const bool onWall = c.viscous && fi < c.ni && fj < c.nj && fk < c.nk && c.wall[nodeIdx(c, fi, fj, fk)];
        flux = boundaryFlux<SCHEME>(c, gs, pidx, load5(U, q), n, qth, fj, it, onWall);
    } else {
        const long long qR = nodeIdx(c, fi, fj, fk);
        const long long qL = qR - st;
        const S5<R> Ul = load5(U, qL), Ur = load5(U, qR);
        S5<R> Ull, Urr;
        if (d == 2 && c.periodic) {
            if (dface == 1) {
                Ull = rotState(load5(U, nodeIdx(c, fi, fj, c.nk - 2)), R(c.per_cos_m), R(c.per_sin_m));
                Urr = load5(U, qR + 1);
            } else {  // dface == nlast - 1
                Ull = load5(U, qR - 2);
                Urr = rotState(load5(U, nodeIdx(c, fi, fj, 1)), R(c.per_cos_p), R(c.per_sin_p));
            }
        } else {
            if (dface == 1) {
                Ull = Ul - (Ur - Ul);
                Urr = load5(U, qR + st);
            } else {  // dface == nlast - 1
                Ull = load5(U, qL - st);
                Urr = Ur + (Ur - Ul);
            }
        }
        if (SCHEME == 0) flux = fluxJst(gs, Ull, Ul, Ur, Urr, n);
        else flux = fluxRoe(gs, c.muscl, c.limiter, Ull, Ul, Ur, Urr, n);
    }
    S5<R> out;
#pragma unroll
    for (int v = 0; v < 5; v++) out.v[v] = flux.v[v] * area;
    return out;
}

template <typename R, int SCHEME, int FL>
__global__ void __launch_bounds__(256, (fusedMinBlocks<SCHEME, R>())) k_stage(const DevCaseT<R>* cases,
                                                                            const Tile* tiles, int stage, int force) {
    __shared__ DevCaseT<R> c;
    extern __shared__ __align__(16) unsigned char fusedSmem[];
    Tile tl;
    if (!enter(cases, tiles, c, stage, force, tl, FL, 0)) return;
    const long long it = c.ctl->it + 1;
    const Gas<R> gs{R(c.gamma), R(c.rgas), FL ? c.lut : nullptr};
    R* const* Uin = stageIn(c, stage);
    const bool three = c.topo == 1;
    FusedBox b;
    fusedLayout(c.fbox[0], c.fbox[1], c.fbox[2], three, b);
    {
        const int box = static_cast<int>(tl.start);
        const int t2 = box / c.fnb[2];
        b.oi = (t2 / c.fnb[1]) * b.bi;
        b.oj = (t2 % c.fnb[1]) * b.bj;
        b.ok = (box % c.fnb[2]) * b.bk;
    }
    const int NW = b.nW;
    const int nF = b.nfI + b.nfJ + b.nfK;
    R* Ws = reinterpret_cast<R*>(fusedSmem);                         // [fields][nW]
    R* Fs = Ws + static_cast<size_t>(fusedNodeFields(SCHEME)) * NW;  // [5][nF]

    // 1. primitives of the box and its cross-shaped halo
    for (int p = threadIdx.x; p < NW; p += blockDim.x) {
        int ii, jj, kk;
        fusedNodeOf(b, p, ii, jj, kk);
        const int gi = b.oi + ii, gj = b.oj + jj, gk = b.ok + kk;
        if (gi < 0 || gi >= c.ni || gj < 0 || gj >= c.nj || gk < 0 || gk >= c.nk) continue;
        const S5<R> W = primOf(load5(Uin, nodeIdx(c, gi, gj, gk)));
#pragma unroll
        for (int v = 0; v < 5; v++) Ws[v * NW + p] = W.v[v];
        if (SCHEME == 0) {
            Ws[5 * NW + p] = pressurePrim(gs, W);
            Ws[6 * NW + p] = jstR(gs, W);
        }
    }
    __syncthreads();

    // 2. every face of the box's nodes: I, J and K faces as one pool
    for (int lf = threadIdx.x; lf < nF; lf += blockDim.x) {
        int d = 0, l = lf;
        if (l >= b.nfI) {
            l -= b.nfI;
            d = 1;
            if (l >= b.nfJ) {
                l -= b.nfJ;
                d = 2;
            }
        }
        const int FJ = b.bj + (d == 1), FK = b.bk + (d == 2);
        const int ak = l % FK;
        const int t2 = l / FK;
        const int aj = t2 % FJ;
        const int ai = t2 / FJ;
        const int fi = b.oi + ai, fj = b.oj + aj, fk = b.ok + ak;
        if (fi > c.ni - (d == 0 ? 0 : 1) || fj > c.nj - (d == 1 ? 0 : 1) || fk > c.nk - (d == 2 ? 0 : 1)) continue;
        if (d == 2 && c.bfm && c.bpresent[nodeIdx(c, fi, fj, 0)] > R(0)) continue;  // blade rows: no K flux
        const int nlast = d == 0 ? c.ni : (d == 1 ? c.nj : c.nk);
        const int dface = d == 0 ? fi : (d == 1 ? fj : fk);
        const long long f = (static_cast<long long>(fi) * (c.nj + (d == 1)) + fj) * (c.nk + (d == 2)) + fk;
        S5<R> fa;
        if (dface >= 2 && dface <= nlast - 2) {
            const DevFacesT<R>& F = c.f[d];
            const V3<R> n = v3(__ldg(F.nx + f), __ldg(F.ny + f), __ldg(F.nz + f));
            const R area = __ldg(F.area + f);
            // the stencil nodes along d: local offsets -2, -1 (left), 0 (right,
            // the face's own i, j, k) and +1
            const int di = d == 0, dj = d == 1, dk = d == 2;
            const int sLL = fusedSlot(b, ai - 2 * di, aj - 2 * dj, ak - 2 * dk);
            const int sL = fusedSlot(b, ai - di, aj - dj, ak - dk);
            const int sR = fusedSlot(b, ai, aj, ak);
            const int sRR = fusedSlot(b, ai + di, aj + dj, ak + dk);
            auto ldW = [&](int p) { return s5(Ws[p], Ws[NW + p], Ws[2 * NW + p], Ws[3 * NW + p], Ws[4 * NW + p]); };
            S5<R> flux;
            if (SCHEME == 0) {
                const long long st = d == 0 ? static_cast<long long>(c.nj) * c.nk : (d == 1 ? c.nk : 1);
                const long long qR = nodeIdx(c, fi, fj, fk);
                const long long qL = qR - st;
                const R* P = Ws + 5 * NW;
                const R* Rr = Ws + 6 * NW;
                flux = fluxJstPR(gs, load5(Uin, qL - st), load5(Uin, qL), load5(Uin, qR), load5(Uin, qR + st),
                                 ldW(sL), ldW(sR), P[sLL], P[sL], P[sR], P[sRR], Rr[sL], Rr[sR], n);
            } else {
                flux = fluxRoeW(gs, c.muscl, c.limiter, c.muscl ? ldW(sLL) : zero5<R>(), ldW(sL), ldW(sR),
                                c.muscl ? ldW(sRR) : zero5<R>(), n);
            }
#pragma unroll
            for (int v = 0; v < 5; v++) fa.v[v] = flux.v[v] * area;
        } else {
            fa = fusedSideFlux<SCHEME>(c, gs, Uin, d, fi, fj, fk, f, it);
        }
#pragma unroll
        for (int v = 0; v < 5; v++) Fs[v * nF + lf] = fa.v[v];
    }
    __syncthreads();

    // 3. residual assembly (I, J, K faces), sources, update and norm partials
    const double t = c.ctl->t;
    const R dtg = R(c.ctl->dt_min);
    const bool resOnly = stage < 0;
    const bool last = !resOnly && stage == c.nstages - 1;
    const R alpha = resOnly ? R(0) : R(c.coeffs[stage]);
    R* const* Uout = stageOut(c, stage);
    const int tk = static_cast<int>(threadIdx.x) % b.bk;
    const int tj = (static_cast<int>(threadIdx.x) / b.bk) % b.bj;
    const int ti = static_cast<int>(threadIdx.x) / (b.bk * b.bj);
    const int i = b.oi + ti, j = b.oj + tj, k = b.ok + tk;
    double acc[5] = {0, 0, 0, 0, 0};
    if (ti < b.bi && i < c.ni && j < c.nj && k < c.nk) {
        S5<R> Res = zero5<R>();
        auto addFaces = [&](int off, int l0, int l1, int g) {
#pragma unroll
            for (int v = 0; v < 5; v++) {
                const R a = Fs[v * nF + off + l0];
                Res.v[v] = (g == 0) ? Res.v[v] + a : Res.v[v] - a;
                Res.v[v] = Res.v[v] + Fs[v * nF + off + l1];
            }
        };
        {
            const int l0 = (ti * b.bj + tj) * b.bk + tk;
            addFaces(0, l0, l0 + b.bj * b.bk, i);
        }
        {
            const int l0 = (ti * (b.bj + 1) + tj) * b.bk + tk;
            addFaces(b.nfI, l0, l0 + b.bk, j);
        }
        if (three && !(c.bfm && c.bpresent[nodeIdx(c, i, j, 0)] > R(0))) {
            const int l0 = (ti * b.bj + tj) * (b.bk + 1) + tk;
            addFaces(b.nfI + b.nfJ, l0, l0 + 1, k);
        }
        const long long q = nodeIdx(c, i, j, k);
        const S5<R> Unode = load5(Uin, q);
        applySources<0>(c, gs, Uin, i, j, k, q, Unode, t, Res);
        if (c.periodic && (k == 0 || k == c.nk - 1)) {
            const long long pq = (k == 0 ? 0 : c.n / c.nk) + static_cast<long long>(i) * c.nj + j;
            store5(c.Rp, pq, Res);
        } else if (resOnly) {
            store5(Uout, q, Res);
        } else {
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
            if (last)
#pragma unroll
                for (int v = 0; v < 5; v++) acc[v] = static_cast<double>(Res.v[v]) * static_cast<double>(Res.v[v]);
        }
    }
    if (last) {
        blockSum<5>(acc);
        if (threadIdx.x == 0) {
            double* part = c.partial + (static_cast<long long>(c.node_tiles) + c.per_tiles) * 5 + c.node_tiles;
#pragma unroll
            for (int v = 0; v < 5; v++) part[tl.local * 5 + v] = acc[v];
        }
    }
}
