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
//      (plus, for JST, each node's pressure and spectral radius |u| + a);
//   2. direction by direction (I, J, then K in 3-D) evaluates every face of
//      the box's nodes (faces on the box's edges are evaluated by both
//      neighbouring boxes) into shared memory, and each thread adds the
//      start and end face of its node to the node's residual, in the order
//      of Solver::computeResiduals (src/solver.cpp:1783-1833);
//   3. applies the sources, the update U(k) = U^n - alpha dt/V R (Kahan-
//      compensated in float) and the residual-norm partials, as k_nodes does.
// Faces whose four stencil nodes are interior read the shared-memory
// primitives; boundary faces and faces next to a boundary or a periodic seam
// go through fusedSideFlux, which reads the conservative states from global
// memory exactly as k_faces does. Every face flux and every residual is the
// same value, bit for bit, as in the split stage (k_prim, k_faces, k_nodes):
// only where the intermediate values live changes (shared memory instead of
// HBM).
#pragma once

// Box geometry of one block.
struct FusedBox {
    int bi, bj, bk;     // box extent
    int oi, oj, ok;     // origin (global node indices)
    int hk;             // halo along k (2 in 3-D, 0 otherwise)
    int pj, pk;         // padded extents along j and k
    int np;             // padded node count
};

// Shared-memory fields per padded node: primitives (5), and for JST the
// node's pressure and spectral radius.
template <int SCHEME>
CTBFM_HD constexpr int fusedNodeFields() {
    return SCHEME == 0 ? 7 : 5;
}

// Boundary faces and faces next to a boundary or a periodic seam, exactly as
// k_faces computes them (conservative states from global memory); returns
// flux * |S|. Not inlined: these faces are few, and their code stays out of
// the fused kernel's registers.
template <int DIR, int SCHEME, typename R>
__device__ __noinline__ S5<R> fusedSideFlux(const DevCaseT<R>& c, Gas<R> gs, R* const* U, int fi, int fj, int fk,
                                            long long f, long long it) {
    const long long st = DIR == 0 ? static_cast<long long>(c.nj) * c.nk : (DIR == 1 ? c.nk : 1);
    const int nlast = DIR == 0 ? c.ni : (DIR == 1 ? c.nj : c.nk);
    const int dface = DIR == 0 ? fi : (DIR == 1 ? fj : fk);
    const DevFacesT<R>& F = c.f[DIR];
    V3<R> n = v3(__ldg(F.nx + f), __ldg(F.ny + f), __ldg(F.nz + f));
    const R area = __ldg(F.area + f);
    S5<R> flux;
    if (dface == 0 || dface == nlast) {
        const int side = dface == 0 ? 0 : 1;
        const int ni_ = DIR == 0 ? (side ? c.ni - 1 : 0) : fi;
        const int nj_ = DIR == 1 ? (side ? c.nj - 1 : 0) : fj;
        const int nk_ = DIR == 2 ? (side ? c.nk - 1 : 0) : fk;
        const long long q = nodeIdx(c, ni_, nj_, nk_);
        if (side == 0) n = -n;
        int pidx;
        if (DIR == 0) pidx = c.mapI[(static_cast<long long>(side) * c.nj + fj) * c.nk + fk];
        else if (DIR == 1) pidx = c.mapJ[(static_cast<long long>(fi) * 2 + side) * c.nk + fk];
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
        if (DIR == 2 && c.periodic) {
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

// The faces of direction DIR of the box's nodes into shared memory, then each
// node's start and end face into its residual (k_nodes' order and signs).
template <int DIR, int SCHEME, typename R>
__device__ __forceinline__ void fusedSweep(const DevCaseT<R>& c, Gas<R> gs, R* const* U, const R* Ws, R* Fs,
                                           const FusedBox& b, long long it, bool valid, int ti, int tj, int tk,
                                           int gi, int gj, int gk, S5<R>& Res) {
    const int FI = b.bi + (DIR == 0), FJ = b.bj + (DIR == 1), FK = b.bk + (DIR == 2);
    const int nf = FI * FJ * FK;
    const int nlast = DIR == 0 ? c.ni : (DIR == 1 ? c.nj : c.nk);
    const int nfj = c.nj + (DIR == 1), nfk = c.nk + (DIR == 2);
    const long long st = DIR == 0 ? static_cast<long long>(c.nj) * c.nk : (DIR == 1 ? c.nk : 1);
    const int sd = DIR == 0 ? b.pj * b.pk : (DIR == 1 ? b.pk : 1);  // padded stride along DIR
    const DevFacesT<R>& F = c.f[DIR];
    const int NP = b.np;
    for (int lf = threadIdx.x; lf < nf; lf += blockDim.x) {
        const int ak = lf % FK;
        const int t2 = lf / FK;
        const int aj = t2 % FJ;
        const int ai = t2 / FJ;
        const int fi = b.oi + ai, fj = b.oj + aj, fk = b.ok + ak;
        if (fi > c.ni - (DIR == 0 ? 0 : 1) || fj > c.nj - (DIR == 1 ? 0 : 1) || fk > c.nk - (DIR == 2 ? 0 : 1))
            continue;
        if (DIR == 2 && c.bfm && c.bpresent[nodeIdx(c, fi, fj, 0)] > R(0)) continue;  // blade rows: no K flux
        const int dface = DIR == 0 ? fi : (DIR == 1 ? fj : fk);
        const long long f = (static_cast<long long>(fi) * nfj + fj) * nfk + fk;
        S5<R> fa;
        if (dface >= 2 && dface <= nlast - 2) {
            const V3<R> n = v3(__ldg(F.nx + f), __ldg(F.ny + f), __ldg(F.nz + f));
            const R area = __ldg(F.area + f);
            const int pR = ((ai + 2) * b.pj + (aj + 2)) * b.pk + (ak + b.hk);  // right node (the face's own i, j, k)
            const int pL = pR - sd;
            auto ldW = [&](int p) {
                return s5(Ws[p], Ws[NP + p], Ws[2 * NP + p], Ws[3 * NP + p], Ws[4 * NP + p]);
            };
            S5<R> flux;
            if (SCHEME == 0) {
                const long long qR = nodeIdx(c, fi, fj, fk);
                const long long qL = qR - st;
                const R* P = Ws + 5 * NP;
                const R* Rr = Ws + 6 * NP;
                flux = fluxJstPR(gs, load5(U, qL - st), load5(U, qL), load5(U, qR), load5(U, qR + st), ldW(pL),
                                 ldW(pR), P[pL - sd], P[pL], P[pR], P[pR + sd], Rr[pL], Rr[pR], n);
            } else {
                flux = fluxRoeW(gs, c.muscl, c.limiter, c.muscl ? ldW(pL - sd) : zero5<R>(), ldW(pL), ldW(pR),
                                c.muscl ? ldW(pR + sd) : zero5<R>(), n);
            }
#pragma unroll
            for (int v = 0; v < 5; v++) fa.v[v] = flux.v[v] * area;
        } else {
            fa = fusedSideFlux<DIR, SCHEME>(c, gs, U, fi, fj, fk, f, it);
        }
#pragma unroll
        for (int v = 0; v < 5; v++) Fs[v * kFusedFaceCap + lf] = fa.v[v];
    }
    __syncthreads();
    if (valid && (DIR != 2 || !(c.bfm && c.bpresent[nodeIdx(c, gi, gj, 0)] > R(0)))) {
        const int l0 = (ti * FJ + tj) * FK + tk;
        const int l1 = l0 + (DIR == 0 ? FJ * FK : (DIR == 1 ? FK : 1));
        const int g = DIR == 0 ? gi : (DIR == 1 ? gj : gk);
#pragma unroll
        for (int v = 0; v < 5; v++) {
            const R a = Fs[v * kFusedFaceCap + l0];
            Res.v[v] = (g == 0) ? Res.v[v] + a : Res.v[v] - a;
            Res.v[v] = Res.v[v] + Fs[v * kFusedFaceCap + l1];
        }
    }
    __syncthreads();
}

// Resident blocks of 256 threads per SM asked of k_stage (its register
// budget), as for the face kernels: double JST 2, otherwise 3.
template <int SCHEME, typename R>
constexpr int fusedMinBlocks() {
    return (sizeof(R) == 8 && SCHEME == 0) ? 2 : 3;
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
    const double t = c.ctl->t;
    const R dtg = R(c.ctl->dt_min);
    const bool resOnly = stage < 0;
    const bool last = !resOnly && stage == c.nstages - 1;
    const R alpha = resOnly ? R(0) : R(c.coeffs[stage]);
    R* const* Uin = stageIn(c, stage);
    R* const* Uout = stageOut(c, stage);
    const bool three = c.topo == 1;
    FusedBox b;
    b.bi = c.fbox[0];
    b.bj = c.fbox[1];
    b.bk = c.fbox[2];
    {
        const int box = static_cast<int>(tl.start);
        const int bk = box % c.fnb[2];
        const int t2 = box / c.fnb[2];
        b.oi = (t2 / c.fnb[1]) * b.bi;
        b.oj = (t2 % c.fnb[1]) * b.bj;
        b.ok = bk * b.bk;
    }
    b.hk = three ? 2 : 0;
    b.pj = b.bj + 4;
    b.pk = b.bk + 2 * b.hk;
    b.np = (b.bi + 4) * b.pj * b.pk;
    R* Ws = reinterpret_cast<R*>(fusedSmem);                   // [fields][np]
    R* Fs = Ws + static_cast<size_t>(fusedNodeFields<SCHEME>()) * b.np;  // [5][kFusedFaceCap]

    // 1. primitives of the box and its cross-shaped halo
    for (int p = threadIdx.x; p < b.np; p += blockDim.x) {
        const int kk = p % b.pk - b.hk;
        const int t2 = p / b.pk;
        const int jj = t2 % b.pj - 2;
        const int ii = t2 / b.pj - 2;
        const int outside = (ii < 0 || ii >= b.bi) + (jj < 0 || jj >= b.bj) + (kk < 0 || kk >= b.bk);
        if (outside > 1) continue;
        const int gi = b.oi + ii, gj = b.oj + jj, gk = b.ok + kk;
        if (gi < 0 || gi >= c.ni || gj < 0 || gj >= c.nj || gk < 0 || gk >= c.nk) continue;
        const S5<R> W = primOf(load5(Uin, nodeIdx(c, gi, gj, gk)));
#pragma unroll
        for (int v = 0; v < 5; v++) Ws[v * b.np + p] = W.v[v];
        if (SCHEME == 0) {
            Ws[5 * b.np + p] = pressurePrim(gs, W);
            Ws[6 * b.np + p] = jstR(gs, W);
        }
    }
    __syncthreads();

    // 2. faces and residual assembly, direction by direction
    const int tk = static_cast<int>(threadIdx.x) % b.bk;
    const int tj = (static_cast<int>(threadIdx.x) / b.bk) % b.bj;
    const int ti = static_cast<int>(threadIdx.x) / (b.bk * b.bj);
    const int i = b.oi + ti, j = b.oj + tj, k = b.ok + tk;
    const bool valid = ti < b.bi && i < c.ni && j < c.nj && k < c.nk;
    S5<R> Res = zero5<R>();
    fusedSweep<0, SCHEME>(c, gs, Uin, Ws, Fs, b, it, valid, ti, tj, tk, i, j, k, Res);
    fusedSweep<1, SCHEME>(c, gs, Uin, Ws, Fs, b, it, valid, ti, tj, tk, i, j, k, Res);
    if (three) fusedSweep<2, SCHEME>(c, gs, Uin, Ws, Fs, b, it, valid, ti, tj, tk, i, j, k, Res);

    // 3. sources, update and norm partials (k_nodes)
    double acc[5] = {0, 0, 0, 0, 0};
    if (valid) {
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
