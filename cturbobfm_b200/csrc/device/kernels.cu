// Kernels of the FP64 explicit residual-and-update loop (sm_100a).
//
// One pseudo-time iteration is a fixed sequence of launches with no host
// synchronisation, so that chunks of iterations can be captured in a CUDA
// graph:
//   k_bint     boundary-plane integrals: mass flows and turbo Pt/Tt sums
//              (only when turbo performance is needed)
//   k_dt       local time step per node + block minima
//   k_pre      min(dt), turbo performance, Greitzer plenum, radial profiles
//   per Runge-Kutta stage:
//     k_faces<I|J|K>  face fluxes * |S| (interior stencils and boundary faces)
//     k_nodes         residual assembly in the reference's order, sources,
//                     U = U^n - alpha*dt/V*R, residual-norm partial sums
//     k_periodic      periodic-plane residual and solution averaging
//   k_finalize residual norms, divergence and convergence test, time advance
// Every kernel first reads the control block and returns at once when the run
// has converged, diverged, or reached the iteration limit the host set.
//
// Compiled with --fmad=false: no multiply-add contraction, so each expression
// rounds as the reference's does.

#include <cuda_runtime.h>

#include "kernels.hpp"
#include "sources.cuh"

namespace ctbfm {

namespace {

__device__ __forceinline__ bool halted(const DevCase& c) {
    return !c.force && (c.ctl->status != 0 || c.ctl->it >= c.ctl->it_stop);
}

__device__ __forceinline__ S5 boundaryFlux(const DevCase& c, Gas gs, int pidx, const S5& Uint, D3 n, long long qtheta,
                                           int fj, long long it) {
    const DevPatch& p = c.patch[pidx];
    switch (p.type) {
        case kBcInlet: return bcInlet(c, gs, p, Uint, n, c.cost[qtheta], c.sint[qtheta]);
        case kBcOutlet: return bcOutlet(c, gs, Uint, n, p.v[0], it);
        case kBcRadialEq:
        case kBcThrottle: {
            // BoundaryOutletThrottle / RadialEquilibrium index the profile by the
            // face's j (src/boundary_outlet_throttle.cpp:14).
            const int m = p.profile;
            const int jj = fj < c.prof_n[m] ? fj : c.prof_n[m] - 1;
            return bcOutlet(c, gs, Uint, n, c.prof_p[c.prof_off[m] + jj], it);
        }
        case kBcInviscidWall: return bcWall(gs, Uint, n);
        default: return zero5();  // periodic / wedge faces: BoundaryFake, zero flux
    }
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

// ------------------------------------------------------------------ faces
// Solver::computeAdvectionFluxResidualsImpl (src/solver.cpp:1865-2040): one
// thread per face of direction DIR; writes flux * |S|.
template <int DIR, int SCHEME>
__global__ void __launch_bounds__(256) k_faces(DevCase c, P5 Uin) {
    if (halted(c)) return;
    const long long it = c.ctl->it + 1;
    const Gas gs{c.gamma, c.rgas};
    const int nfi = c.ni + (DIR == 0), nfj = c.nj + (DIR == 1), nfk = c.nk + (DIR == 2);
    const long long nf = static_cast<long long>(nfi) * nfj * nfk;
    const long long st = DIR == 0 ? static_cast<long long>(c.nj) * c.nk : (DIR == 1 ? c.nk : 1);
    const int nlast = DIR == 0 ? c.ni : (DIR == 1 ? c.nj : c.nk);
    const DevFaces& F = c.f[DIR];
    double* const* U = Uin.p;
    for (long long f = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; f < nf;
         f += static_cast<long long>(gridDim.x) * blockDim.x) {
        const int fk = static_cast<int>(f % nfk);
        const long long t = f / nfk;
        const int fj = static_cast<int>(t % nfj);
        const int fi = static_cast<int>(t / nfj);
        const int dface = DIR == 0 ? fi : (DIR == 1 ? fj : fk);
        if (DIR == 2 && c.bfm && c.bpresent[nodeIdx(c, fi, fj, 0)] > 0.0) continue;  // blade rows: no K flux
        D3 n = d3(__ldg(F.nx + f), __ldg(F.ny + f), __ldg(F.nz + f));
        const double area = __ldg(F.area + f);
        S5 flux;
        if (dface == 0 || dface == nlast) {
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
            const long long qth = nodeIdx(c, fi < c.ni ? fi : c.ni - 1, fj < c.nj ? fj : c.nj - 1, fk < c.nk ? fk : c.nk - 1);
            flux = boundaryFlux(c, gs, pidx, load5(U, q), n, qth, fj, it);
        } else {
            const long long qR = nodeIdx(c, fi, fj, fk);
            const long long qL = qR - st;
            // faces whose four stencil nodes are plain interior nodes read the
            // primitives k_prim computed once per node (bitwise the same values
            // as converting here); faces next to a boundary or a periodic seam
            // extrapolate or rotate conservative states first
            const bool plain = dface >= 2 && dface <= nlast - 2;
            if (plain) {
                if (SCHEME == 0) {
                    flux = fluxJstW(gs, load5(U, qL - st), load5(U, qL), load5(U, qR), load5(U, qR + st),
                                    load5(c.W, qL - st), load5(c.W, qL), load5(c.W, qR), load5(c.W, qR + st), n);
                } else {
                    flux = fluxRoeW(gs, c.muscl, c.limiter, c.muscl ? load5(c.W, qL - st) : zero5(), load5(c.W, qL),
                                    load5(c.W, qR), c.muscl ? load5(c.W, qR + st) : zero5(), n);
                }
            } else {
                const S5 Ul = load5(U, qL), Ur = load5(U, qR);
                S5 Ull, Urr;
                if (DIR == 2 && c.periodic) {
                    if (dface == 1) {
                        Ull = rotState(load5(U, nodeIdx(c, fi, fj, c.nk - 2)), c.per_cos_m, c.per_sin_m);
                        Urr = load5(U, qR + 1);
                    } else {  // dface == nlast - 1
                        Ull = load5(U, qR - 2);
                        Urr = rotState(load5(U, nodeIdx(c, fi, fj, 1)), c.per_cos_p, c.per_sin_p);
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
        }
#pragma unroll
        for (int v = 0; v < 5; v++) F.c[v][f] = flux.v[v] * area;
    }
}

// Primitives of the stage input (getPrimitiveVariablesFromConservative,
// src/math_utils.cpp:49-57), once per node for the face kernels.
__global__ void __launch_bounds__(256) k_prim(DevCase c, P5 Uin) {
    if (halted(c)) return;
    for (long long q = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; q < c.n;
         q += static_cast<long long>(gridDim.x) * blockDim.x)
        store5(c.W, q, primOf(load5(Uin.p, q)));
}

// ------------------------------------------------------------------ nodes
// Residual assembly in the reference's accumulation order (I faces, J faces,
// K faces, then sources), then Solver::updateSolution (src/solver.cpp:2230-2249).
// mode 0: U_out = U^n - R * (alpha*dt/V); mode 1: write R to Rout.
__global__ void __launch_bounds__(256, 2) k_nodes(DevCase c, P5 Uin, P5 Uout, double alpha, int last, int mode, P5 Rout) {
    if (halted(c)) return;
    const Gas gs{c.gamma, c.rgas};
    const double t = c.ctl->t;
    const double dtg = c.ctl->dt_min;
    double acc[5] = {0, 0, 0, 0, 0};
    const int nj = c.nj, nk = c.nk;
    for (long long q = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; q < c.n;
         q += static_cast<long long>(gridDim.x) * blockDim.x) {
        const int k = static_cast<int>(q % nk);
        const long long tq = q / nk;
        const int j = static_cast<int>(tq % nj);
        const int i = static_cast<int>(tq / nj);
        S5 R = zero5();
        {  // I faces: face i (node is right, or the start boundary) then face i+1
            const long long f0 = (static_cast<long long>(i) * nj + j) * nk + k;
            const long long f1 = f0 + static_cast<long long>(nj) * nk;
#pragma unroll
            for (int v = 0; v < 5; v++) {
                const double a = c.f[0].c[v][f0];
                R.v[v] = (i == 0) ? R.v[v] + a : R.v[v] - a;
                R.v[v] = R.v[v] + c.f[0].c[v][f1];
            }
        }
        {  // J faces
            const long long f0 = (static_cast<long long>(i) * (nj + 1) + j) * nk + k;
            const long long f1 = f0 + nk;
#pragma unroll
            for (int v = 0; v < 5; v++) {
                const double a = c.f[1].c[v][f0];
                R.v[v] = (j == 0) ? R.v[v] + a : R.v[v] - a;
                R.v[v] = R.v[v] + c.f[1].c[v][f1];
            }
        }
        if (c.topo == 1 && !(c.bfm && c.bpresent[nodeIdx(c, i, j, 0)] > 0.0)) {  // K faces
            const long long f0 = (static_cast<long long>(i) * nj + j) * (nk + 1) + k;
            const long long f1 = f0 + 1;
#pragma unroll
            for (int v = 0; v < 5; v++) {
                const double a = c.f[2].c[v][f0];
                R.v[v] = (k == 0) ? R.v[v] + a : R.v[v] - a;
                R.v[v] = R.v[v] + c.f[2].c[v][f1];
            }
        }
        const S5 Unode = load5(Uin.p, q);
        applySources(c, gs, Uin.p, i, j, k, q, Unode, t, R);
        if (c.periodic && (k == 0 || k == nk - 1)) {
            const long long pq = (k == 0 ? 0 : c.n / nk) + static_cast<long long>(i) * nj + j;
            store5(c.Rp, pq, R);
            continue;
        }
        if (mode == 1) {
            store5(Rout.p, q, R);
            continue;
        }
        const double dt = c.dt_method == 1 ? dtg : (c.dt_method == 2 ? c.fixed_dt : c.dt[q]);
        const double fac = alpha * dt / c.vol[q];
        const S5 Un = load5(c.U, q);
        S5 Un1;
#pragma unroll
        for (int v = 0; v < 5; v++) Un1.v[v] = Un.v[v] - R.v[v] * fac;
        store5(Uout.p, q, Un1);
        if (last)
#pragma unroll
            for (int v = 0; v < 5; v++) acc[v] += R.v[v] * R.v[v];
    }
    if (last && mode == 0) {
        blockSum<5>(acc);
        if (threadIdx.x == 0)
#pragma unroll
            for (int v = 0; v < 5; v++) c.partial[blockIdx.x * 5 + v] = acc[v];
    }
}

// Solver::enforcePeriodicityOnResiduals (src/solver.cpp:1836-1853), the update
// of the two periodic planes and Solver::enforcePeriodicityOnSolution
// (src/solver.cpp:2308-2327). One thread per (i, j) pair.
__global__ void __launch_bounds__(256) k_periodic(DevCase c, P5 Uout, double alpha, int last, int mode, P5 Rout) {
    if (halted(c)) return;
    const double dtg = c.ctl->dt_min;
    const long long np = static_cast<long long>(c.ni) * c.nj;
    double acc[5] = {0, 0, 0, 0, 0};
    for (long long p = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; p < np;
         p += static_cast<long long>(gridDim.x) * blockDim.x) {
        const S5 R1 = load5(c.Rp, p), R2 = load5(c.Rp, np + p);
        const S5 Ra = (R1 + rotState(R2, c.per_cos_m, c.per_sin_m)) * 0.5;
        const S5 Rb = rotState(Ra, c.per_cos_p, c.per_sin_p);
        const long long q0 = p * c.nk, q1 = p * c.nk + c.nk - 1;
        if (mode == 1) {
            store5(Rout.p, q0, Ra);
            store5(Rout.p, q1, Rb);
            continue;
        }
        const double dt0 = c.dt_method == 1 ? dtg : (c.dt_method == 2 ? c.fixed_dt : c.dt[q0]);
        const double dt1 = c.dt_method == 1 ? dtg : (c.dt_method == 2 ? c.fixed_dt : c.dt[q1]);
        const double f0 = alpha * dt0 / c.vol[q0];
        const double f1 = alpha * dt1 / c.vol[q1];
        const S5 U0 = load5(c.U, q0) - Ra * f0;
        const S5 U1 = load5(c.U, q1) - Rb * f1;
        const S5 Ua = (U0 + rotState(U1, c.per_cos_m, c.per_sin_m)) * 0.5;
        store5(Uout.p, q0, Ua);
        store5(Uout.p, q1, rotState(Ua, c.per_cos_p, c.per_sin_p));
        if (last)
#pragma unroll
            for (int v = 0; v < 5; v++) acc[v] += Ra.v[v] * Ra.v[v] + Rb.v[v] * Rb.v[v];
    }
    if (last && mode == 0) {
        blockSum<5>(acc);
        if (threadIdx.x == 0)
#pragma unroll
            for (int v = 0; v < 5; v++) c.partial[(c.node_blocks + blockIdx.x) * 5 + v] = acc[v];
    }
}

// ------------------------------------------------------------- time step
// Solver::computeTimestepArray (src/solver.cpp:1531-1630), inviscid:
// dt = CFL / sum_d (|u . e_d| + a) / |e_d| over the dual-node edges.
__global__ void __launch_bounds__(256) k_dt(DevCase c, P5 Uin) {
    if (halted(c)) return;
    const Gas gs{c.gamma, c.rgas};
    double mn = INFINITY;
    for (long long q = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; q < c.n;
         q += static_cast<long long>(gridDim.x) * blockDim.x) {
        const S5 W = primOf(load5(Uin.p, q));
        const D3 u = velOf(W);
        const double a = soundSpeed_rho_u_et(gs, W.v[0], u, W.v[4]);
        const D3 dI = d3(c.edge[0][q], c.edge[1][q], c.edge[2][q]);
        const D3 dJ = d3(c.edge[4][q], c.edge[5][q], c.edge[6][q]);
        const double ui = fabs(dot(u, dI)), uj = fabs(dot(u, dJ));
        double lc = (ui + a) / c.edge[3][q];
        lc += (uj + a) / c.edge[7][q];
        if (c.topo == 1) {
            const D3 dK = d3(c.edge[8][q], c.edge[9][q], c.edge[10][q]);
            lc += (fabs(dot(u, dK)) + a) / c.edge[11][q];
        }
        const double dt = c.cfl / lc;
        c.dt[q] = dt;
        mn = fmin(mn, dt);
    }
    mn = blockMin(mn);
    if (threadIdx.x == 0) c.partial[(c.node_blocks + c.per_blocks) * 5 + blockIdx.x] = mn;
}

// ------------------------------------------------------ boundary integrals
// Solver::updateMassFlows (src/solver.cpp:1633-1649) and the mass-weighted
// total pressure / temperature integrals of Solver::updateTurboPerformance
// (src/solver.cpp:1652-1781). Block b < 6: mass flow through plane b;
// blocks 6, 7: Pt and Tt integrals over the inlet / outlet planes.
__device__ __forceinline__ void planeExtent(const DevCase& c, int b, int& na, int& nb) {
    if (b <= 1) { na = c.nj; nb = c.nk; }
    else if (b <= 3) { na = c.ni; nb = c.nk; }
    else { na = c.ni; nb = c.nj; }
}
__device__ __forceinline__ long long planeNode(const DevCase& c, int b, int a, int bb) {
    switch (b) {
        case 0: return nodeIdx(c, 0, a, bb);
        case 1: return nodeIdx(c, c.ni - 1, a, bb);
        case 2: return nodeIdx(c, a, 0, bb);
        case 3: return nodeIdx(c, a, c.nj - 1, bb);
        case 4: return nodeIdx(c, a, bb, 0);
        default: return nodeIdx(c, a, bb, c.nk - 1);
    }
}
__device__ __forceinline__ int turboPlane(const DevCase& c, int m) {
    switch (c.turbo_dir) {
        case 1: return m == 0 ? 1 : 0;
        case 2: return m == 0 ? 2 : 3;
        case 3: return m == 0 ? 3 : 2;
        default: return m == 0 ? 0 : 1;
    }
}

__global__ void __launch_bounds__(256) k_bint(DevCase c, P5 Uin) {
    if (halted(c)) return;
    const Gas gs{c.gamma, c.rgas};
    const int blk = blockIdx.x;
    const int plane = blk < 6 ? blk : turboPlane(c, blk - 6);
    int na, nb;
    planeExtent(c, plane, na, nb);
    const long long cnt = static_cast<long long>(na) * nb;
    double s[2] = {0.0, 0.0};
    for (long long e = threadIdx.x; e < cnt; e += blockDim.x) {
        const int a = static_cast<int>(e / nb), bb = static_cast<int>(e % nb);
        const long long q = planeNode(c, plane, a, bb);
        const double sx = c.bsx[plane][e], sy = c.bsy[plane][e], sz = c.bsz[plane][e];
        if (blk < 6) {
            s[0] += sx * __ldg(Uin.p[1] + q) + sy * __ldg(Uin.p[2] + q) + sz * __ldg(Uin.p[3] + q);
        } else {
            const S5 W = primOf(load5(Uin.p, q));
            const double rho = W.v[0];
            const D3 u = velOf(W);
            const double P = totalPressure_rho_u_et(gs, rho, u, W.v[4]);
            const double T = totalTemperature_rho_u_et(gs, rho, u, W.v[4]);
            s[0] += sx * (rho * u.x * P) + sy * (rho * u.y * P) + sz * (rho * u.z * P);
            s[1] += sx * (rho * u.x * T) + sy * (rho * u.y * T) + sz * (rho * u.z * T);
        }
    }
    blockSum<2>(s);
    if (threadIdx.x == 0) {
        if (blk < 6) c.ctl->massflow[blk] = s[0];
        else {
            c.ctl->pt_int[blk - 6] = s[0];
            c.ctl->tt_int[blk - 6] = s[1];
        }
    }
}

// ------------------------------------------------------------ pre-stage
// Global min(dt); FluidIdeal::computeTotalEfficiency_PRtt_TRt
// (src/fluid_ideal.cpp:179-191); GreitzerModel::computePlenumPressure
// (src/greitzer_model.cpp:36-56); Solver::updateRadialProfiles
// (src/solver.cpp:2688-2787) with integrateRadialEquilibrium
// (src/math_utils.cpp:141-170).
__global__ void __launch_bounds__(256) k_pre(DevCase c, P5 Uin, int turbo, int profiles, int dtpart) {
    if (halted(c)) return;
    Control* ctl = c.ctl;
    if (!dtpart) {
    } else if (c.dt_method == 2) {
        if (threadIdx.x == 0) ctl->dt_min = c.fixed_dt;
    } else {
        double mn = INFINITY;
        const double* part = c.partial + (c.node_blocks + c.per_blocks) * 5;
        for (int b = threadIdx.x; b < c.dt_blocks; b += blockDim.x) mn = fmin(mn, part[b]);
        mn = blockMin(mn);
        if (threadIdx.x == 0) ctl->dt_min = mn;
    }
    if (threadIdx.x != 0) return;
    const Gas gs{c.gamma, c.rgas};
    if (turbo) {
        const int p0 = turboPlane(c, 0), p1 = turboPlane(c, 1);
        double mflow = 0.5 * (fabs(ctl->massflow[p0]) + fabs(ctl->massflow[p1]));
        if (c.topo == 2) mflow *= 2.0 * M_PI / c.wedge;
        else if (c.per_angle_deg != 0.0) mflow *= 360.0 / c.per_angle_deg;
        double pt[2], tt[2];
        for (int m = 0; m < 2; m++) {
            double mf = ctl->massflow[m == 0 ? p0 : p1];
            if (fabs(mf) < 1e-12) mf = (mf >= 0.0 ? 1e-12 : -1e-12);
            pt[m] = ctl->pt_int[m] / mf;
            tt[m] = ctl->tt_int[m] / mf;
        }
        const double pr = (fabs(pt[0]) > 1e-12) ? pt[1] / pt[0] : 1.0;
        const double tr = (fabs(tt[0]) > 1e-12) ? tt[1] / tt[0] : 1.0;
        const double dT = tr - 1.0;
        const double dTs = pow(pr, (c.gamma - 1.0) / c.gamma) - 1.0;
        double eta;
        if (fabs(dT) < 1e-12) eta = 1.0;
        else if (dT >= 0.0) eta = dTs / dT;
        else eta = (fabs(dTs) < 1e-12) ? 1.0 : dT / dTs;
        ctl->turbo[0] = mflow;
        ctl->turbo[1] = pr;
        ctl->turbo[2] = tr;
        ctl->turbo[3] = eta;
        ctl->has_turbo = 1;
    }
    if (!profiles) return;
    if (c.greitzer) {
        ctl->gz_min = ctl->turbo[0];
        ctl->gz_t += c.fixed_dt;
        const double a = sqrt(c.gamma * c.rgas * ctl->gz_T);
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
        } else if (c.prof_type[m] == kBcRadialEq) {
            ctl->hub_p = p[0];
        }
        // sample density and |u_theta| at (prof_i, j, 0) and integrate dp/dr
        double rho1 = 0, ut1 = 0;
        p[0] = ctl->hub_p;
        for (int jj = 0; jj < n; jj++) {
            const long long q = nodeIdx(c, c.prof_i[m], c.prof_j0[m] + jj, 0);
            const S5 W = primOf(load5(Uin.p, q));
            const D3 vc = cylOfCart(velOf(W), c.cost[q], c.sint[q]);
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

// ------------------------------------------------------------- finalize
// Solver::computeLogResidualNorm (src/solver.cpp:1488-1508),
// printInfoResiduals' initial maximum (src/solver.cpp:1426-1439),
// Solver::checkConvergence (src/solver.cpp:2985-3015) and the time advance
// t += min(dt) (src/solver.cpp:1389).
__global__ void __launch_bounds__(256) k_finalize(DevCase c, int nparts) {
    if (halted(c)) return;
    Control* ctl = c.ctl;
    double s[5] = {0, 0, 0, 0, 0};
    for (int b = threadIdx.x; b < nparts; b += blockDim.x)
#pragma unroll
        for (int v = 0; v < 5; v++) s[v] += c.partial[b * 5 + v];
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
        for (int v = 0; v < 5; v++) ctl->init_log[v] = dmax(ctl->init_log[v], lr[v]);
    }
    const long long row = it - 1 - ctl->hist_base;
    if (c.hist && row >= 0 && row < c.hist_cap) {
        double* h = c.hist + row * 16;
        for (int v = 0; v < 5; v++) h[v] = lr[v];
        for (int b = 0; b < 6; b++) h[5 + b] = ctl->massflow[b];
        for (int b = 0; b < 4; b++) h[11 + b] = c.need_turbo ? ctl->turbo[b] : 0.0;
        h[15] = ctl->hub_p;
    }
    if (c.steady) {
        bool conv = true;
        for (int v = 0; v < 5; ++v) {
            if (v == 3 && c.topo != 1 && c.topo != 2) continue;
            if (ctl->init_log[v] <= -15.99) continue;
            if (lr[v] <= -15.0) continue;
            if (lr[v] >= ctl->init_log[v] - static_cast<double>(c.drop)) {
                conv = false;
                break;
            }
        }
        if (conv) ctl->status = 1;
    }
}

// Sets the iteration limit and the history origin of the next enqueue.
__global__ void k_set_limits(Control* ctl, long long itStop, long long histBase) {
    ctl->it_stop = itStop;
    ctl->hist_base = histBase;
}

}  // namespace

// ------------------------------------------------------------- launchers

static int gridFor(long long n, int block, int cap) {
    long long g = (n + block - 1) / block;
    if (g > cap) g = cap;
    if (g < 1) g = 1;
    return static_cast<int>(g);
}

int nodeBlocks(long long n) { return gridFor(n, 256, 148 * 64); }
int periodicBlocks(long long np) { return gridFor(np, 256, 148 * 8); }

cudaError_t launchBoundaryIntegrals(const DevCase& c, P5 Uin, bool turbo, cudaStream_t s) {
    k_bint<<<turbo ? 8 : 6, 256, 0, s>>>(c, Uin);
    return cudaGetLastError();
}

cudaError_t launchTimeStep(const DevCase& c, P5 Uin, cudaStream_t s) {
    if (c.dt_method == 2) return cudaSuccess;
    k_dt<<<c.dt_blocks, 256, 0, s>>>(c, Uin);
    return cudaGetLastError();
}

cudaError_t launchPre(const DevCase& c, P5 Uin, bool turbo, bool profiles, bool dtpart, cudaStream_t s) {
    k_pre<<<1, 256, 0, s>>>(c, Uin, turbo ? 1 : 0, profiles ? 1 : 0, dtpart ? 1 : 0);
    return cudaGetLastError();
}

cudaError_t launchSetLimits(const DevCase& c, long long itStop, long long histBase, cudaStream_t s) {
    k_set_limits<<<1, 1, 0, s>>>(c.ctl, itStop, histBase);
    return cudaGetLastError();
}

cudaError_t launchFaces(const DevCase& c, int d, P5 Uin, cudaStream_t s) {
    const long long nf = static_cast<long long>(c.ni + (d == 0)) * (c.nj + (d == 1)) * (c.nk + (d == 2));
    const int g = gridFor(nf, 256, 148 * 64);
    if (c.scheme == 0) {
        if (d == 0) k_faces<0, 0><<<g, 256, 0, s>>>(c, Uin);
        else if (d == 1) k_faces<1, 0><<<g, 256, 0, s>>>(c, Uin);
        else k_faces<2, 0><<<g, 256, 0, s>>>(c, Uin);
    } else {
        if (d == 0) k_faces<0, 1><<<g, 256, 0, s>>>(c, Uin);
        else if (d == 1) k_faces<1, 1><<<g, 256, 0, s>>>(c, Uin);
        else k_faces<2, 1><<<g, 256, 0, s>>>(c, Uin);
    }
    return cudaGetLastError();
}

cudaError_t launchNodes(const DevCase& c, P5 Uin, P5 Uout, double alpha, bool last, int mode, P5 Rout, cudaStream_t s) {
    k_nodes<<<c.node_blocks, 256, 0, s>>>(c, Uin, Uout, alpha, last ? 1 : 0, mode, Rout);
    return cudaGetLastError();
}

cudaError_t launchPeriodic(const DevCase& c, P5 Uout, double alpha, bool last, int mode, P5 Rout, cudaStream_t s) {
    k_periodic<<<c.per_blocks, 256, 0, s>>>(c, Uout, alpha, last ? 1 : 0, mode, Rout);
    return cudaGetLastError();
}

cudaError_t launchPrim(const DevCase& c, P5 Uin, cudaStream_t s) {
    k_prim<<<c.node_blocks, 256, 0, s>>>(c, Uin);
    return cudaGetLastError();
}

cudaError_t launchStage(const DevCase& c, P5 Uin, P5 Uout, double alpha, bool last, int mode, P5 Rout, cudaStream_t s) {
    const int dirs = c.topo == 1 ? 3 : 2;
    k_prim<<<c.node_blocks, 256, 0, s>>>(c, Uin);
    for (int d = 0; d < dirs; d++) {
        const cudaError_t e = launchFaces(c, d, Uin, s);
        if (e != cudaSuccess) return e;
    }
    k_nodes<<<c.node_blocks, 256, 0, s>>>(c, Uin, Uout, alpha, last ? 1 : 0, mode, Rout);
    if (c.periodic) k_periodic<<<c.per_blocks, 256, 0, s>>>(c, Uout, alpha, last ? 1 : 0, mode, Rout);
    return cudaGetLastError();
}

cudaError_t launchFinalize(const DevCase& c, cudaStream_t s) {
    k_finalize<<<1, 256, 0, s>>>(c, c.node_blocks + (c.periodic ? c.per_blocks : 0));
    return cudaGetLastError();
}

}  // namespace ctbfm
