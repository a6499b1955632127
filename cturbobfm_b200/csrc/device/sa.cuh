// Spalart-Allmaras model (TURBULENCE_MODEL = SA, src/turbulence_model_sa.cpp)
// on the device: TurbulenceModelSA::solve, once per iteration before the
// Runge-Kutta stages (Solver::updateTurbulenceSolution, src/solver.cpp:
// 3061-3071), with the iteration's time step and the solution gradient of the
// iteration's start state. Included by kernels_impl.cuh inside its anonymous
// namespace (it uses enter() and the instance description).
//
// Sequence per iteration (one SA instance per tile of the SA tile lists):
//   k_sa_bc      boundary values (updateBoundaryValues), patch by patch;
//   k_sa_prep    Green-Gauss gradient of nu hat, laminar kinematic viscosity
//                (updateMeanFlowTerms) and node velocities, per node;
//   k_sa_res     flux terms, sources and the diagonal of the implicit update,
//                per node (every interior face is evaluated by both its nodes,
//                the same value twice);
//   k_sa_sweep   the forward and the backward Gauss-Seidel sweep: a node
//                depends on its lower (upper) neighbour in i, j and k, so the
//                sweep runs plane by plane over i + j + k (each plane's nodes
//                are independent), which keeps every node's arithmetic that
//                of the reference's lexicographic sweep;
//   k_sa_update  under-relaxed, clamped update of nu hat (NaN/Inf stops the
//                instance as diverged);
//   k_sa_bc      boundary values again.
#pragma once

// TurbulenceModelSA constants (include/turbulence_model_sa.hpp:80-93).
struct SaConst {
    static constexpr double cb1 = 0.1355, cb2 = 0.622, kappa = 0.41, cw2 = 0.3, cw3 = 2.0, cv1 = 7.1, ct3 = 0.0,
                            ct4 = 0.5, cn1 = 16.0, c2 = 0.7, c3 = 0.9;
};
__device__ __forceinline__ double saSigma() { return 2.0 / 3.0; }
__device__ __forceinline__ double saCw1() {
    return SaConst::cb1 / (SaConst::kappa * SaConst::kappa) + (1.0 + SaConst::cb2) / saSigma();
}

// TurbulenceModelSA::updateBoundaryValues (src/turbulence_model_sa.cpp:250-345):
// one block per instance; the patches in the boundary file's order (a node on
// two patches takes the later one's value), the nodes of one patch in
// parallel (a donor is never a node of its own patch).
template <typename R>
__global__ void __launch_bounds__(256) k_sa_bc(const DevCaseT<R>* cases, const Tile* tiles, int force) {
    __shared__ DevCaseT<R> c;
    Tile tl;
    if (!enter(cases, tiles, c, 0, force, tl)) return;
    for (int m = 0; m < c.sa_npatch; m++) {
        const int* row = c.sa_bc + 10 * m;
        const int kind = row[0];
        const int ni = row[2] - row[1], nj = row[4] - row[3], nk = row[6] - row[5];
        const long long cnt = static_cast<long long>(ni) * nj * nk;
        const R ff = R(c.sa_init_nu * c.sa_ff);
        for (long long e = threadIdx.x; e < cnt; e += blockDim.x) {
            const int k = row[5] + static_cast<int>(e % nk);
            const long long t = e / nk;
            const int j = row[3] + static_cast<int>(t % nj);
            const int i = row[1] + static_cast<int>(t / nj);
            const long long q = nodeIdx(c, i, j, k);
            if (kind == 0) c.nuhat[q] = R(0);
            else if (kind == 1) c.nuhat[q] = ff;
            else c.nuhat[q] = c.nuhat[nodeIdx(c, i + row[7], j + row[8], k + row[9])];
        }
        __syncthreads();
    }
}

// computeGradientGreenGauss (src/math_utils.cpp:173-234) of nu hat with
// interpolateScalar (:395-466) and computeGreenGaussDivergence
// (include/math_utils.hpp:95-106); updateMeanFlowTerms
// (src/turbulence_model_sa.cpp:370-390): mu(T) / rho; and the node velocity
// rho u * (1 / rho) of updateSolution (:663-672). Per node of U^n.
template <typename R, int FL>
__global__ void __launch_bounds__(256) k_sa_prep(const DevCaseT<R>* cases, const Tile* tiles, int force) {
    __shared__ DevCaseT<R> c;
    Tile tl;
    if (!enter(cases, tiles, c, 0, force, tl, FL)) return;
    const Gas<R> gs{R(c.gamma), R(c.rgas), FL ? c.lut : nullptr};
    const int ni = c.ni, nj = c.nj, nk = c.nk;
    const long long sI = static_cast<long long>(nj) * nk;
    for (long long q = tl.start + threadIdx.x; q < tl.start + tl.count; q += blockDim.x) {
        const int k = static_cast<int>(q % nk);
        const long long tq = q / nk;
        const int j = static_cast<int>(tq % nj);
        const int i = static_cast<int>(tq / nj);
        const R f0 = c.nuhat[q];
        R g[3] = {R(0), R(0), R(0)};
        // face of direction d at index fidx; the node is its left (lower) node
        // or its right node; nb the neighbour across it, -1 on a boundary face
        auto face = [&](int d, long long fidx, long long nb, bool neg, bool left) {
            R sc = f0;
            if (nb >= 0) {
                const R d0 = left ? __ldg(c.sa_dL[d] + fidx) : __ldg(c.sa_dR[d] + fidx);
                const R d1 = left ? __ldg(c.sa_dR[d] + fidx) : __ldg(c.sa_dL[d] + fidx);
                sc = f0 + (c.nuhat[nb] - f0) * d0 / (d0 + d1);
            }
            R S[3] = {__ldg(c.sraw[d][0] + fidx), __ldg(c.sraw[d][1] + fidx), __ldg(c.sraw[d][2] + fidx)};
            if (neg) S[0] = -S[0], S[1] = -S[1], S[2] = -S[2];
#pragma unroll
            for (int x = 0; x < 3; x++) g[x] = addRn(g[x], mulRn(S[x], sc));
        };
        const long long fI = (static_cast<long long>(i) * nj + j) * nk + k;
        const long long fJ = (static_cast<long long>(i) * (nj + 1) + j) * nk + k;
        const long long fK = (static_cast<long long>(i) * nj + j) * (nk + 1) + k;
        face(0, fI, i > 0 ? q - sI : -1, true, false);            // west
        face(0, fI + sI, i < ni - 1 ? q + sI : -1, false, true);  // east
        face(1, fJ + nk, j < nj - 1 ? q + nk : -1, false, true);  // north
        face(1, fJ, j > 0 ? q - nk : -1, true, false);            // south
        face(2, fK, k > 0 ? q - 1 : -1, true, false);             // bottom
        face(2, fK + 1, k < nk - 1 ? q + 1 : -1, false, true);    // top
        const R vol = c.vol[q];
#pragma unroll
        for (int x = 0; x < 3; x++) c.sa_g[x][q] = g[x] / vol;
        const R rho = c.U[0][q];
        const V3<R> u = v3(c.U[1][q] / rho, c.U[2][q] / rho, c.U[3][q] / rho);
        const R T = temperature_rho_u_et(gs, rho, u, c.U[4][q] / rho);
        c.nul[q] = molecularViscosity(c, T) / rho;
        const R inv = R(1) / rho;
        c.sa_vel[0][q] = c.U[1][q] * inv;
        c.sa_vel[1][q] = c.U[2][q] * inv;
        c.sa_vel[2][q] = c.U[3][q] * inv;
    }
}

// nu + nu_hat fn of a node (computeViscousFlux, src/turbulence_model_sa.cpp:513-545).
template <typename R>
__device__ __forceinline__ R saNuTotal(const DevCaseT<R>& c, long long q) {
    const R nuL = c.nul[q], nuHat = c.nuhat[q];
    if (nuHat >= R(0)) return nuL + nuHat;
    const R chi = (nuL > R(0)) ? (nuHat / nuL) : R(0);
    const R chi3 = chi * chi * chi;
    const R fn = (R(SaConst::cn1) + chi3) / (R(SaConst::cn1) - chi3);
    return nuL + nuHat * fn;
}

// (adv - visc) |S| of the interior face f of direction d between nodes qL and
// qR (computeAdvectionFlux / computeViscousFlux, src/turbulence_model_sa.cpp:
// 480-558): first-order upwind nu hat by the mean face-normal velocity, and
// the averaged diffusion (nu + nu_hat fn) grad nu_hat / sigma.
template <typename R>
__device__ __forceinline__ R saFaceFlux(const DevCaseT<R>& c, int d, long long f, long long qL, long long qR) {
    const DevFacesT<R>& F = c.f[d];
    const V3<R> n = v3(__ldg(F.nx + f), __ldg(F.ny + f), __ldg(F.nz + f));
    const R area = __ldg(F.area + f);
    const S5<R> WL = primOf(load5(c.U, qL)), WR = primOf(load5(c.U, qR));
    const R un = R(0.5) * dot(velOf(WL) + velOf(WR), n);
    const R phi = (un >= R(0)) ? c.nuhat[qL] : c.nuhat[qR];
    const R adv = phi * un;
    const R sig = R(saSigma());
    const R tL = saNuTotal(c, qL), tR = saNuTotal(c, qR);
    const V3<R> tauL = v3(c.sa_g[0][qL] / sig, c.sa_g[1][qL] / sig, c.sa_g[2][qL] / sig) * tL;
    const V3<R> tauR = v3(c.sa_g[0][qR] / sig, c.sa_g[1][qR] / sig, c.sa_g[2][qR] / sig) * tR;
    const R visc = R(0.5) * dot(tauL + tauR, n);
    return (adv - visc) * area;
}

// TurbulenceModelSA::computeSource (src/turbulence_model_sa.cpp:578-647) with
// computeRotationRateMagnitude (src/math_utils.cpp:620-639) from the velocity
// gradients of the solution gradient (G).
template <typename R>
__device__ R saSource(const DevCaseT<R>& c, long long q) {
    const R d = c.sa_wd[q];
    if (d <= R(0)) return R(0);
    const R nuHat = c.nuhat[q];
    R nuL = c.nul[q];
    if (nuL <= R(0)) nuL = R(1e-14);
    const R o12 = R(0.5) * (c.G[1][q] - c.G[3][q]);
    const R o13 = R(0.5) * (c.G[2][q] - c.G[6][q]);
    const R o23 = R(0.5) * (c.G[5][q] - c.G[7][q]);
    const R Sv = R(2) * sqrt(o12 * o12 + o13 * o13 + o23 * o23);
    const R gx = c.sa_g[0][q], gy = c.sa_g[1][q], gz = c.sa_g[2][q];
    const R gsq = gx * gx + gy * gy + gz * gz;
    const R sig = R(saSigma());
    const R cross = (R(SaConst::cb2) / sig) * gsq;
    const R cw1 = R(saCw1());
    const R kap = R(SaConst::kappa);
    if (nuHat >= R(0)) {
        const R chi = nuHat / nuL;
        const R chi3 = chi * chi * chi;
        const R cv1_3 = R(SaConst::cv1) * R(SaConst::cv1) * R(SaConst::cv1);
        const R fv1 = chi3 / (chi3 + cv1_3);
        const R fv2 = R(1) - chi / (R(1) + chi * fv1);
        const R dSq = d * d;
        const R kd = kap * kap * dSq;
        const R Sbar = (nuHat / kd) * fv2;
        const R c2 = R(SaConst::c2), c3 = R(SaConst::c3);
        R Shat;
        if (Sbar >= -c2 * Sv) Shat = Sv + Sbar;
        else Shat = Sv + (Sv * (c2 * c2 * Sv + c3 * Sbar)) / ((c3 - R(2) * c2) * Sv - Sbar);
        R r;
        if (Shat * kd <= R(0)) r = R(10);
        else r = rmin(nuHat / (Shat * kd), R(10));
        const R r2 = r * r;
        const R r6 = r2 * r2 * r2;
        const R g = r + R(SaConst::cw2) * (r6 - r);
        const R g6 = pow(g, R(6));
        const R cw3_6 = pow(R(SaConst::cw3), R(6));
        const R fw = g * pow((R(1) + cw3_6) / (g6 + cw3_6), R(1) / R(6));
        const R ft2 = R(SaConst::ct3) * exp(-R(SaConst::ct4) * chi * chi);
        const R P = R(SaConst::cb1) * (R(1) - ft2) * Shat * nuHat;
        const R D = (cw1 * fw - (R(SaConst::cb1) / (kap * kap)) * ft2) * (nuHat * nuHat / dSq);
        return P - D + cross;
    }
    const R dSq = d * d;
    const R Pn = R(SaConst::cb1) * (R(1) - R(SaConst::ct3)) * Sv * nuHat;
    const R Dn = cw1 * (nuHat * nuHat / dSq);
    return Pn + Dn + cross;
}

// Flux terms (computeFluxTerms, src/turbulence_model_sa.cpp:392-478) in the
// reference's accumulation order per node (I, J, K; the face the node is the
// right node of first), sources (computeSourceTerms, :560-576: minus Q V), and
// the diagonal of the implicit update (updateSolution, :674-717: V / dt,
// convective and diffusive spectral radii, destruction Jacobian).
template <typename R>
__global__ void __launch_bounds__(256) k_sa_res(const DevCaseT<R>* cases, const Tile* tiles, int force) {
    __shared__ DevCaseT<R> c;
    Tile tl;
    if (!enter(cases, tiles, c, 0, force, tl)) return;
    const int ni = c.ni, nj = c.nj, nk = c.nk;
    const long long sI = static_cast<long long>(nj) * nk;
    const bool three = c.topo == 1;
    const R dtg = R(c.ctl->dt_min);
    for (long long q = tl.start + threadIdx.x; q < tl.start + tl.count; q += blockDim.x) {
        const int k = static_cast<int>(q % nk);
        const long long tq = q / nk;
        const int j = static_cast<int>(tq % nj);
        const int i = static_cast<int>(tq / nj);
        const long long fI = (static_cast<long long>(i) * nj + j) * nk + k;
        const long long fJ = (static_cast<long long>(i) * (nj + 1) + j) * nk + k;
        const long long fK = (static_cast<long long>(i) * nj + j) * (nk + 1) + k;
        R res = R(0);
        if (i >= 1) res = res - saFaceFlux(c, 0, fI, q - sI, q);
        if (i + 1 <= ni - 1) res = res + saFaceFlux(c, 0, fI + sI, q, q + sI);
        if (j >= 1) res = res - saFaceFlux(c, 1, fJ, q - nk, q);
        if (j + 1 <= nj - 1) res = res + saFaceFlux(c, 1, fJ + nk, q, q + nk);
        if (three) {
            if (k >= 1) res = res - saFaceFlux(c, 2, fK, q - 1, q);
            if (k + 1 <= nk - 1) res = res + saFaceFlux(c, 2, fK + 1, q, q + 1);
        }
        const R vol = c.vol[q];
        res = res - saSource(c, q) * vol;
        c.sa_res[q] = res;
        // diagonal
        const V3<R> v = v3(c.sa_vel[0][q], c.sa_vel[1][q], c.sa_vel[2][q]);
        auto sv = [&](int d, long long f) {
            return v3(__ldg(c.sraw[d][0] + f), __ldg(c.sraw[d][1] + f), __ldg(c.sraw[d][2] + f));
        };
        const V3<R> sW = sv(0, fI), sE = sv(0, fI + sI), sS = sv(1, fJ), sN = sv(1, fJ + nk);
        const R lamW = fabs(dot(v, sW)), lamE = fabs(dot(v, sE));
        const R lamS = fabs(dot(v, sS)), lamN = fabs(dot(v, sN));
        R lamB = R(0), lamT = R(0);
        V3<R> sB = v3(R(0), R(0), R(0)), sT = sB;
        if (three) {
            sB = sv(2, fK);
            sT = sv(2, fK + 1);
            lamB = fabs(dot(v, sB));
            lamT = fabs(dot(v, sT));
        }
        const R sigC = R(0.5) * (lamW + lamE + lamS + lamN + lamB + lamT);
        const R nuHat = c.nuhat[q];
        const R nuDiff = (c.nul[q] + rmax(R(0), nuHat)) / R(saSigma());
        R sq = dot(sW, sW) + dot(sE, sE);
        sq += dot(sS, sS) + dot(sN, sN);
        if (three) sq += dot(sB, sB) + dot(sT, sT);
        const R sigV = (nuDiff / vol) * sq;
        const R dw = c.sa_wd[q];
        const R dSq = rmax(dw * dw, R(1e-16));
        const R sigD = vol * (R(2) * R(saCw1()) * fabs(nuHat) / dSq);
        const R dt = c.dt_method == 1 ? dtg : (c.dt_method == 2 ? R(c.fixed_dt) : c.dt[q]);
        c.sa_diag[q] = (vol / dt) + sigC + sigV + sigD;
    }
}

// The forward (FWD = 1) or backward Gauss-Seidel sweep of updateSolution
// (src/turbulence_model_sa.cpp:719-806): node (i, j, k) needs the increments
// of its lower (upper) neighbours in i, j and k, all on the plane i + j + k
// one below (above) its own, so one block per instance walks the planes in
// order and updates each plane's nodes in parallel; every node's sum keeps the
// reference's I, J, K order. Faces: the I face (i, j, k) joins nodes i - 1 and
// i; the upwind weights are 0.5 (Vn + |Vn|) forward and 0.5 (|Vn| - Vn)
// backward with Vn the neighbour's velocity on the face's raw S.
template <typename R, int FWD>
__global__ void __launch_bounds__(1024) k_sa_sweep(const DevCaseT<R>* cases, const Tile* tiles, int force) {
    __shared__ DevCaseT<R> c;
    Tile tl;
    if (!enter(cases, tiles, c, 0, force, tl)) return;
    const int ni = c.ni, nj = c.nj, nk = c.nk;
    const bool three = c.topo == 1;
    const long long sI = static_cast<long long>(nj) * nk;
    const long long pairs = static_cast<long long>(ni) * nj;
    const int planes = ni + nj + nk - 2;
    auto vdotS = [&](long long qn, int d, long long f) {
        return c.sa_vel[0][qn] * c.sraw[d][0][f] + c.sa_vel[1][qn] * c.sraw[d][1][f] +
               c.sa_vel[2][qn] * c.sraw[d][2][f];
    };
    for (int p = 0; p <= planes; p++) {
        const int h = FWD ? p : planes - p;
        for (long long e = threadIdx.x; e < pairs; e += blockDim.x) {
            const int i = static_cast<int>(e / nj), j = static_cast<int>(e % nj);
            const int k = h - i - j;
            if (k < 0 || k >= nk) continue;
            const long long q = (static_cast<long long>(i) * nj + j) * nk + k;
            const long long fI = q;                                                  // I face (i, j, k)
            const long long fJ = (static_cast<long long>(i) * (nj + 1) + j) * nk + k;  // J face (i, j, k)
            const long long fK = (static_cast<long long>(i) * nj + j) * (nk + 1) + k;  // K face (i, j, k)
            if (FWD) {
                R rhs = -c.sa_res[q];
                if (i > 0) {
                    const R Vn = vdotS(q - sI, 0, fI);
                    rhs += R(0.5) * (Vn + fabs(Vn)) * c.sa_dstar[q - sI];
                }
                if (j > 0) {
                    const R Vn = vdotS(q - nk, 1, fJ);
                    rhs += R(0.5) * (Vn + fabs(Vn)) * c.sa_dstar[q - nk];
                }
                if (three && k > 0) {
                    const R Vn = vdotS(q - 1, 2, fK);
                    rhs += R(0.5) * (Vn + fabs(Vn)) * c.sa_dstar[q - 1];
                }
                c.sa_dstar[q] = rhs / c.sa_diag[q];
            } else {
                R sum = R(0);
                if (i + 1 < ni) {
                    const R Vn = vdotS(q + sI, 0, fI + sI);
                    sum += R(0.5) * (fabs(Vn) - Vn) * c.sa_dnu[q + sI];
                }
                if (j + 1 < nj) {
                    const R Vn = vdotS(q + nk, 1, fJ + nk);
                    sum += R(0.5) * (fabs(Vn) - Vn) * c.sa_dnu[q + nk];
                }
                if (three && k + 1 < nk) {
                    const R Vn = vdotS(q + 1, 2, fK + 1);
                    sum += R(0.5) * (fabs(Vn) - Vn) * c.sa_dnu[q + 1];
                }
                c.sa_dnu[q] = c.sa_dstar[q] + sum / c.sa_diag[q];
            }
        }
        __syncthreads();
    }
}

// Step 4 of updateSolution (src/turbulence_model_sa.cpp:808-840): nu hat +
// under-relaxed increment, clamped to +-1e5 max(nu, 1e-12); an increment that
// is NaN or Inf stops the instance as diverged (the reference throws
// "Turbulence model diverged").
template <typename R>
__global__ void __launch_bounds__(256) k_sa_update(const DevCaseT<R>* cases, const Tile* tiles, int force) {
    __shared__ DevCaseT<R> c;
    Tile tl;
    if (!enter(cases, tiles, c, 0, force, tl)) return;
    const R relax = R(c.sa_relax);
    bool bad = false;
    for (long long q = tl.start + threadIdx.x; q < tl.start + tl.count; q += blockDim.x) {
        const R dNu = c.sa_dnu[q] * relax;
        if (isnan(dNu) || isinf(dNu)) bad = true;
        R nn = c.nuhat[q] + dNu;
        const R mx = R(1.0e5) * rmax(c.nul[q], R(1e-12));
        nn = rmax(-mx, rmin(nn, mx));
        c.nuhat[q] = nn;
    }
    if (bad) c.ctl->status = 2;
}
