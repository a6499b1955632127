// Node source terms of the explicit loop: axisymmetric and blade-row
// geometric sources, the Gong term and the body-force models (blockage, Hall,
// Hall-Thollet, Lift-Drag), templated on the working precision, reference
// evaluation order.
#pragma once

#include "physics.cuh"

namespace ctbfm {

template <typename R>
CTBFM_DI long long nodeIdx(const DevCaseT<R>& c, long long i, long long j, long long k) {
    return (i * c.nj + j) * c.nk + k;
}

// Config::getRotationalSpeedScalingFactor(time) (src/config.cpp:695-718).
template <typename R>
CTBFM_DI double speedScaling(const DevCaseT<R>& c, double t) {
    if (!c.accel) return c.speed_scale;
    if (t < c.acc_t0 || t > c.acc_t1) return c.speed_scale;
    return c.acc_s0 + (c.acc_s1 - c.acc_s0) * (t - c.acc_t0) / (c.acc_t1 - c.acc_t0);
}

// Solver::computeGongSource (src/solver.cpp:3074-3145).
template <typename R>
CTBFM_DI S5<R> gongSource(const DevCaseT<R>& c, R* const* U, R omega, int i, int j, int k, R vol) {
    if (fabs(omega) < R(1E-3)) return zero5<R>();
    const int nk = c.nk;
    long long q0, q1, q2;
    if (omega > R(0)) {
        if (k == 0) { q0 = nodeIdx(c, i, j, k); q1 = nodeIdx(c, i, j, nk - 2); q2 = nodeIdx(c, i, j, nk - 3); }
        else if (k == 1) { q0 = nodeIdx(c, i, j, k); q1 = nodeIdx(c, i, j, 0); q2 = nodeIdx(c, i, j, nk - 2); }
        else { q0 = nodeIdx(c, i, j, k); q1 = nodeIdx(c, i, j, k - 1); q2 = nodeIdx(c, i, j, k - 2); }
    } else {
        if (k == nk - 1) { q0 = nodeIdx(c, i, j, 0); q1 = nodeIdx(c, i, j, 1); q2 = nodeIdx(c, i, j, 2); }
        else if (k == nk - 2) { q0 = nodeIdx(c, i, j, k); q1 = nodeIdx(c, i, j, 0); q2 = nodeIdx(c, i, j, 1); }
        else { q0 = nodeIdx(c, i, j, k); q1 = nodeIdx(c, i, j, k + 1); q2 = nodeIdx(c, i, j, k + 2); }
    }
    const S5<R> U0 = load5(U, q0), U1 = load5(U, q1), U2 = load5(U, q2);
    const R dth = R(2 * M_PI / static_cast<double>(nk - 1));
    S5<R> d;
    if (omega > R(0)) d = ((U0 * R(3) - U1 * R(4)) + U2) / (R(2) * dth);
    else d = ((U0 * R(-3) + U1 * R(4)) - U2) / (R(2) * dth);
    S5<R> src;
#pragma unroll
    for (int v = 0; v < 5; v++) src.v[v] = -d.v[v] * omega;
    return src * vol;
}

// SourceBFMBase::computeFlowState (src/source_bfm_base.cpp:104-149).
template <typename R>
struct BfmState {
    R radius, omega, pitch, staggered, blockage, flowAngle, dev, cth, sth, vmer;
    V3<R> relCyl, relCart, nCyl, invDirCyl, viscDirCyl;
};

// SourceBFMBase::computeDeviationAngle (src/source_bfm_base.cpp:152-166),
// given the camber normal over its magnitude nn.
template <typename R>
CTBFM_DI R bfmDeviation(V3<R> rel, V3<R> nn) {
    const V3<R> vm = v3(rel.x, rel.y, R(0));
    V3<R> span = v3(-vm.y, vm.x, R(0));
    span = span / mag(span);
    const V3<R> vin = rel - span * dot(rel, span);
    const R nv = dot(vin, nn);
    return -asin(nv / mag(vin));
}

// SourceBFMBase::computeInviscidForceDirection (src/source_bfm_base.cpp:168-199),
// given the normalized camber normal nd (zero for a zero normal).
template <typename R>
CTBFM_DI V3<R> bfmInviscidDir(const DevCaseT<R>& c, V3<R> rel, V3<R> nd, R dev, long long q) {
    const V3<R> rd = normalized(rel);
    V3<R> ver;
    if (c.stalled && dev > c.devstall[q]) ver = nd;
    else ver = normalized(nd - rd * dot(nd, rd));
    const V3<R> vm = v3(rel.x, rel.y, R(0));
    const V3<R> sd = normalized(v3(vm.y, -vm.x, R(0)));
    return normalized(ver - sd * dot(ver, sd));
}

// A node's blade fields, loaded together before the tests that decide
// whether they are used (blockage gradient, blade count), so that the loads
// overlap instead of waiting on one another.
template <typename R>
struct BfmNode {
    V3<R> gb;  // blockage gradient
    R blk, nbl;
    R radius, cth, sth, omega0, pitch;  // the force models' fields (zero for None / Blockage)
    V3<R> n, nhat;
};

template <typename R>
CTBFM_DI bool bfmForceModel(const DevCaseT<R>& c) {
    return c.bfm_model == 1 || c.bfm_model == 2 || c.bfm_model == 3 || c.bfm_model == 5 || c.bfm_model == 6;
}

template <typename R>
CTBFM_DI BfmNode<R> loadBfmNode(const DevCaseT<R>& c, long long q) {
    BfmNode<R> f;
    f.gb = v3(c.gbx[q], c.gby[q], c.gbz[q]);
    f.blk = c.blk[q];
    f.nbl = c.nblades[q];
    if (bfmForceModel(c)) {
        f.radius = c.radius[q];
        f.cth = c.cost[q];
        f.sth = c.sint[q];
        f.omega0 = c.omega0[q];
        f.pitch = c.pitch[q];
        f.n = v3(c.nax[q], c.nrad[q], c.ntan[q]);
        f.nhat = v3(c.nhat[0][q], c.nhat[1][q], c.nhat[2][q]);
    } else {
        f.radius = f.cth = f.sth = f.omega0 = f.pitch = R(0);
        f.n = f.nhat = v3(R(0), R(0), R(0));
    }
    return f;
}

template <typename R>
CTBFM_DI void bfmFlowState(const DevCaseT<R>& c, long long q, const S5<R>& W, double t, const BfmNode<R>& f,
                           BfmState<R>& b) {
    b.radius = f.radius;
    b.cth = f.cth;
    b.sth = f.sth;
    const V3<R> velCyl = cylOfCart(velOf(W), b.cth, b.sth);
    b.omega = f.omega0;  // rpm 2 pi / 60
    b.omega *= R(speedScaling(c, t));
    const V3<R> drag = v3(R(0), R(0), b.omega * b.radius);
    b.relCyl = velCyl - drag;
    b.relCart = cartOfCyl(b.relCyl, b.cth, b.sth);
    const R vmer = sqrt(velCyl.x * velCyl.x + velCyl.y * velCyl.y);
    b.vmer = vmer;
    b.pitch = f.pitch;  // 2 pi r / N
    b.nCyl = f.n;
    // the camber normal over its magnitude; normalized() gives zero where the
    // magnitude is zero, which the division leaves non-finite
    const V3<R> nn = f.nhat;
    const bool finite = isfinite(nn.x) && isfinite(nn.y) && isfinite(nn.z);
    b.blockage = f.blk;
    if (c.bfm_model == 3) {  // only Lift-Drag reads the staggered pitch and flow angle
        b.staggered = b.pitch * c.cosmetal[q];
        b.flowAngle = atan2(b.relCyl.z, vmer);
    } else {
        b.staggered = R(0);
        b.flowAngle = R(0);
    }
    b.dev = bfmDeviation(b.relCyl, nn);
    b.invDirCyl = bfmInviscidDir(c, b.relCyl, finite ? nn : v3(R(0), R(0), R(0)), b.dev, q);
    b.viscDirCyl = -normalized(b.relCyl);
}

template <typename R>
CTBFM_DI S5<R> forceSource(V3<R> fcyl, const BfmState<R>& b, R vol, R rho) {
    const V3<R> fc = cartOfCyl(fcyl, b.cth, b.sth);
    const S5<R> src = s5(R(0), fc.x, fc.y, fc.z, fcyl.z * b.omega * b.radius);
    return (src * vol) * rho;
}

// SourceBFMThollet::computeCompressibilityCorrection (src/source_bfm_thollet.cpp:48-70).
template <typename R>
CTBFM_DI R tholletKmach(Gas<R> gs, V3<R> rel, const S5<R>& W) {
    const R a = soundSpeed_rho_u_et(gs, W.v[0], velOf(W), W.v[4]);
    R M = mag(rel) / a;
    if (fabs(M - R(1)) < R(1E-03)) M = R(0.999);
    R kp;
    if (M < R(1)) kp = R(1) / sqrt(R(1) - M * M);
    else kp = R(2) / R(M_PI) / sqrt(M * M - R(1));
    return rmin(R(3), kp);
}

// SourceBFMChima::computeBodyForceSource (src/source_bfm_chima.cpp:16-190).
// Not inlined, like correlationsForce: the rarely used models stay out of
// the node kernel's registers.
template <typename R>
__device__ __noinline__ S5<R> chimaForce(const DevCaseT<R>& c, Gas<R> gs, int j, int k, long long q, const S5<R>& W,
                                         const BfmState<R>& b, R vol) {
    // SourceBFMChima::computeDerivativeFunction (:180-190): parabolic
    auto deriv = [](R yF, R xL, R xF) { return R(-2.0) * yF * xL / (xF * xF) + R(2.0) * yF / xF; };
    const R sLoc = c.stwl[q];
    const R sTe = c.stwl[nodeIdx(c, c.te_idx, j, k)];
    const V3<R> u = velOf(W);
    // viscous component first (:146-178); its tangential force enters the inviscid one
    const R dSdM = deriv(c.dentropy[q], sLoc, sTe) * R(c.ctl->chima_loss);
    const R T = temperature_rho_u_et(gs, W.v[0], u, W.v[4]);
    const R fv = T * b.vmer / mag(b.relCyl) * dSdM;
    const V3<R> fvCyl = b.viscDirCyl * fv;
    const S5<R> visc = forceSource(fvCyl, b, vol, W.v[0]);
    // inviscid component (:51-83)
    const R dLdM = deriv(c.dangmom[q], sLoc, sTe) * R(c.ctl->chima_turn);
    const R ftan = dLdM * b.vmer / b.radius;
    const R fi = (ftan - fvCyl.z) / b.invDirCyl.z;
    const S5<R> inv = forceSource(b.invDirCyl * fi, b, vol, W.v[0]);
    return inv + visc;
}

// SourceBFMCorrelations (src/source_bfm_correlations.cpp:12-236): the
// turning force from incidence / deviation correlations evaluated between the
// leading and trailing edge of the node's (j, k) line, on the stage state U;
// the viscous component is zero.
template <typename R>
__device__ __noinline__ S5<R> correlationsForce(const DevCaseT<R>& c, Gas<R> gs, R* const* U, int j, int k, long long q,
                                 const S5<R>& W, const BfmState<R>& b, R vol) {
    const long long qle = nodeIdx(c, c.le_idx, j, k), qte = nodeIdx(c, c.te_idx, j, k);
    // computeCorrelationParameters (:33-85)
    const R sle = c.stwl[qle], ste = c.stwl[qte];
    const R sol = (ste - sle) / b.pitch;
    const S5<R> Wi = primOf(load5(U, qle)), Wo = primOf(load5(U, qte));
    const V3<R> vic = cylOfCart(velOf(Wi), b.cth, b.sth), voc = cylOfCart(velOf(Wo), b.cth, b.sth);
    const R rIn = c.radius[qle], rOut = c.radius[qte];
    const V3<R> relIn = vic - v3(R(0), R(0), b.omega * rIn);
    const V3<R> relOut = voc - v3(R(0), R(0), b.omega * rOut);
    const R vmIn = sqrt(relIn.x * relIn.x + relIn.y * relIn.y);
    const R flowInDeg = atan2(relIn.z, vmIn) * R(180.0) / R(M_PI);
    const R chordM = ste - sle;
    const R camberAbs = fabs(c.metal[qte] - c.metal[qle]) * R(180) / R(M_PI);
    // computeInviscidComponent (:88-210)
    const R k1 = c.metal[qle] * R(180) / R(M_PI);
    const R k2 = c.metal[qte] * R(180) / R(M_PI);
    const R inc = flowInDeg - k1;
    const R aAbs = fabs(flowInDeg);
    const R n = R(0.025) * sol - R(0.06) - (pow(aAbs / R(90.0), R(1.0) + R(1.2) * sol)) / (R(1.5) + R(0.43) * sol);
    const R p = R(0.914) + sol * sol * sol / R(160.0);
    const R i0 = pow(aAbs, p) / (R(5.0) + R(46.0) * exp(R(-2.3) * sol)) -
                 R(0.1) * pow(sol, R(3.0)) * exp((aAbs - R(70.0)) / R(4.0));
    R thk = R(0);
    for (int s = c.le_idx; s <= c.te_idx; ++s) {
        const long long qs = nodeIdx(c, s, j, k);
        const R pitch = R(2.0) * R(M_PI) * c.radius[qs] / c.nblades[q];
        const R t = pitch * (R(1.0) - c.blk[qs]);
        if (t > thk) thk = t;
    }
    const R tc = thk / chordM;
    const R Kti = pow(R(10.0) * tc, R(0.28) / (R(0.1) + pow(tc, R(0.3))));
    const R Ksh = R(0.8);
    const R istar = Ksh * Kti * i0 + n * camberAbs;
    const R a = soundSpeed_rho_u_et(gs, W.v[0], velOf(W), W.v[4]);
    const R mach = mag(b.relCart) / a;
    const R istarC = istar + R(1.3026) * mach + R(5.7380);
    const R dev10 = R(0.01) * sol * aAbs +
                    (R(0.74) * pow(sol, R(1.9)) + R(3.0) * sol) * pow(aAbs / R(90.0), R(1.67) + R(1.09) * sol);
    const R Ktd = R(6.25) * tc + R(37.5) * tc * tc;
    const R ac = R(0.3);
    const R devStar = (R(0.92) * ac * ac + R(0.002) * fabs(k2)) / (R(1) - R(0.002) * camberAbs / sqrt(sol)) *
                          camberAbs / sqrt(sol) +
                      (Ksh * Ktd - R(1.0)) * dev10;
    const R devStarC = R(-1.099379) + R(3.0186) * devStar - R(0.1988) * devStar * devStar;
    const R ddi = (R(1.0) + (sol + R(0.25) * pow(sol, R(4.0))) * pow((aAbs / R(53.0)), R(2.5))) / exp(R(3.1) * sol);
    const R umIn = sqrt(relIn.x * relIn.x + relIn.y * relIn.y);
    const R umOut = sqrt(relOut.x * relOut.x + relOut.y * relOut.y);
    const R incMag = b.omega > R(0.0) ? inc * R(-1.0) : inc;
    const R devOut = devStarC + ddi * (incMag - istarC) + R(10.0) * (R(1.0) - umOut / umIn);
    const R loc = (c.stwl[q] - sle) / (ste - sle);
    const R devExpDeg = incMag + loc * (devOut - incMag);
    const R devExp = devExpDeg * R(M_PI) / R(180.0);
    const R uth = b.relCyl.z;
    const R kappa = c.metal[q];
    R Wn;
    if (b.omega > R(0.0)) {
        const R uexp = b.vmer * tan(-devExp + kappa);
        Wn = uexp - uth;
    } else {
        const R uexp = b.vmer * tan(devExp + kappa);
        Wn = -uexp + uth;
    }
    const R fn = R(c.kn) * b.vmer * Wn / (b.pitch * fabs(c.cosmetal[q]));
    const V3<R> dirCart = cartOfCyl(b.invDirCyl, b.cth, b.sth);
    const V3<R> fc = dirCart * fn;
    const V3<R> fy = b.invDirCyl * fn;
    const S5<R> inv = (s5(R(0), fc.x, fc.y, fc.z, fy.z * b.omega * b.radius) * vol) * W.v[0];
    const R zero = R(0);
    const S5<R> visc = (s5(R(0), zero, zero, zero, zero * b.omega * b.radius) * vol) * W.v[0];
    return inv + visc;
}

// computeBodyForceSource of SourceBFMHall (src/source_bfm_hall.cpp:3-34),
// SourceBFMThollet (src/source_bfm_thollet.cpp:3-138) and SourceBFMLiftDrag
// (src/source_bfm_lift_drag.cpp:3-88).
template <int BX, typename R>
CTBFM_DI S5<R> bfmBodyForce(const DevCaseT<R>& c, Gas<R> gs, R* const* U, int i, int j, int k, long long q,
                            const S5<R>& W, double t, const BfmNode<R>& f) {
    // SourceBFMBase::computeBodyForceSource: no force for "None" / "Blockage"
    if (c.bfm_model != 1 && c.bfm_model != 2 && c.bfm_model != 3 && c.bfm_model != 5 && c.bfm_model != 6)
        return zero5<R>();
    BfmState<R> b;
    bfmFlowState(c, q, W, t, f, b);
    const R vol = c.vol[q];
    if (BX) {  // the node-kernel variant of the Chima and Correlations models
        if (c.bfm_model == 5) return chimaForce(c, gs, j, k, q, W, b, vol);
        return correlationsForce(c, gs, U, j, k, q, W, b, vol);
    }
    const R w2 = dot(b.relCyl, b.relCyl);
    if (c.bfm_model == 1) {  // Hall
        const R fm = w2 * R(M_PI) * b.dev / b.pitch / fabs(b.nCyl.z);
        return forceSource(b.invDirCyl * fm, b, vol, W.v[0]);
    }
    if (c.bfm_model == 2) {  // Hall-Thollet
        const R km = tholletKmach(gs, b.relCyl, W);
        const R fm = R(c.kn) * km * w2 * R(M_PI) * b.dev / b.pitch / fabs(b.nCyl.z) / b.blockage;
        const S5<R> inv = forceSource(b.invDirCyl * fm, b, vol, W.v[0]);
        S5<R> visc;
        if (c.stalled && b.dev > c.devstall[q]) {
            visc = zero5<R>();
        } else {
            R stwl = c.stwl[q];
            if (stwl < R(1E-06)) {
                if (i + 1 < c.ni) stwl = (c.stwl[nodeIdx(c, i + 1, j, k)] + c.stwl[q]) / R(2);
                if (stwl < R(1E-06)) stwl = R(1E-06);
            }
            const R rex = mag(b.relCyl) * stwl / R(c.nu);
            const R cf = R(0.0592) * pow(rex, R(-0.2));
            R fmv;
            if (!c.offdesign) {
                fmv = w2 / (b.pitch * b.blockage * fabs(b.nCyl.z)) * (R(c.kf) * cf);
            } else {
                const R km2 = tholletKmach(gs, b.relCyl, W);
                fmv = w2 / (b.pitch * b.blockage * fabs(b.nCyl.z)) *
                      (R(c.kf) * cf + R(M_PI) * km2 * pow(fabs(b.dev - c.devpivot[q]), R(2) * R(c.kd)));
            }
            visc = forceSource(b.viscDirCyl * fmv, b, vol, W.v[0]);
        }
        return inv + visc;
    }
    // Lift-Drag
    const R chord = c.stwl[nodeIdx(c, c.te_idx, j, k)] - c.stwl[nodeIdx(c, c.le_idx, j, k)];
    const R sol = chord / b.pitch;
    const R w = mag(b.relCart);
    const R beta0 = c.ldbeta0[q];
    const R sgn = (b.nCyl.z >= R(0)) ? R(1) : R(-1);
    const R fm = R(0.5) * w * w * R(2) * R(M_PI) / b.staggered * sgn * (-b.flowAngle + beta0);
    const S5<R> inv = forceSource(b.invDirCyl * fm, b, vol, W.v[0]);
    const R d = b.flowAngle - beta0;
    const R kp = c.ldkp[q] + R(2) * R(M_PI) * sol * (d * d);
    const R fmv = kp * w * w / b.staggered;
    const S5<R> visc = forceSource(b.viscDirCyl * fmv, b, vol, W.v[0]);
    return inv + visc;
}

// SourceBFMBase::computePerturbationFactor (src/source_bfm_base.cpp:215-243).
template <typename R>
CTBFM_DI R bfmPerturbation(const DevCaseT<R>& c, long long q, double t) {
    if (!c.perturb) return R(0);
    if (t < c.pert_t0 || t > c.pert_t0 + c.pert_dur) return R(0);
    const V3<double> p = v3(c.vx[q], c.vy[q], c.vz[q]);
    const double dist = mag(p - v3(c.pert_c[0], c.pert_c[1], c.pert_c[2]));
    if (dist > 3.0 * c.pert_r) return R(0);
    const double sm = exp(-(dist * dist) / (c.pert_r * c.pert_r));
    const double peak = c.pert_t0 + c.pert_dur / 2.0;
    const double sig = c.pert_dur / 3.0;
    const double dtp = t - peak;
    const double tm = exp(-(dtp * dtp) / (sig * sig));
    return R(c.pert_s * sm * tm);
}

// SourceBFMBase::computeTotalSource (src/source_bfm_base.cpp:25-84).
template <int BX, typename R>
CTBFM_DI S5<R> bfmTotalSource(const DevCaseT<R>& c, Gas<R> gs, R* const* U, int i, int j, int k, long long q,
                              const S5<R>& W, double t, const BfmNode<R>& f) {
    S5<R> blk = zero5<R>();
    if (c.blockage) {
        const V3<R> u = velOf(W);
        const R ht = totalEnthalpy_rho_u_et(gs, W.v[0], u, W.v[4]);
        const R ct = R(-1) / f.blk * W.v[0] * dot(u, f.gb);
        blk = s5(ct, ct * u.x, ct * u.y, ct * u.z, ct * ht) * c.vol[q];
    }
    if (f.nbl == R(0)) return blk;
    const S5<R> bf = bfmBodyForce<BX>(c, gs, U, i, j, k, q, W, t, f);
    const R pf = bfmPerturbation(c, q, t);
    return blk + bf * (R(1) + pf);
}

// Solver::computeSourceResiduals (src/solver.cpp:2790-2924) applied to one
// node's residual R, given the node's primitives W and pressure p of the
// stage input (the values primOf and pressure_rho_u_et give for it).
template <int BX, typename R>
CTBFM_DI void applySourcesW(const DevCaseT<R>& c, Gas<R> gs, R* const* U, int i, int j, int k, long long q,
                            const S5<R>& W, R p, double t, S5<R>& Res) {
    const R vol = c.vol[q];
    bool geo = false, gong = false;
    if (c.topo == 1) geo = gong = (c.bpresent[q] > R(0));
    else if (c.topo == 2) geo = true;
    if (geo) {
        const R cth = c.cost[q], sth = c.sint[q];
        const V3<R> vc = cylOfCart(velOf(W), cth, sth);
        V3<R> sc;
        sc.x = R(0);
        if (c.topo == 2) {
            const R gf = c.areaK0[q] * R(c.wedge);
            sc.y = (+W.v[0] * vc.z * vc.z + p) * gf;
            sc.z = -W.v[0] * vc.y * vc.z * gf;
            const V3<R> sCart = cartOfCyl(sc, cth, sth);
            Res = Res - s5(R(0), sCart.x, sCart.y, sCart.z, R(0));
        } else {
            const R r = c.radius[q];
            sc.y = (+W.v[0] * vc.z * vc.z + p) / r;
            sc.z = -W.v[0] * vc.y * vc.z / r;
            const V3<R> sCart = cartOfCyl(sc, cth, sth);
            Res = Res - s5(R(0), sCart.x, sCart.y, sCart.z, R(0)) * vol;
        }
    }
    if (gong) {
        R om = c.rpm[q] * R(2) * R(M_PI) / R(60);
        om *= R(speedScaling(c, t));
        Res = Res - gongSource(c, U, om, i, j, k, vol);
    }
    if (c.bfm) {
        const BfmNode<R> f = loadBfmNode(c, q);
        if (mag(f.gb) > R(1E-10)) Res = Res - bfmTotalSource<BX>(c, gs, U, i, j, k, q, W, t, f);
    }
}

template <typename R>
CTBFM_DI bool hasSources(const DevCaseT<R>& c) {
    return c.topo == 2 || c.bfm;
}

// The same from the node's conservative stage input.
template <int BX, typename R>
CTBFM_DI void applySources(const DevCaseT<R>& c, Gas<R> gs, R* const* U, int i, int j, int k, long long q,
                           const S5<R>& Unode, double t, S5<R>& Res) {
    if (!hasSources(c)) return;
    const S5<R> W = primOf(Unode);
    applySourcesW<BX>(c, gs, U, i, j, k, q, W, pressure_rho_u_et(gs, W.v[0], velOf(W), W.v[4]), t, Res);
}

}  // namespace ctbfm
