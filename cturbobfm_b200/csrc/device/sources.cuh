// Node source terms of the explicit loop: axisymmetric and blade-row
// geometric sources, the Gong term and the body-force models (blockage, Hall,
// Hall-Thollet, Lift-Drag) as device functions, reference evaluation order.
#pragma once

#include "physics.cuh"

namespace ctbfm {

CTBFM_DI long long nodeIdx(const DevCase& c, long long i, long long j, long long k) {
    return (i * c.nj + j) * c.nk + k;
}

// Config::getRotationalSpeedScalingFactor(time) (src/config.cpp:695-718).
CTBFM_DI double speedScaling(const DevCase& c, double t) {
    if (!c.accel) return c.speed_scale;
    if (t < c.acc_t0 || t > c.acc_t1) return c.speed_scale;
    return c.acc_s0 + (c.acc_s1 - c.acc_s0) * (t - c.acc_t0) / (c.acc_t1 - c.acc_t0);
}

// Solver::computeGongSource (src/solver.cpp:3074-3145).
CTBFM_DI S5 gongSource(const DevCase& c, double* const* U, double omega, int i, int j, int k, double vol) {
    if (fabs(omega) < 1E-3) return zero5();
    const int nk = c.nk;
    long long q0, q1, q2;
    if (omega > 0) {
        if (k == 0) { q0 = nodeIdx(c, i, j, k); q1 = nodeIdx(c, i, j, nk - 2); q2 = nodeIdx(c, i, j, nk - 3); }
        else if (k == 1) { q0 = nodeIdx(c, i, j, k); q1 = nodeIdx(c, i, j, 0); q2 = nodeIdx(c, i, j, nk - 2); }
        else { q0 = nodeIdx(c, i, j, k); q1 = nodeIdx(c, i, j, k - 1); q2 = nodeIdx(c, i, j, k - 2); }
    } else {
        if (k == nk - 1) { q0 = nodeIdx(c, i, j, 0); q1 = nodeIdx(c, i, j, 1); q2 = nodeIdx(c, i, j, 2); }
        else if (k == nk - 2) { q0 = nodeIdx(c, i, j, k); q1 = nodeIdx(c, i, j, 0); q2 = nodeIdx(c, i, j, 1); }
        else { q0 = nodeIdx(c, i, j, k); q1 = nodeIdx(c, i, j, k + 1); q2 = nodeIdx(c, i, j, k + 2); }
    }
    const S5 U0 = load5(U, q0), U1 = load5(U, q1), U2 = load5(U, q2);
    const double dth = (2 * M_PI / static_cast<double>(nk - 1));
    S5 d;
    if (omega > 0.0) d = ((U0 * 3.0 - U1 * 4.0) + U2) / (2 * dth);
    else d = ((U0 * (-3.0) + U1 * 4.0) - U2) / (2 * dth);
    S5 src;
#pragma unroll
    for (int v = 0; v < 5; v++) src.v[v] = -d.v[v] * omega;
    return src * vol;
}

// SourceBFMBase::computeFlowState (src/source_bfm_base.cpp:104-149).
struct BfmState {
    double radius, omega, pitch, staggered, blockage, flowAngle, dev, cth, sth;
    D3 relCyl, relCart, nCyl, invDirCyl, viscDirCyl;
};

// SourceBFMBase::computeDeviationAngle (src/source_bfm_base.cpp:152-166).
CTBFM_DI double bfmDeviation(D3 rel, D3 ncam) {
    const D3 nn = ncam / mag(ncam);
    const D3 vm = d3(rel.x, rel.y, 0.0);
    D3 span = d3(-vm.y, vm.x, 0.0);
    span = span / mag(span);
    const D3 vin = rel - span * dot(rel, span);
    const double nv = dot(vin, nn);
    return -asin(nv / mag(vin));
}

// SourceBFMBase::computeInviscidForceDirection (src/source_bfm_base.cpp:168-199).
CTBFM_DI D3 bfmInviscidDir(const DevCase& c, D3 rel, D3 ncam, double dev, long long q) {
    const D3 rd = normalized(rel);
    const D3 nd = normalized(ncam);
    D3 ver;
    if (c.stalled && dev > c.devstall[q]) ver = nd;
    else ver = normalized(nd - rd * dot(nd, rd));
    const D3 vm = d3(rel.x, rel.y, 0.0);
    const D3 sd = normalized(d3(vm.y, -vm.x, 0.0));
    return normalized(ver - sd * dot(ver, sd));
}

CTBFM_DI void bfmFlowState(const DevCase& c, long long q, const S5& W, double t, BfmState& b) {
    b.radius = c.radius[q];
    b.cth = c.cost[q];
    b.sth = c.sint[q];
    const D3 velCyl = cylOfCart(velOf(W), b.cth, b.sth);
    b.omega = c.rpm[q] * 2 * M_PI / 60;
    b.omega *= speedScaling(c, t);
    const D3 drag = d3(0, 0, b.omega * b.radius);
    b.relCyl = velCyl - drag;
    b.relCart = cartOfCyl(b.relCyl, b.cth, b.sth);
    const double vmer = sqrt(velCyl.x * velCyl.x + velCyl.y * velCyl.y);
    const double nb = c.nblades[q];
    b.pitch = 2.0 * M_PI * b.radius / nb;
    b.nCyl = d3(c.nax[q], c.nrad[q], c.ntan[q]);
    b.blockage = c.blk[q];
    if (c.bfm_model == 3) {  // only Lift-Drag reads the staggered pitch and flow angle
        b.staggered = b.pitch * c.cosmetal[q];
        b.flowAngle = atan2(b.relCyl.z, vmer);
    } else {
        b.staggered = 0.0;
        b.flowAngle = 0.0;
    }
    b.dev = bfmDeviation(b.relCyl, b.nCyl);
    b.invDirCyl = bfmInviscidDir(c, b.relCyl, b.nCyl, b.dev, q);
    b.viscDirCyl = -normalized(b.relCyl);
}

CTBFM_DI S5 forceSource(D3 fcyl, const BfmState& b, double vol, double rho) {
    const D3 fc = cartOfCyl(fcyl, b.cth, b.sth);
    const S5 src = s5(0, fc.x, fc.y, fc.z, fcyl.z * b.omega * b.radius);
    return (src * vol) * rho;
}

// SourceBFMThollet::computeCompressibilityCorrection (src/source_bfm_thollet.cpp:48-70).
CTBFM_DI double tholletKmach(Gas gs, D3 rel, const S5& W) {
    const double a = soundSpeed_rho_u_et(gs, W.v[0], velOf(W), W.v[4]);
    double M = mag(rel) / a;
    if (fabs(M - 1.0) < 1E-03) M = 0.999;
    double kp;
    if (M < 1.0) kp = 1.0 / sqrt(1.0 - M * M);
    else kp = 2.0 / M_PI / sqrt(M * M - 1.0);
    return dmin(3.0, kp);
}

// computeBodyForceSource of SourceBFMHall (src/source_bfm_hall.cpp:3-34),
// SourceBFMThollet (src/source_bfm_thollet.cpp:3-138) and SourceBFMLiftDrag
// (src/source_bfm_lift_drag.cpp:3-88).
CTBFM_DI S5 bfmBodyForce(const DevCase& c, Gas gs, int i, int j, int k, long long q, const S5& W, double t) {
    // SourceBFMBase::computeBodyForceSource: no force for "None" / "Blockage"
    if (c.bfm_model != 1 && c.bfm_model != 2 && c.bfm_model != 3) return zero5();
    BfmState b;
    bfmFlowState(c, q, W, t, b);
    const double vol = c.vol[q];
    const double w2 = dot(b.relCyl, b.relCyl);
    if (c.bfm_model == 1) {  // Hall
        const double fm = w2 * M_PI * b.dev / b.pitch / fabs(b.nCyl.z);
        return forceSource(b.invDirCyl * fm, b, vol, W.v[0]);
    }
    if (c.bfm_model == 2) {  // Hall-Thollet
        const double km = tholletKmach(gs, b.relCyl, W);
        const double fm = c.kn * km * w2 * M_PI * b.dev / b.pitch / fabs(b.nCyl.z) / b.blockage;
        const S5 inv = forceSource(b.invDirCyl * fm, b, vol, W.v[0]);
        S5 visc;
        if (c.stalled && b.dev > c.devstall[q]) {
            visc = zero5();
        } else {
            double stwl = c.stwl[q];
            if (stwl < 1E-06) {
                if (i + 1 < c.ni) stwl = (c.stwl[nodeIdx(c, i + 1, j, k)] + c.stwl[q]) / 2.0;
                if (stwl < 1E-06) stwl = 1E-06;
            }
            const double rex = mag(b.relCyl) * stwl / c.nu;
            const double cf = 0.0592 * pow(rex, -0.2);
            double fmv;
            if (!c.offdesign) {
                fmv = w2 / (b.pitch * b.blockage * fabs(b.nCyl.z)) * (c.kf * cf);
            } else {
                const double km2 = tholletKmach(gs, b.relCyl, W);
                fmv = w2 / (b.pitch * b.blockage * fabs(b.nCyl.z)) *
                      (c.kf * cf + M_PI * km2 * pow(fabs(b.dev - c.devpivot[q]), 2.0 * c.kd));
            }
            visc = forceSource(b.viscDirCyl * fmv, b, vol, W.v[0]);
        }
        return inv + visc;
    }
    if (c.bfm_model == 3) {  // Lift-Drag
        const double chord = c.stwl[nodeIdx(c, c.te_idx, j, k)] - c.stwl[nodeIdx(c, c.le_idx, j, k)];
        const double sol = chord / b.pitch;
        const double w = mag(b.relCart);
        const double beta0 = c.ldbeta0[q];
        const double sgn = (b.nCyl.z >= 0.0) ? 1.0 : -1.0;
        const double fm = 0.5 * w * w * 2.0 * M_PI / b.staggered * sgn * (-b.flowAngle + beta0);
        const S5 inv = forceSource(b.invDirCyl * fm, b, vol, W.v[0]);
        const double d = b.flowAngle - beta0;
        const double kp = c.ldkp[q] + 2.0 * M_PI * sol * (d * d);
        const double fmv = kp * w * w / b.staggered;
        const S5 visc = forceSource(b.viscDirCyl * fmv, b, vol, W.v[0]);
        return inv + visc;
    }
    return zero5();
}

// SourceBFMBase::computePerturbationFactor (src/source_bfm_base.cpp:215-243).
CTBFM_DI double bfmPerturbation(const DevCase& c, long long q, double t) {
    if (!c.perturb) return 0.0;
    if (t < c.pert_t0 || t > c.pert_t0 + c.pert_dur) return 0.0;
    const D3 p = d3(c.vx[q], c.vy[q], c.vz[q]);
    const double dist = mag(p - d3(c.pert_c[0], c.pert_c[1], c.pert_c[2]));
    if (dist > 3.0 * c.pert_r) return 0.0;
    const double sm = exp(-(dist * dist) / (c.pert_r * c.pert_r));
    const double peak = c.pert_t0 + c.pert_dur / 2.0;
    const double sig = c.pert_dur / 3.0;
    const double dtp = t - peak;
    const double tm = exp(-(dtp * dtp) / (sig * sig));
    return c.pert_s * sm * tm;
}

// SourceBFMBase::computeTotalSource (src/source_bfm_base.cpp:25-84).
CTBFM_DI S5 bfmTotalSource(const DevCase& c, Gas gs, int i, int j, int k, long long q, const S5& W, double t) {
    S5 blk = zero5();
    if (c.blockage) {
        const D3 u = velOf(W);
        const double ht = totalEnthalpy_rho_u_et(gs, W.v[0], u, W.v[4]);
        const D3 gb = d3(c.gbx[q], c.gby[q], c.gbz[q]);
        const double ct = -1.0 / c.blk[q] * W.v[0] * dot(u, gb);
        blk = s5(ct, ct * u.x, ct * u.y, ct * u.z, ct * ht) * c.vol[q];
    }
    if (c.nblades[q] == 0) return blk;
    const S5 bf = bfmBodyForce(c, gs, i, j, k, q, W, t);
    const double pf = bfmPerturbation(c, q, t);
    return blk + bf * (1.0 + pf);
}

// Solver::computeSourceResiduals (src/solver.cpp:2790-2924) applied to one
// node's residual R.
CTBFM_DI void applySources(const DevCase& c, Gas gs, double* const* U, int i, int j, int k, long long q, const S5& Unode,
                           double t, S5& R) {
    if (c.topo == 1 && !c.bfm) return;
    if (c.topo == 0 && !c.bfm) return;
    const S5 W = primOf(Unode);
    const double vol = c.vol[q];
    const double p = pressure_rho_u_et(gs, W.v[0], velOf(W), W.v[4]);
    bool geo = false, gong = false;
    if (c.topo == 1) geo = gong = (c.bpresent[q] > 0.0);
    else if (c.topo == 2) geo = true;
    if (geo) {
        const double cth = c.cost[q], sth = c.sint[q];
        const D3 vc = cylOfCart(velOf(W), cth, sth);
        D3 sc;
        sc.x = 0.0;
        if (c.topo == 2) {
            const double gf = c.areaK0[q] * c.wedge;
            sc.y = (+W.v[0] * vc.z * vc.z + p) * gf;
            sc.z = -W.v[0] * vc.y * vc.z * gf;
            const D3 sCart = cartOfCyl(sc, cth, sth);
            R = R - s5(0.0, sCart.x, sCart.y, sCart.z, 0.0);
        } else {
            const double r = c.radius[q];
            sc.y = (+W.v[0] * vc.z * vc.z + p) / r;
            sc.z = -W.v[0] * vc.y * vc.z / r;
            const D3 sCart = cartOfCyl(sc, cth, sth);
            R = R - s5(0.0, sCart.x, sCart.y, sCart.z, 0.0) * vol;
        }
    }
    if (gong) {
        double om = c.rpm[q] * 2 * M_PI / 60;
        om *= speedScaling(c, t);
        R = R - gongSource(c, U, om, i, j, k, vol);
    }
    if (c.bfm) {
        const D3 gb = d3(c.gbx[q], c.gby[q], c.gbz[q]);
        if (mag(gb) > 1E-10) R = R - bfmTotalSource(c, gs, i, j, k, q, W, t);
    }
}

}  // namespace ctbfm
