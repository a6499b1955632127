// Per-face and per-node physics of the CTurboBFM explicit loop as device
// functions. Every expression keeps the reference's evaluation order (the
// translation unit is compiled with --fmad=false, and IEEE division and square
// root are the CUDA defaults for double), so that +, -, *, / and sqrt round
// exactly as the reference's do; pow, asin, atan2, exp and log10 are CUDA's.
#pragma once

#include "case.cuh"

namespace ctbfm {

struct D3 {
    double x, y, z;
};
struct S5 {
    double v[5];
};

#define CTBFM_DI __device__ __forceinline__

CTBFM_DI D3 d3(double x, double y, double z) { return D3{x, y, z}; }
CTBFM_DI D3 operator+(D3 a, D3 b) { return d3(a.x + b.x, a.y + b.y, a.z + b.z); }
CTBFM_DI D3 operator-(D3 a, D3 b) { return d3(a.x - b.x, a.y - b.y, a.z - b.z); }
CTBFM_DI D3 operator*(D3 a, double s) { return d3(a.x * s, a.y * s, a.z * s); }
CTBFM_DI D3 operator/(D3 a, double s) { return d3(a.x / s, a.y / s, a.z / s); }
CTBFM_DI D3 operator-(D3 a) { return d3(-a.x, -a.y, -a.z); }
CTBFM_DI double dot(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
CTBFM_DI double mag(D3 a) { return sqrt(a.x * a.x + a.y * a.y + a.z * a.z); }
CTBFM_DI D3 normalized(D3 a) {  // Vector3D::normalized (include/types.hpp:107-110)
    const double m = mag(a);
    return (m == 0) ? d3(0, 0, 0) : a / m;
}
CTBFM_DI D3 cross(D3 a, D3 b) {
    return d3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}

CTBFM_DI S5 s5(double a, double b, double c, double d, double e) { return S5{{a, b, c, d, e}}; }
CTBFM_DI S5 operator+(const S5& a, const S5& b) {
    S5 r;
#pragma unroll
    for (int i = 0; i < 5; i++) r.v[i] = a.v[i] + b.v[i];
    return r;
}
CTBFM_DI S5 operator-(const S5& a, const S5& b) {
    S5 r;
#pragma unroll
    for (int i = 0; i < 5; i++) r.v[i] = a.v[i] - b.v[i];
    return r;
}
CTBFM_DI S5 operator*(const S5& a, double s) {
    S5 r;
#pragma unroll
    for (int i = 0; i < 5; i++) r.v[i] = a.v[i] * s;
    return r;
}
CTBFM_DI S5 operator/(const S5& a, double s) {
    S5 r;
#pragma unroll
    for (int i = 0; i < 5; i++) r.v[i] = a.v[i] / s;
    return r;
}
CTBFM_DI S5 zero5() { return s5(0, 0, 0, 0, 0); }

CTBFM_DI double dmax(double a, double b) { return (a < b) ? b : a; }  // std::max
CTBFM_DI double dmin(double a, double b) { return (b < a) ? b : a; }  // std::min

CTBFM_DI S5 load5(double* const* U, long long q) {
    return s5(__ldg(U[0] + q), __ldg(U[1] + q), __ldg(U[2] + q), __ldg(U[3] + q), __ldg(U[4] + q));
}
CTBFM_DI void store5(double* const* U, long long q, const S5& s) {
#pragma unroll
    for (int c = 0; c < 5; c++) U[c][q] = s.v[c];
}

// ---------------------------------------------------------- ideal gas
// FluidIdeal (src/fluid_ideal.cpp).
struct Gas {
    double g, R;
};

CTBFM_DI double staticEnergy_u_et(D3 u, double et) {  // :74-77 (pow(|u|,2) == |u|*|u|)
    const double m = mag(u);
    const double m2 = m * m;
    return et - 0.5 * m2;
}
CTBFM_DI double pressure_rho_e(Gas gs, double rho, double e) { return (gs.g - 1) * rho * e; }  // :14-16
CTBFM_DI double pressure_rho_u_et(Gas gs, double rho, D3 u, double et) {                     // :89-92
    return pressure_rho_e(gs, rho, staticEnergy_u_et(u, et));
}
CTBFM_DI double soundSpeed_p_rho(Gas gs, double p, double rho) { return sqrt(gs.g * p / rho); }  // :70-72
CTBFM_DI double soundSpeed_rho_u_et(Gas gs, double rho, D3 u, double et) {                      // :83-87
    const double p = pressure_rho_e(gs, rho, staticEnergy_u_et(u, et));
    return soundSpeed_p_rho(gs, p, rho);
}
CTBFM_DI double soundSpeed_rho_e(Gas gs, double e) { return sqrt(gs.g * (gs.g - 1.0) * e); }  // :22-24
CTBFM_DI double totalEnthalpy_rho_u_et(Gas gs, double rho, D3 u, double et) {                 // :114-118
    const double p = pressure_rho_e(gs, rho, staticEnergy_u_et(u, et));
    return et + p / rho;
}
CTBFM_DI double temperature_rho_u_et(Gas gs, double rho, D3 u, double et) {  // :109-112
    return pressure_rho_u_et(gs, rho, u, et) / (rho * gs.R);
}
CTBFM_DI double staticEnergy_p_rho(Gas gs, double p, double rho) { return p / ((gs.g - 1) * rho); }  // :10-12
CTBFM_DI double mach_rho_u_et(Gas gs, double rho, D3 u, double et) {                                // :137-141
    const double a = soundSpeed_rho_u_et(gs, rho, u, et);
    return mag(u) / a;
}
CTBFM_DI double totalPressure_rho_u_et(Gas gs, double rho, D3 u, double et) {  // :94-98
    const double p = pressure_rho_u_et(gs, rho, u, et);
    const double M = mach_rho_u_et(gs, rho, u, et);
    return p * pow(1.0 + (gs.g - 1.0) / 2.0 * M * M, gs.g / (gs.g - 1));
}
CTBFM_DI double totalTemperature_rho_u_et(Gas gs, double rho, D3 u, double et) {  // :100-104
    const double T = temperature_rho_u_et(gs, rho, u, et);
    const double M = mach_rho_u_et(gs, rho, u, et);
    return T * (1.0 + (gs.g - 1.0) / 2.0 * M * M);
}

// getPrimitiveVariablesFromConservative (src/math_utils.cpp:49-57).
CTBFM_DI S5 primOf(const S5& U) {
    return s5(U.v[0], U.v[1] / U.v[0], U.v[2] / U.v[0], U.v[3] / U.v[0], U.v[4] / U.v[0]);
}
CTBFM_DI D3 velOf(const S5& W) { return d3(W.v[1], W.v[2], W.v[3]); }

// computeAdvectionFluxFromPrimitive (src/math_utils.cpp:71-86) with the unit
// normal n = S/|S| precomputed on the host with the same division.
CTBFM_DI S5 advFlux(Gas gs, const S5& W, D3 n) {
    const D3 u = velOf(W);
    const double un = dot(u, n);
    const double p = pressure_rho_u_et(gs, W.v[0], u, W.v[4]);
    const double ht = totalEnthalpy_rho_u_et(gs, W.v[0], u, W.v[4]);
    return s5(W.v[0] * un, W.v[0] * un * u.x + p * n.x, W.v[0] * un * u.y + p * n.y,
              W.v[0] * un * u.z + p * n.z, W.v[0] * un * ht);
}

// Rotations about the x axis (src/math_utils.cpp:109-138) with host-computed
// cos/sin.
CTBFM_DI S5 rotState(const S5& a, double c, double s) {
    return s5(a.v[0], a.v[1], a.v[2] * c - a.v[3] * s, a.v[2] * s + a.v[3] * c, a.v[4]);
}
CTBFM_DI D3 cylOfCart(D3 v, double c, double s) { return d3(v.x, v.y * c + v.z * s, -v.y * s + v.z * c); }
CTBFM_DI D3 cartOfCyl(D3 v, double c, double s) { return d3(v.x, v.y * c - v.z * s, v.y * s + v.z * c); }

// ------------------------------------------------------------ JST flux
// AdvectionJst::computeFlux (src/advection_jst.cpp:4-57); kappa2 = 0.5,
// kappa4 = 0.02, c4 = 2 (include/advection_jst.hpp:23).
CTBFM_DI double jstR(Gas gs, const S5& W) {
    const D3 u = velOf(W);
    return mag(u) + soundSpeed_rho_u_et(gs, W.v[0], u, W.v[4]);
}
CTBFM_DI double pressurePrim(Gas gs, const S5& W) { return pressure_rho_u_et(gs, W.v[0], velOf(W), W.v[4]); }
CTBFM_DI double jstS(double p1, double p2, double p3) { return fabs((p1 - 2 * p2 + p3) / (p1 + 2 * p2 + p3)); }

CTBFM_DI S5 fluxJstW(Gas gs, const S5& Ull, const S5& Ul, const S5& Ur, const S5& Urr, const S5& Wll,
                     const S5& Wl, const S5& Wr, const S5& Wrr, D3 n) {
    const S5 Wavg = (Wl + Wr) * 0.5;
    const double rL = jstR(gs, Wl), rR = jstR(gs, Wr);
    const double pll = pressurePrim(gs, Wll), pl = pressurePrim(gs, Wl), pr = pressurePrim(gs, Wr),
                 prr = pressurePrim(gs, Wrr);
    const double sL = jstS(pll, pl, pr), sR = jstS(pl, pr, prr);
    const double r = dmax(rL, rR);
    const double sf = dmax(sL, sR);
    const double psi2 = 0.5 * sf * r;
    const double psi4 = dmax(0.0, 0.02 * r - 2.0 * psi2);
    const S5 F = advFlux(gs, Wavg, n);
    const S5 d = (Ur - Ul) * psi2 - (((Urr - Ur) - (Ur - Ul) * 2) + (Ul - Ull)) * psi4;
    return F - d;
}

CTBFM_DI S5 fluxJst(Gas gs, const S5& Ull, const S5& Ul, const S5& Ur, const S5& Urr, D3 n) {
    return fluxJstW(gs, Ull, Ul, Ur, Urr, primOf(Ull), primOf(Ul), primOf(Ur), primOf(Urr), n);
}

// ------------------------------------------------------ Roe + MUSCL flux
// AdvectionBase::computeReconstructionSmoothness / computeLimiter
// (src/advection_base.cpp:28-64).
CTBFM_DI double smooth1(double l, double c, double r) {
    const double dR = r - c;
    const double dL = c - l;
    return (fabs(dR) < 1E-12) ? 0.0 : dL / dR;
}
CTBFM_DI double limiter1(int lim, double x) {
    switch (lim) {
        case 1: return (x <= 0.0) ? 0.0 : (x * x + x) / (1.0 + x * x);  // van Albada
        case 2: return (x + fabs(x)) / (1.0 + fabs(x));                 // van Leer
        case 3: return dmax(0.0, dmin(1.0, x));                         // minmod
        default: return 0.0;
    }
}
CTBFM_DI double roeAvg(double sl, double sr, double pl, double pr) {  // roeAverage with sl = sqrt(rhoL)
    return (sl * pl + sr * pr) / (sl + sr);
}

// AdvectionRoe::computeFlux (src/advection_roe.cpp:6-220), entropy fix 0.01
// (include/advection_roe.hpp:63).
CTBFM_DI S5 fluxRoeW(Gas gs, int muscl, int lim, const S5& Wll, S5 Wl, S5 Wr, const S5& Wrr, D3 n1) {
    if (muscl) {
        S5 limL, limR;
#pragma unroll
        for (int i = 0; i < 5; i++) {
            limL.v[i] = limiter1(lim, smooth1(Wll.v[i], Wl.v[i], Wr.v[i]));
            limR.v[i] = limiter1(lim, smooth1(Wl.v[i], Wr.v[i], Wrr.v[i]));
        }
#pragma unroll
        for (int i = 0; i < 5; i++) Wl.v[i] += limL.v[i] * (Wr.v[i] - Wl.v[i]) * 0.5;
#pragma unroll
        for (int i = 0; i < 5; i++) Wr.v[i] -= limR.v[i] * (Wrr.v[i] - Wr.v[i]) * 0.5;
    }
    // normal triad (:41-58); n1 = S.normalized() equals the stored unit normal
    D3 n2 = (n1.x == 0 && n1.y == 0) ? d3(1, 0, 0) : d3(-n1.y, n1.x, 0);
    n2 = normalized(n2);
    const D3 n3 = cross(n1, n2);
    const D3 uL = velOf(Wl), uR = velOf(Wr);
    const double rhoL = Wl.v[0], rhoR = Wr.v[0];
    const double u1L = dot(uL, n1), u2L = dot(uL, n2), u3L = dot(uL, n3);
    const double u1R = dot(uR, n1), u2R = dot(uR, n2), u3R = dot(uR, n3);
    const double etL = Wl.v[4], etR = Wr.v[4];
    // Roe averages (:68-143)
    const double htL = totalEnthalpy_rho_u_et(gs, rhoL, d3(u1L, u2L, u3L), etL);
    const double htR = totalEnthalpy_rho_u_et(gs, rhoR, d3(u1R, u2R, u3R), etR);
    const double rhoA = sqrt(rhoL * rhoR);
    const double sl = sqrt(rhoL), sr = sqrt(rhoR);
    const double u1A = roeAvg(sl, sr, u1L, u1R);
    const double u2A = roeAvg(sl, sr, u2L, u2R);
    const double u3A = roeAvg(sl, sr, u3L, u3R);
    const double htA = roeAvg(sl, sr, htL, htR);
    const double eL = etL - 0.5 * (u1L * u1L + u2L * u2L + u3L * u3L);
    const double eR = etR - 0.5 * (u1R * u1R + u2R * u2R + u3R * u3R);
    const double pL = pressure_rho_e(gs, rhoL, eL);
    const double pR = pressure_rho_e(gs, rhoR, eR);
    const double chiL = (gs.g - 1.0) * eL, kapL = (gs.g - 1.0) * rhoL;
    const double chiR = (gs.g - 1.0) * eR, kapR = (gs.g - 1.0) * rhoR;
    const double barChi = 0.5 * (chiL + chiR);
    const double barKap = 0.5 * (kapL + kapR);
    const double barRho = 0.5 * (rhoL + rhoR);
    const double barE = 0.5 * (eL + eR);
    const double dP = pR - pL, dRho = rhoR - rhoL, dE = eR - eL;
    const double dRhoHat = (barRho > 1e-12) ? dRho / barRho : 0.0;
    const double dEHat = (fabs(barE) > 1e-12) ? dE / fabs(barE) : 0.0;
    const double dNorm2 = dRhoHat * dRhoHat + dEHat * dEHat;
    double chiT = barChi, kapT = barKap;
    if (dNorm2 > 1e-12) {
        const double res = dP - (barChi * dRho + barKap * dE);
        chiT += (res * dRhoHat) / (dNorm2 * barRho);
        kapT += (res * dEHat) / (dNorm2 * fabs(barE));
    }
    if (barKap > 0.0 && kapT <= 0.0) kapT = 0.01 * barKap;
    const double kapP = (rhoA > 1e-12) ? kapT / rhoA : 0.4;
    const double eA = roeAvg(sl, sr, eL, eR);
    const double chiP = chiT - kapP * eA;
    const double q2 = u1A * u1A + u2A * u2A + u3A * u3A;
    const double hA = htA - 0.5 * q2;
    double a2 = chiP + kapP * hA;
    if (a2 <= 0.0) {
        const double aL = soundSpeed_rho_e(gs, eL), aR = soundSpeed_rho_e(gs, eR);
        a2 = 0.5 * (aL * aL + aR * aR);
    }
    const double aA = sqrt(a2);
    // eigenvalues, eigenvectors, wave strengths (:146-185)
    const double lam[5] = {u1A - aA, u1A, u1A, u1A, u1A + aA};
    const double cE5 = htA - (aA * aA) / kapP;
    const double ev[5][5] = {{1.0, u1A - aA, u2A, u3A, htA - aA * u1A},
                             {1.0, u1A, u2A, u3A, cE5},
                             {0.0, 0.0, 1.0, 0.0, u2A},
                             {0.0, 0.0, 0.0, 1.0, u3A},
                             {1.0, u1A + aA, u2A, u3A, htA + aA * u1A}};
    const double ddRho = rhoR - rhoL;
    const double du1 = u1R - u1L, du2 = u2R - u2L, du3 = u3R - u3L;
    const double ppL = pressure_rho_u_et(gs, rhoL, d3(u1L, u2L, u3L), etL);
    const double ppR = pressure_rho_u_et(gs, rhoR, d3(u1R, u2R, u3R), etR);
    const double ddP = ppR - ppL;
    double ws[5];
    ws[0] = 1.0 / (2.0 * aA * aA) * (ddP - rhoA * aA * du1);
    ws[1] = ddRho - ddP / (aA * aA);
    ws[2] = rhoA * du2;
    ws[3] = rhoA * du3;
    ws[4] = 1.0 / (2.0 * aA * aA) * (ddP + rhoA * aA * du1);
    // assembly (:188-220)
    const D3 e1 = d3(1.0, 0.0, 0.0);
    const S5 FL = advFlux(gs, s5(rhoL, u1L, u2L, u3L, etL), e1);
    const S5 FR = advFlux(gs, s5(rhoR, u1R, u2R, u3R, etR), e1);
    double fix[5];
#pragma unroll
    for (int i = 0; i < 5; i++) fix[i] = (fabs(lam[i]) < 0.01) ? 0.01 : fabs(lam[i]);
    S5 Fr = (FL + FR) * 0.5;
#pragma unroll
    for (int i = 0; i < 5; i++)
#pragma unroll
        for (int j = 0; j < 5; j++) Fr.v[i] -= 0.5 * ws[j] * fix[j] * ev[j][i];
    const D3 ex = d3(1.0, 0.0, 0.0), ey = d3(0.0, 1.0, 0.0), ez = d3(0.0, 0.0, 1.0);
    return s5(Fr.v[0],
              Fr.v[1] * (dot(n1, ex)) + Fr.v[2] * (dot(n2, ex)) + Fr.v[3] * (dot(n3, ex)),
              Fr.v[1] * (dot(n1, ey)) + Fr.v[2] * (dot(n2, ey)) + Fr.v[3] * (dot(n3, ey)),
              Fr.v[1] * (dot(n1, ez)) + Fr.v[2] * (dot(n2, ez)) + Fr.v[3] * (dot(n3, ez)),
              Fr.v[4]);
}

CTBFM_DI S5 fluxRoe(Gas gs, int muscl, int lim, const S5& Ull, const S5& Ul, const S5& Ur, const S5& Urr, D3 n1) {
    return fluxRoeW(gs, muscl, lim, muscl ? primOf(Ull) : zero5(), primOf(Ul), primOf(Ur),
                    muscl ? primOf(Urr) : zero5(), n1);
}

// ----------------------------------------------------------- boundaries

// Config::computeRampedOutletPressure (src/config.cpp:430-439).
CTBFM_DI double rampedOutletPressure(const DevCase& c, long long it, double p) {
    const double ratio = static_cast<double>(it) / c.ramp_iters;
    if (ratio >= 1.0) return p;
    return c.init_p + (p - c.init_p) * ratio;
}

// BoundaryBase::computeOutletFlux (src/boundary_base.cpp:181-224).
CTBFM_DI S5 bcOutlet(const DevCase& c, Gas gs, const S5& Uint, D3 n, double pOut, long long it) {
    const S5 W = primOf(Uint);
    const D3 u = velOf(W);
    const double rho = W.v[0];
    const double p = pressure_rho_u_et(gs, rho, u, W.v[4]);
    const double a = soundSpeed_p_rho(gs, p, W.v[0]);
    if (mag(u) >= a) return advFlux(gs, W, n);
    const double pb = rampedOutletPressure(c, it, pOut);
    const double rhob = pb * rho / p;
    const double eb = staticEnergy_p_rho(gs, pb, rhob);
    const double etb = eb + 0.5 * dot(u, u);
    return advFlux(gs, s5(rhob, u.x, u.y, u.z, etb), n);
}

// BoundaryInviscidWall::computeBoundaryFlux (src/boundary_inviscid_wall.cpp:5-30).
CTBFM_DI S5 bcWall(Gas gs, const S5& Uint, D3 n) {
    const S5 W = primOf(Uint);
    const D3 u = velOf(W);
    const double p = pressure_rho_u_et(gs, W.v[0], u, W.v[4]);
    const double un = dot(u, n);
    const double a = soundSpeed_p_rho(gs, p, W.v[0]);
    double pw = p + W.v[0] * un * a;
    if (pw < 0.01 * p) pw = 0.01 * p;
    return s5(0.0, pw * n.x, pw * n.y, pw * n.z, 0.0);
}

// BoundaryInlet::computeBoundaryFlux (src/boundary_inlet.cpp:4-43) and
// BoundaryBase::computeSubsonicInletFlux (src/boundary_base.cpp:7-124);
// cth/sth are cos/sin of the node's theta for the cylindrical frame.
CTBFM_DI S5 bcInlet(const DevCase& c, Gas gs, const DevPatch& pt, const S5& Uint, D3 n, double cth, double sth) {
    const double Pt = pt.v[0], Tt = pt.v[1];
    D3 dir = d3(pt.v[2], pt.v[3], pt.v[4]);
    if (c.inlet_cyl) dir = cartOfCyl(dir, cth, sth);
    if (dir.x == 1.0 && dir.y == 1.0 && dir.z == 1.0) dir = -n;  // -S / |S|
    else dir = dir / mag(dir);
    const S5 W = primOf(Uint);
    const D3 u = velOf(W);
    const double aInt = soundSpeed_rho_u_et(gs, W.v[0], u, W.v[4]);
    const double unInt = dot(u, n);
    const double Z = W.v[0] * aInt;
    const double pInt = pressure_rho_u_et(gs, W.v[0], u, W.v[4]);
    double Cg = dot(dir, n);
    if (Cg >= 0.0) Cg = -1.0;
    const double Rout = pInt + Z * unInt;
    const double g = gs.g, Rg = gs.R;
    const double cp = g * Rg / (g - 1.0);
    const double htIn = cp * Tt;
    double pLow = 0.05 * Pt, pHigh = 0.999999 * Pt;
    double pB = 0.5 * (pLow + pHigh);
    const double ex = (g - 1.0) / g;
    for (int iter = 0; iter < 30; ++iter) {
        const double pMid = 0.5 * (pLow + pHigh);
        const double TMid = Tt * pow(pMid / Pt, ex);
        const double hMid = cp * TMid;
        const double VMid = sqrt(2.0 * dmax(0.0, htIn - hMid));
        const double res = pMid + Z * Cg * VMid - Rout;
        if (fabs(res) < 1e-4 * Pt) {
            pB = pMid;
            break;
        }
        if (res < 0.0) pLow = pMid;
        else pHigh = pMid;
        pB = pMid;
    }
    const double TB = Tt * pow(pB / Pt, ex);
    const double hB = cp * TB;
    const double VB = sqrt(2.0 * dmax(0.0, htIn - hB));
    const D3 uB = dir * VB;
    const double rhoB = pB / (Rg * TB);
    const double eB = staticEnergy_p_rho(gs, pB, rhoB);
    const double etB = eB + 0.5 * dot(uB, uB);
    return advFlux(gs, s5(rhoB, uB.x, uB.y, uB.z, etB), n);
}

}  // namespace ctbfm
