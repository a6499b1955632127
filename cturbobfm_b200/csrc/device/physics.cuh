// Per-face physics of the CTurboBFM explicit loop as device functions,
// templated on the working precision R. Every expression keeps the reference's
// evaluation order; the double instantiation is compiled with --fmad=false
// (and IEEE division and square root are the CUDA defaults), so that +, -, *,
// / and sqrt round exactly as the reference's do, while pow, asin, atan2, exp
// and log10 are CUDA's. Literals are written as R(...) so that the float
// instantiation stays in float.
#pragma once

#include "case.cuh"

namespace ctbfm {

#define CTBFM_DI __device__ __forceinline__

template <typename R>
struct V3 {
    R x, y, z;
};
template <typename R>
struct S5 {
    R v[5];
};

template <typename R>
CTBFM_DI V3<R> v3(R x, R y, R z) {
    return V3<R>{x, y, z};
}
template <typename R>
CTBFM_DI V3<R> operator+(V3<R> a, V3<R> b) {
    return v3(a.x + b.x, a.y + b.y, a.z + b.z);
}
template <typename R>
CTBFM_DI V3<R> operator-(V3<R> a, V3<R> b) {
    return v3(a.x - b.x, a.y - b.y, a.z - b.z);
}
template <typename R>
CTBFM_DI V3<R> operator*(V3<R> a, R s) {
    return v3(a.x * s, a.y * s, a.z * s);
}
template <typename R>
CTBFM_DI V3<R> operator/(V3<R> a, R s) {
    return v3(a.x / s, a.y / s, a.z / s);
}
template <typename R>
CTBFM_DI V3<R> operator-(V3<R> a) {
    return v3(-a.x, -a.y, -a.z);
}
template <typename R>
CTBFM_DI R dot(V3<R> a, V3<R> b) {
    return a.x * b.x + a.y * b.y + a.z * b.z;
}
template <typename R>
CTBFM_DI R mag(V3<R> a) {
    return sqrt(a.x * a.x + a.y * a.y + a.z * a.z);
}
template <typename R>
CTBFM_DI V3<R> normalized(V3<R> a) {  // Vector3D::normalized (include/types.hpp:107-110)
    const R m = mag(a);
    return (m == R(0)) ? v3(R(0), R(0), R(0)) : a / m;
}
template <typename R>
CTBFM_DI V3<R> cross(V3<R> a, V3<R> b) {
    return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}

template <typename R>
CTBFM_DI S5<R> s5(R a, R b, R c, R d, R e) {
    return S5<R>{{a, b, c, d, e}};
}
template <typename R>
CTBFM_DI S5<R> operator+(const S5<R>& a, const S5<R>& b) {
    S5<R> r;
#pragma unroll
    for (int i = 0; i < 5; i++) r.v[i] = a.v[i] + b.v[i];
    return r;
}
template <typename R>
CTBFM_DI S5<R> operator-(const S5<R>& a, const S5<R>& b) {
    S5<R> r;
#pragma unroll
    for (int i = 0; i < 5; i++) r.v[i] = a.v[i] - b.v[i];
    return r;
}
template <typename R>
CTBFM_DI S5<R> operator*(const S5<R>& a, R s) {
    S5<R> r;
#pragma unroll
    for (int i = 0; i < 5; i++) r.v[i] = a.v[i] * s;
    return r;
}
template <typename R>
CTBFM_DI S5<R> operator/(const S5<R>& a, R s) {
    S5<R> r;
#pragma unroll
    for (int i = 0; i < 5; i++) r.v[i] = a.v[i] / s;
    return r;
}
template <typename R>
CTBFM_DI S5<R> zero5() {
    return s5(R(0), R(0), R(0), R(0), R(0));
}

template <typename R>
CTBFM_DI R rmax(R a, R b) {  // std::max
    return (a < b) ? b : a;
}
template <typename R>
CTBFM_DI R rmin(R a, R b) {  // std::min
    return (b < a) ? b : a;
}

// Loads of arrays the loop rewrites (states, primitives): through the
// read-only data path in kernels that never see them change while they run;
// plain coherent loads in the persistent kernel, whose later phases read
// what its earlier phases wrote (CTBFM_COHERENT_LOADS).
#ifdef CTBFM_COHERENT_LOADS
#define CTBFM_LDS(p) (*(p))
#else
#define CTBFM_LDS(p) __ldg(p)
#endif

template <typename R>
CTBFM_DI S5<R> load5(R* const* U, long long q) {
    return s5(CTBFM_LDS(U[0] + q), CTBFM_LDS(U[1] + q), CTBFM_LDS(U[2] + q), CTBFM_LDS(U[3] + q),
              CTBFM_LDS(U[4] + q));
}
template <typename R>
CTBFM_DI void store5(R* const* U, long long q, const S5<R>& s) {
#pragma unroll
    for (int c = 0; c < 5; c++) U[c][q] = s.v[c];
}

// ------------------------------------------------------------- fluids
// Gas: the ideal gas of FluidIdeal (src/fluid_ideal.cpp) when lut is null,
// otherwise the look-up tables of FluidReal (src/fluid_real.cpp) with the
// FluidBase defaults it inherits (include/fluid_base.hpp). Each function
// below takes the ideal branch exactly as before for the ideal gas.
template <typename R>
struct Gas {
    R g, R_;
    const DevLut* lut;
};

// Table2D::interpolate (include/fluid_real.hpp:35-57): clamp, cell index by
// truncation (a NaN coordinate gives a NaN result on both sides), bilinear
// weights summed in the reference's order. Double: the double tables; float:
// the float copy, in float.
CTBFM_DI double lutInterp(const DevTable& t, double x, double y) {
    const double xc = (x < t.xmin) ? t.xmin : ((t.xmax < x) ? t.xmax : x);
    const double yc = (y < t.ymin) ? t.ymin : ((t.ymax < y) ? t.ymax : y);
    const double rx = (xc - t.xmin) / t.dx;
    const double ry = (yc - t.ymin) / t.dy;
    unsigned long long i = static_cast<unsigned long long>(rx);
    unsigned long long j = static_cast<unsigned long long>(ry);
    if (i >= static_cast<unsigned long long>(t.nx - 1)) i = (t.nx >= 2) ? t.nx - 2 : 0;
    if (j >= static_cast<unsigned long long>(t.ny - 1)) j = (t.ny >= 2) ? t.ny - 2 : 0;
    const double wx = rx - static_cast<double>(i);
    const double wy = ry - static_cast<double>(j);
    const double* d = t.d + i * t.ny + j;
    const double f00 = __ldg(d), f01 = __ldg(d + 1), f10 = __ldg(d + t.ny), f11 = __ldg(d + t.ny + 1);
    return (1.0 - wx) * (1.0 - wy) * f00 + wx * (1.0 - wy) * f10 + (1.0 - wx) * wy * f01 + wx * wy * f11;
}
CTBFM_DI float lutInterp(const DevTable& t, float x, float y) {
    const float xc = (x < t.fxmin) ? t.fxmin : ((t.fxmax < x) ? t.fxmax : x);
    const float yc = (y < t.fymin) ? t.fymin : ((t.fymax < y) ? t.fymax : y);
    const float rx = (xc - t.fxmin) / t.fdx;
    const float ry = (yc - t.fymin) / t.fdy;
    unsigned int i = static_cast<unsigned int>(rx);
    unsigned int j = static_cast<unsigned int>(ry);
    if (i >= static_cast<unsigned int>(t.nx - 1)) i = (t.nx >= 2) ? t.nx - 2 : 0;
    if (j >= static_cast<unsigned int>(t.ny - 1)) j = (t.ny >= 2) ? t.ny - 2 : 0;
    const float wx = rx - static_cast<float>(i);
    const float wy = ry - static_cast<float>(j);
    const float* d = t.f + i * t.ny + j;
    const float f00 = __ldg(d), f01 = __ldg(d + 1), f10 = __ldg(d + t.ny), f11 = __ldg(d + t.ny + 1);
    return (1.0f - wx) * (1.0f - wy) * f00 + wx * (1.0f - wy) * f10 + (1.0f - wx) * wy * f01 + wx * wy * f11;
}

// FluidReal::computeStaticEnergy_p_rho (src/fluid_real.cpp:227-250): bisection
// on e, always in double (the table inversion).
CTBFM_DI double lutStaticEnergy_p_rho(const DevLut& L, double p, double rho) {
    const DevTable& tp = L.re[kReP];
    double eLo = tp.ymin, eHi = tp.ymax;
    const double pLo = lutInterp(tp, rho, eLo);
    const double pHi = lutInterp(tp, rho, eHi);
    if (p <= pLo) return eLo;
    if (p >= pHi) return eHi;
    for (int it = 0; it < 30; ++it) {
        const double eMid = 0.5 * (eLo + eHi);
        const double pMid = lutInterp(tp, rho, eMid);
        if (fabs(pMid - p) <= 1e-4 * p) return eMid;
        if (pMid < p) eLo = eMid;
        else eHi = eMid;
    }
    return 0.5 * (eLo + eHi);
}
// FluidBase::computeEnthalpy_p_s (include/fluid_base.hpp:73-75) on the (p, s) tables.
template <typename R>
CTBFM_DI R lutEnthalpy_p_s(const DevLut& L, R p, R s) {
    return lutInterp(L.ps[kPsE], p, s) + p / lutInterp(L.ps[kPsRho], p, s);
}
// FluidReal::computeTotalPressure_rho_u_et (src/fluid_real.cpp:299-321) given
// the static energy: 25 bisection steps on the (p, s) tables, in double.
CTBFM_DI double lutTotalPressure(const DevLut& L, double rho, double e, double et) {
    const double p = lutInterp(L.re[kReP], rho, e);
    const double s = lutInterp(L.re[kReS], rho, e);
    const double ht = et + p / rho;
    double pLo = p, pHi = L.ps[kPsRho].xmax;
    for (int it = 0; it < 25; ++it) {
        const double pMid = 0.5 * (pLo + pHi);
        const double rhoMid = lutInterp(L.ps[kPsRho], pMid, s);
        const double eMid = lutInterp(L.ps[kPsE], pMid, s);
        const double hMid = eMid + pMid / rhoMid;
        if (hMid < ht) pLo = pMid;
        else pHi = pMid;
    }
    return 0.5 * (pLo + pHi);
}

template <typename R>
CTBFM_DI R staticEnergy_u_et(V3<R> u, R et) {  // FluidIdeal :74-77 (pow(|u|,2) == |u|*|u|)
    const R m = mag(u);
    const R m2 = m * m;
    return et - R(0.5) * m2;
}
template <typename R>
CTBFM_DI R staticEnergy_u_et(Gas<R> gs, V3<R> u, R et) {
    if (gs.lut) return et - R(0.5) * dot(u, u);  // FluidBase (include/fluid_base.hpp:78-80)
    return staticEnergy_u_et(u, et);
}
template <typename R>
CTBFM_DI R pressure_rho_e(Gas<R> gs, R rho, R e) {  // :14-16; FluidReal :211-213
    if (gs.lut) return lutInterp(gs.lut->re[kReP], rho, e);
    return (gs.g - R(1)) * rho * e;
}
template <typename R>
CTBFM_DI R pressure_rho_u_et(Gas<R> gs, R rho, V3<R> u, R et) {  // :89-92; fluid_base.hpp:91-94
    return pressure_rho_e(gs, rho, staticEnergy_u_et(gs, u, et));
}
template <typename R>
CTBFM_DI R soundSpeed_p_rho(Gas<R> gs, R p, R rho) {  // :70-72; FluidReal :252-255 (inversion in double)
    if (gs.lut) {
        const double e = lutStaticEnergy_p_rho(*gs.lut, static_cast<double>(p), static_cast<double>(rho));
        return R(lutInterp(gs.lut->re[kReA], static_cast<double>(rho), e));
    }
    return sqrt(gs.g * p / rho);
}
template <typename R>
CTBFM_DI R soundSpeed_rho_u_et(Gas<R> gs, R rho, V3<R> u, R et) {  // :83-87; fluid_base.hpp:86-89
    if (gs.lut) return lutInterp(gs.lut->re[kReA], rho, staticEnergy_u_et(gs, u, et));
    const R p = pressure_rho_e(gs, rho, staticEnergy_u_et(u, et));
    return soundSpeed_p_rho(gs, p, rho);
}
template <typename R>
CTBFM_DI R soundSpeed_rho_e(Gas<R> gs, R rho, R e) {  // :22-24; FluidReal :219-221
    if (gs.lut) return lutInterp(gs.lut->re[kReA], rho, e);
    return sqrt(gs.g * (gs.g - R(1)) * e);
}
template <typename R>
CTBFM_DI R dpdrho_e(Gas<R> gs, R rho, R e) {  // :50-52; FluidReal :410-412
    if (gs.lut) return lutInterp(gs.lut->re[kReDpDrho], rho, e);
    return (gs.g - R(1)) * e;
}
template <typename R>
CTBFM_DI R dpde_rho(Gas<R> gs, R rho, R e) {  // :54-56; FluidReal :414-416
    if (gs.lut) return lutInterp(gs.lut->re[kReDpDe], rho, e);
    return (gs.g - R(1)) * rho;
}
template <typename R>
CTBFM_DI R totalEnthalpy_rho_u_et(Gas<R> gs, R rho, V3<R> u, R et) {  // :114-118; fluid_base.hpp:106-109
    const R p = pressure_rho_e(gs, rho, staticEnergy_u_et(gs, u, et));
    return et + p / rho;
}
template <typename R>
CTBFM_DI R temperature_rho_u_et(Gas<R> gs, R rho, V3<R> u, R et) {  // :109-112; fluid_base.hpp:96-99
    if (gs.lut) return lutInterp(gs.lut->re[kReT], rho, staticEnergy_u_et(gs, u, et));
    return pressure_rho_u_et(gs, rho, u, et) / (rho * gs.R_);
}
template <typename R>
CTBFM_DI R entropy_rho_u_et(Gas<R> gs, R rho, V3<R> u, R et) {  // real gas only: fluid_base.hpp:101-104
    return lutInterp(gs.lut->re[kReS], rho, staticEnergy_u_et(gs, u, et));
}
template <typename R>
CTBFM_DI R staticEnergy_p_rho(Gas<R> gs, R p, R rho) {  // :10-12; FluidReal :227-250 (double)
    if (gs.lut) return R(lutStaticEnergy_p_rho(*gs.lut, static_cast<double>(p), static_cast<double>(rho)));
    return p / ((gs.g - R(1)) * rho);
}
template <typename R>
CTBFM_DI R mach_rho_u_et(Gas<R> gs, R rho, V3<R> u, R et) {  // :137-141
    const R a = soundSpeed_rho_u_et(gs, rho, u, et);
    return mag(u) / a;
}
template <typename R>
CTBFM_DI R totalPressure_rho_u_et(Gas<R> gs, R rho, V3<R> u, R et) {  // :94-98; FluidReal :299-321
    if (gs.lut) return R(lutTotalPressure(*gs.lut, rho, staticEnergy_u_et(gs, u, et), et));
    const R p = pressure_rho_u_et(gs, rho, u, et);
    const R M = mach_rho_u_et(gs, rho, u, et);
    return p * pow(R(1) + (gs.g - R(1)) / R(2) * M * M, gs.g / (gs.g - R(1)));
}
template <typename R>
CTBFM_DI R totalTemperature_rho_u_et(Gas<R> gs, R rho, V3<R> u, R et) {  // :100-104; FluidReal :323-328
    if (gs.lut) {
        const double pt = lutTotalPressure(*gs.lut, rho, staticEnergy_u_et(gs, u, et), et);
        const double e = staticEnergy_u_et(gs, u, et);
        const double s = lutInterp(gs.lut->re[kReS], static_cast<double>(rho), e);
        return R(lutInterp(gs.lut->ps[kPsT], pt, s));
    }
    const R T = temperature_rho_u_et(gs, rho, u, et);
    const R M = mach_rho_u_et(gs, rho, u, et);
    return T * (R(1) + (gs.g - R(1)) / R(2) * M * M);
}

// getPrimitiveVariablesFromConservative (src/math_utils.cpp:49-57).
template <typename R>
CTBFM_DI S5<R> primOf(const S5<R>& U) {
    return s5(U.v[0], U.v[1] / U.v[0], U.v[2] / U.v[0], U.v[3] / U.v[0], U.v[4] / U.v[0]);
}
template <typename R>
CTBFM_DI V3<R> velOf(const S5<R>& W) {
    return v3(W.v[1], W.v[2], W.v[3]);
}

// computeAdvectionFluxFromPrimitive (src/math_utils.cpp:71-86) with the unit
// normal n = S/|S| precomputed on the host with the same division.
template <typename R>
CTBFM_DI S5<R> advFlux(Gas<R> gs, const S5<R>& W, V3<R> n) {
    const V3<R> u = velOf(W);
    const R un = dot(u, n);
    const R p = pressure_rho_u_et(gs, W.v[0], u, W.v[4]);
    const R ht = totalEnthalpy_rho_u_et(gs, W.v[0], u, W.v[4]);
    return s5(W.v[0] * un, W.v[0] * un * u.x + p * n.x, W.v[0] * un * u.y + p * n.y, W.v[0] * un * u.z + p * n.z,
              W.v[0] * un * ht);
}

// Rotations about the x axis (src/math_utils.cpp:109-138) with host-computed
// cos/sin.
template <typename R>
CTBFM_DI S5<R> rotState(const S5<R>& a, R c, R s) {
    return s5(a.v[0], a.v[1], a.v[2] * c - a.v[3] * s, a.v[2] * s + a.v[3] * c, a.v[4]);
}
template <typename R>
CTBFM_DI V3<R> cylOfCart(V3<R> v, R c, R s) {
    return v3(v.x, v.y * c + v.z * s, -v.y * s + v.z * c);
}
template <typename R>
CTBFM_DI V3<R> cartOfCyl(V3<R> v, R c, R s) {
    return v3(v.x, v.y * c - v.z * s, v.y * s + v.z * c);
}

// ------------------------------------------------------------ JST flux
// AdvectionJst::computeFlux (src/advection_jst.cpp:4-57); kappa2 = 0.5,
// kappa4 = 0.02, c4 = 2 (include/advection_jst.hpp:23).
template <typename R>
CTBFM_DI R jstR(Gas<R> gs, const S5<R>& W) {
    const V3<R> u = velOf(W);
    return mag(u) + soundSpeed_rho_u_et(gs, W.v[0], u, W.v[4]);
}
template <typename R>
CTBFM_DI R pressurePrim(Gas<R> gs, const S5<R>& W) {
    return pressure_rho_u_et(gs, W.v[0], velOf(W), W.v[4]);
}
template <typename R>
CTBFM_DI R jstS(R p1, R p2, R p3) {
    return fabs((p1 - R(2) * p2 + p3) / (p1 + R(2) * p2 + p3));
}

// The JST flux given the nodes' pressures p and spectral radii r = |u| + a,
// which depend on one node each: the fused stage kernel evaluates them once
// per node, the face kernels once per face (the same values either way).
template <typename R>
CTBFM_DI S5<R> fluxJstPR(Gas<R> gs, const S5<R>& Ull, const S5<R>& Ul, const S5<R>& Ur, const S5<R>& Urr,
                         const S5<R>& Wl, const S5<R>& Wr, R pll, R pl, R pr, R prr, R rL, R rR, V3<R> n) {
    const S5<R> Wavg = (Wl + Wr) * R(0.5);
    const R sL = jstS(pll, pl, pr), sR = jstS(pl, pr, prr);
    const R r = rmax(rL, rR);
    const R sf = rmax(sL, sR);
    const R psi2 = R(0.5) * sf * r;
    const R psi4 = rmax(R(0), R(0.02) * r - R(2) * psi2);
    const S5<R> F = advFlux(gs, Wavg, n);
    const S5<R> d = (Ur - Ul) * psi2 - (((Urr - Ur) - (Ur - Ul) * R(2)) + (Ul - Ull)) * psi4;
    return F - d;
}

template <typename R>
CTBFM_DI S5<R> fluxJstW(Gas<R> gs, const S5<R>& Ull, const S5<R>& Ul, const S5<R>& Ur, const S5<R>& Urr,
                        const S5<R>& Wll, const S5<R>& Wl, const S5<R>& Wr, const S5<R>& Wrr, V3<R> n) {
    return fluxJstPR(gs, Ull, Ul, Ur, Urr, Wl, Wr, pressurePrim(gs, Wll), pressurePrim(gs, Wl), pressurePrim(gs, Wr),
                     pressurePrim(gs, Wrr), jstR(gs, Wl), jstR(gs, Wr), n);
}

template <typename R>
CTBFM_DI S5<R> fluxJst(Gas<R> gs, const S5<R>& Ull, const S5<R>& Ul, const S5<R>& Ur, const S5<R>& Urr, V3<R> n) {
    return fluxJstW(gs, Ull, Ul, Ur, Urr, primOf(Ull), primOf(Ul), primOf(Ur), primOf(Urr), n);
}

// ------------------------------------------------------ Roe + MUSCL flux
// AdvectionBase::computeReconstructionSmoothness / computeLimiter
// (src/advection_base.cpp:28-64).
template <typename R>
CTBFM_DI R smooth1(R l, R c, R r) {
    const R dR = r - c;
    const R dL = c - l;
    return (fabs(dR) < R(1E-12)) ? R(0) : dL / dR;
}
template <typename R>
CTBFM_DI R limiter1(int lim, R x) {
    switch (lim) {
        case 1: return (x <= R(0)) ? R(0) : (x * x + x) / (R(1) + x * x);  // van Albada
        case 2: return (x + fabs(x)) / (R(1) + fabs(x));                  // van Leer
        case 3: return rmax(R(0), rmin(R(1), x));                         // minmod
        default: return R(0);
    }
}
template <typename R>
CTBFM_DI R roeAvg(R sl, R sr, R pl, R pr) {  // roeAverage with sl = sqrt(rhoL)
    return (sl * pl + sr * pr) / (sl + sr);
}

// AdvectionRoe::computeFlux (src/advection_roe.cpp:6-220), entropy fix 0.01
// (include/advection_roe.hpp:63), on primitive states.
template <typename R>
CTBFM_DI S5<R> fluxRoeW(Gas<R> gs, int muscl, int lim, const S5<R>& Wll, S5<R> Wl, S5<R> Wr, const S5<R>& Wrr,
                        V3<R> n1, V3<R> n2);

// The same, with the triad's second vector computed here from n1.
template <typename R>
CTBFM_DI S5<R> fluxRoeW(Gas<R> gs, int muscl, int lim, const S5<R>& Wll, const S5<R>& Wl, const S5<R>& Wr,
                        const S5<R>& Wrr, V3<R> n1) {
    // normal triad (:41-58); n1 = S.normalized() equals the stored unit normal
    V3<R> n2 = (n1.x == R(0) && n1.y == R(0)) ? v3(R(1), R(0), R(0)) : v3(-n1.y, n1.x, R(0));
    return fluxRoeW(gs, muscl, lim, Wll, Wl, Wr, Wrr, n1, normalized(n2));
}

template <typename R>
CTBFM_DI S5<R> fluxRoeW(Gas<R> gs, int muscl, int lim, const S5<R>& Wll, S5<R> Wl, S5<R> Wr, const S5<R>& Wrr,
                        V3<R> n1, V3<R> n2) {
    if (muscl) {
        S5<R> limL, limR;
#pragma unroll
        for (int i = 0; i < 5; i++) {
            limL.v[i] = limiter1(lim, smooth1(Wll.v[i], Wl.v[i], Wr.v[i]));
            limR.v[i] = limiter1(lim, smooth1(Wl.v[i], Wr.v[i], Wrr.v[i]));
        }
#pragma unroll
        for (int i = 0; i < 5; i++) Wl.v[i] += limL.v[i] * (Wr.v[i] - Wl.v[i]) * R(0.5);
#pragma unroll
        for (int i = 0; i < 5; i++) Wr.v[i] -= limR.v[i] * (Wrr.v[i] - Wr.v[i]) * R(0.5);
    }
    const V3<R> n3 = cross(n1, n2);
    const V3<R> uL = velOf(Wl), uR = velOf(Wr);
    const R rhoL = Wl.v[0], rhoR = Wr.v[0];
    const R u1L = dot(uL, n1), u2L = dot(uL, n2), u3L = dot(uL, n3);
    const R u1R = dot(uR, n1), u2R = dot(uR, n2), u3R = dot(uR, n3);
    const R etL = Wl.v[4], etR = Wr.v[4];
    // Roe averages (:68-143)
    const R htL = totalEnthalpy_rho_u_et(gs, rhoL, v3(u1L, u2L, u3L), etL);
    const R htR = totalEnthalpy_rho_u_et(gs, rhoR, v3(u1R, u2R, u3R), etR);
    const R rhoA = sqrt(rhoL * rhoR);
    const R sl = sqrt(rhoL), sr = sqrt(rhoR);
    const R u1A = roeAvg(sl, sr, u1L, u1R);
    const R u2A = roeAvg(sl, sr, u2L, u2R);
    const R u3A = roeAvg(sl, sr, u3L, u3R);
    const R htA = roeAvg(sl, sr, htL, htR);
    const R eL = etL - R(0.5) * (u1L * u1L + u2L * u2L + u3L * u3L);
    const R eR = etR - R(0.5) * (u1R * u1R + u2R * u2R + u3R * u3R);
    const R pL = pressure_rho_e(gs, rhoL, eL);
    const R pR = pressure_rho_e(gs, rhoR, eR);
    const R chiL = dpdrho_e(gs, rhoL, eL), kapL = dpde_rho(gs, rhoL, eL);
    const R chiR = dpdrho_e(gs, rhoR, eR), kapR = dpde_rho(gs, rhoR, eR);
    const R barChi = R(0.5) * (chiL + chiR);
    const R barKap = R(0.5) * (kapL + kapR);
    const R barRho = R(0.5) * (rhoL + rhoR);
    const R barE = R(0.5) * (eL + eR);
    const R dP = pR - pL, dRho = rhoR - rhoL, dE = eR - eL;
    const R dRhoHat = (barRho > R(1e-12)) ? dRho / barRho : R(0);
    const R dEHat = (fabs(barE) > R(1e-12)) ? dE / fabs(barE) : R(0);
    const R dNorm2 = dRhoHat * dRhoHat + dEHat * dEHat;
    R chiT = barChi, kapT = barKap;
    if (dNorm2 > R(1e-12)) {
        const R res = dP - (barChi * dRho + barKap * dE);
        chiT += (res * dRhoHat) / (dNorm2 * barRho);
        kapT += (res * dEHat) / (dNorm2 * fabs(barE));
    }
    if (barKap > R(0) && kapT <= R(0)) kapT = R(0.01) * barKap;
    const R kapP = (rhoA > R(1e-12)) ? kapT / rhoA : R(0.4);
    const R eA = roeAvg(sl, sr, eL, eR);
    const R chiP = chiT - kapP * eA;
    const R q2 = u1A * u1A + u2A * u2A + u3A * u3A;
    const R hA = htA - R(0.5) * q2;
    R a2 = chiP + kapP * hA;
    if (a2 <= R(0)) {
        const R aL = soundSpeed_rho_e(gs, rhoL, eL), aR = soundSpeed_rho_e(gs, rhoR, eR);
        a2 = R(0.5) * (aL * aL + aR * aR);
    }
    const R aA = sqrt(a2);
    // eigenvalues, eigenvectors, wave strengths (:146-185)
    const R lam[5] = {u1A - aA, u1A, u1A, u1A, u1A + aA};
    const R cE5 = htA - (aA * aA) / kapP;
    const R ev[5][5] = {{R(1), u1A - aA, u2A, u3A, htA - aA * u1A},
                        {R(1), u1A, u2A, u3A, cE5},
                        {R(0), R(0), R(1), R(0), u2A},
                        {R(0), R(0), R(0), R(1), u3A},
                        {R(1), u1A + aA, u2A, u3A, htA + aA * u1A}};
    const R ddRho = rhoR - rhoL;
    const R du1 = u1R - u1L, du2 = u2R - u2L, du3 = u3R - u3L;
    const R ppL = pressure_rho_u_et(gs, rhoL, v3(u1L, u2L, u3L), etL);
    const R ppR = pressure_rho_u_et(gs, rhoR, v3(u1R, u2R, u3R), etR);
    const R ddP = ppR - ppL;
    R ws[5];
    ws[0] = R(1) / (R(2) * aA * aA) * (ddP - rhoA * aA * du1);
    ws[1] = ddRho - ddP / (aA * aA);
    ws[2] = rhoA * du2;
    ws[3] = rhoA * du3;
    ws[4] = R(1) / (R(2) * aA * aA) * (ddP + rhoA * aA * du1);
    // assembly (:188-220)
    const V3<R> e1 = v3(R(1), R(0), R(0));
    const S5<R> FL = advFlux(gs, s5(rhoL, u1L, u2L, u3L, etL), e1);
    const S5<R> FR = advFlux(gs, s5(rhoR, u1R, u2R, u3R, etR), e1);
    R fix[5];
#pragma unroll
    for (int i = 0; i < 5; i++) fix[i] = (fabs(lam[i]) < R(0.01)) ? R(0.01) : fabs(lam[i]);
    S5<R> Fr = (FL + FR) * R(0.5);
#pragma unroll
    for (int i = 0; i < 5; i++)
#pragma unroll
        for (int j = 0; j < 5; j++) Fr.v[i] -= R(0.5) * ws[j] * fix[j] * ev[j][i];
    const V3<R> ex = v3(R(1), R(0), R(0)), ey = v3(R(0), R(1), R(0)), ez = v3(R(0), R(0), R(1));
    return s5(Fr.v[0], Fr.v[1] * (dot(n1, ex)) + Fr.v[2] * (dot(n2, ex)) + Fr.v[3] * (dot(n3, ex)),
              Fr.v[1] * (dot(n1, ey)) + Fr.v[2] * (dot(n2, ey)) + Fr.v[3] * (dot(n3, ey)),
              Fr.v[1] * (dot(n1, ez)) + Fr.v[2] * (dot(n2, ez)) + Fr.v[3] * (dot(n3, ez)), Fr.v[4]);
}

template <typename R>
CTBFM_DI S5<R> fluxRoe(Gas<R> gs, int muscl, int lim, const S5<R>& Ull, const S5<R>& Ul, const S5<R>& Ur,
                       const S5<R>& Urr, V3<R> n1) {
    return fluxRoeW(gs, muscl, lim, muscl ? primOf(Ull) : zero5<R>(), primOf(Ul), primOf(Ur),
                    muscl ? primOf(Urr) : zero5<R>(), n1);
}

// ----------------------------------------------------------- boundaries

// Config::computeRampedOutletPressure (src/config.cpp:430-439).
template <typename R>
CTBFM_DI R rampedOutletPressure(const DevCaseT<R>& c, long long it, R p) {
    const double ratio = static_cast<double>(it) / c.ramp_iters;
    if (ratio >= 1.0) return p;
    return R(c.init_p + (static_cast<double>(p) - c.init_p) * ratio);
}

// BoundaryBase::computeOutletFlux (src/boundary_base.cpp:181-224).
template <typename R>
CTBFM_DI S5<R> bcOutlet(const DevCaseT<R>& c, Gas<R> gs, const S5<R>& Uint, V3<R> n, R pOut, long long it) {
    const S5<R> W = primOf(Uint);
    const V3<R> u = velOf(W);
    const R rho = W.v[0];
    const R p = pressure_rho_u_et(gs, rho, u, W.v[4]);
    const R a = soundSpeed_p_rho(gs, p, W.v[0]);
    if (mag(u) >= a) return advFlux(gs, W, n);
    const R pb = rampedOutletPressure(c, it, pOut);
    R rhob, eb;
    if (gs.lut) {  // isentropic extrapolation (src/boundary_base.cpp:206-211)
        const R eInt = W.v[4] - R(0.5) * dot(u, u);
        const R sInt = lutInterp(gs.lut->re[kReS], rho, eInt);
        rhob = lutInterp(gs.lut->ps[kPsRho], pb, sInt);
        eb = lutInterp(gs.lut->ps[kPsE], pb, sInt);
    } else {
        rhob = pb * rho / p;
        eb = staticEnergy_p_rho(gs, pb, rhob);
    }
    const R etb = eb + R(0.5) * dot(u, u);
    return advFlux(gs, s5(rhob, u.x, u.y, u.z, etb), n);
}

// BoundaryInviscidWall::computeBoundaryFlux (src/boundary_inviscid_wall.cpp:5-30).
template <typename R>
CTBFM_DI S5<R> bcWall(Gas<R> gs, const S5<R>& Uint, V3<R> n) {
    const S5<R> W = primOf(Uint);
    const V3<R> u = velOf(W);
    const R p = pressure_rho_u_et(gs, W.v[0], u, W.v[4]);
    const R un = dot(u, n);
    const R a = soundSpeed_p_rho(gs, p, W.v[0]);
    R pw = p + W.v[0] * un * a;
    if (pw < R(0.01) * p) pw = R(0.01) * p;
    return s5(R(0), pw * n.x, pw * n.y, pw * n.z, R(0));
}

template <typename R>
CTBFM_DI R density_p_T(Gas<R> gs, R p, R T) {  // :134-136; FluidReal::computeDensity_p_T (the (p, T) table)
    if (gs.lut) return lutInterp(gs.lut->pt[kPtRho], p, T);
    return p / (gs.R_ * T);
}

// BoundaryOutletSupersonic::computeBoundaryFlux (src/boundary_outlet_supersonic.cpp:4-14).
template <typename R>
CTBFM_DI S5<R> bcOutletSupersonic(Gas<R> gs, const S5<R>& Uint, V3<R> n) {
    return advFlux(gs, primOf(Uint), n);
}

// BoundaryInletSupersonic::computeBoundaryFlux (src/boundary_inlet_supersonic.cpp:4-34):
// the state of the patch values (p, T, u, v, w).
template <typename R>
CTBFM_DI S5<R> bcInletSupersonic(Gas<R> gs, const DevPatch& pt, V3<R> n) {
    const R p = R(pt.v[0]), T = R(pt.v[1]);
    const V3<R> u = v3(R(pt.v[2]), R(pt.v[3]), R(pt.v[4]));
    const R rho = density_p_T(gs, p, T);
    const R e = staticEnergy_p_rho(gs, p, rho);
    const R et = e + R(0.5) * dot(u, u);
    return advFlux(gs, s5(rho, u.x, u.y, u.z, et), n);
}

// BoundaryFarfield::computeBoundaryFlux (src/boundary_farfield.cpp:5-144):
// freestream (Mach, p, T, direction) from the patch values; supersonic
// outflow takes the interior state, supersonic inflow the freestream, and
// subsonic faces combine the outgoing and incoming characteristics, with
// Riemann invariants for the ideal gas and acoustic impedance plus (p, s)
// tables for the real gas.
template <typename R>
CTBFM_DI S5<R> bcFarfield(Gas<R> gs, const DevPatch& pt, const S5<R>& Uint, V3<R> n) {
    const R g = gs.g;
    const R machInf = R(pt.v[0]), pInf = R(pt.v[1]), TInf = R(pt.v[2]);
    V3<R> dir = v3(R(pt.v[3]), R(pt.v[4]), R(pt.v[5]));
    dir = dir / mag(dir);
    const R rhoInf = density_p_T(gs, pInf, TInf);
    const R aInf = soundSpeed_p_rho(gs, pInf, rhoInf);
    const V3<R> uInf = dir * (machInf * aInf);
    const S5<R> W = primOf(Uint);
    const R rhoI = W.v[0];
    const V3<R> uI = velOf(W);
    const R pI = pressure_rho_u_et(gs, rhoI, uI, W.v[4]);
    const R aI = soundSpeed_p_rho(gs, pI, rhoI);
    const R unI = dot(uI, n);
    const R unInf = dot(uInf, n);
    if (unI >= aI) return advFlux(gs, W, n);
    if (unI <= -aI) {
        const R eInf = staticEnergy_p_rho(gs, pInf, rhoInf);
        const R etInf = eInf + R(0.5) * dot(uInf, uInf);
        return advFlux(gs, s5(rhoInf, uInf.x, uInf.y, uInf.z, etInf), n);
    }
    R rhoB, eB;
    R unB;
    V3<R> uRef;
    if (!gs.lut) {
        const R Rp = unI + R(2) * aI / (g - R(1));
        const R Rm = unInf - R(2) * aInf / (g - R(1));
        unB = R(0.5) * (Rp + Rm);
        const R aB = R(0.25) * (g - R(1)) * (Rp - Rm);
        R rhoRef, pRef;
        if (unB > R(0)) {
            rhoRef = rhoI;
            pRef = pI;
            uRef = uI;
        } else {
            rhoRef = rhoInf;
            pRef = pInf;
            uRef = uInf;
        }
        const R ent = pRef / pow(rhoRef, g);
        rhoB = pow(aB * aB / (g * ent), R(1) / (g - R(1)));
        const R pB = rhoB * aB * aB / g;
        eB = staticEnergy_p_rho(gs, pB, rhoB);
    } else {
        const R rhoAvg = R(0.5) * (rhoI + rhoInf);
        const R aAvg = R(0.5) * (aI + aInf);
        const R Z = rhoAvg * aAvg;
        const R Rp = unI + pI / Z;
        const R Rm = unInf - pInf / Z;
        unB = R(0.5) * (Rp + Rm);
        const R pB = R(0.5) * (Rp - Rm) * Z;
        R sRef;
        if (unB > R(0)) {
            const R eI = W.v[4] - R(0.5) * dot(uI, uI);
            sRef = lutInterp(gs.lut->re[kReS], rhoI, eI);
            uRef = uI;
        } else {
            sRef = lutInterp(gs.lut->pt[kPtS], pInf, TInf);
            uRef = uInf;
        }
        rhoB = lutInterp(gs.lut->ps[kPsRho], pB, sRef);
        eB = lutInterp(gs.lut->ps[kPsE], pB, sRef);
    }
    const V3<R> ut = uRef - n * dot(uRef, n);
    const V3<R> uB = ut + n * unB;
    const R etB = eB + R(0.5) * dot(uB, uB);
    return advFlux(gs, s5(rhoB, uB.x, uB.y, uB.z, etB), n);
}

// BoundaryInlet::computeBoundaryFlux (src/boundary_inlet.cpp:4-43) and
// BoundaryBase::computeSubsonicInletFlux (src/boundary_base.cpp:7-124);
// cth/sth are cos/sin of the node's theta for the cylindrical frame.
template <typename R>
CTBFM_DI S5<R> bcInlet(const DevCaseT<R>& c, Gas<R> gs, const DevPatch& pt, const S5<R>& Uint, V3<R> n, R cth,
                       R sth) {
    const R Pt = R(pt.v[0]), Tt = R(pt.v[1]);
    V3<R> dir = v3(R(pt.v[2]), R(pt.v[3]), R(pt.v[4]));
    if (c.inlet_cyl) dir = cartOfCyl(dir, cth, sth);
    if (dir.x == R(1) && dir.y == R(1) && dir.z == R(1)) dir = -n;  // -S / |S|
    else dir = dir / mag(dir);
    const S5<R> W = primOf(Uint);
    const V3<R> u = velOf(W);
    const R aInt = soundSpeed_rho_u_et(gs, W.v[0], u, W.v[4]);
    const R unInt = dot(u, n);
    const R Z = W.v[0] * aInt;
    const R pInt = pressure_rho_u_et(gs, W.v[0], u, W.v[4]);
    R Cg = dot(dir, n);
    if (Cg >= R(0)) Cg = R(-1);
    const R Rout = pInt + Z * unInt;
    if (gs.lut) {  // src/boundary_base.cpp:78-111, the search in double on the (p, s) tables
        const DevLut& L = *gs.lut;
        const double Ptd = pt.v[0], Ttd = pt.v[1];
        const double Zd = Z, Cgd = Cg, Routd = Rout;
        const double sIn = lutInterp(L.pt[kPtS], Ptd, Ttd);
        const double htIn = lutEnthalpy_p_s(L, Ptd, sIn);
        double pLow = 0.05 * Ptd, pHigh = 0.999999 * Ptd;
        double pB = 0.5 * (pLow + pHigh);
        for (int iter = 0; iter < 30; ++iter) {
            const double pMid = 0.5 * (pLow + pHigh);
            const double hMid = lutEnthalpy_p_s(L, pMid, sIn);
            const double VMid = sqrt(2.0 * rmax(0.0, htIn - hMid));
            const double res = pMid + Zd * Cgd * VMid - Routd;
            if (fabs(res) < 1e-4 * Ptd) {
                pB = pMid;
                break;
            }
            if (res < 0.0) pLow = pMid;
            else pHigh = pMid;
            pB = pMid;
        }
        const double hB = lutEnthalpy_p_s(L, pB, sIn);
        const R VB = R(sqrt(2.0 * rmax(0.0, htIn - hB)));
        const V3<R> uB = dir * VB;
        const R rhoB = R(lutInterp(L.ps[kPsRho], pB, sIn));
        const R eB = R(lutInterp(L.ps[kPsE], pB, sIn));
        const R etB = eB + R(0.5) * dot(uB, uB);
        return advFlux(gs, s5(rhoB, uB.x, uB.y, uB.z, etB), n);
    }
    const R g = gs.g, Rg = gs.R_;
    const R cp = g * Rg / (g - R(1));
    const R htIn = cp * Tt;
    R pLow = R(0.05) * Pt, pHigh = R(0.999999) * Pt;
    R pB = R(0.5) * (pLow + pHigh);
    const R ex = (g - R(1)) / g;
    for (int iter = 0; iter < 30; ++iter) {
        const R pMid = R(0.5) * (pLow + pHigh);
        const R TMid = Tt * pow(pMid / Pt, ex);
        const R hMid = cp * TMid;
        const R VMid = sqrt(R(2) * rmax(R(0), htIn - hMid));
        const R res = pMid + Z * Cg * VMid - Rout;
        if (fabs(res) < R(1e-4) * Pt) {
            pB = pMid;
            break;
        }
        if (res < R(0)) pLow = pMid;
        else pHigh = pMid;
        pB = pMid;
    }
    const R TB = Tt * pow(pB / Pt, ex);
    const R hB = cp * TB;
    const R VB = sqrt(R(2) * rmax(R(0), htIn - hB));
    const V3<R> uB = dir * VB;
    const R rhoB = pB / (Rg * TB);
    const R eB = staticEnergy_p_rho(gs, pB, rhoB);
    const R etB = eB + R(0.5) * dot(uB, uB);
    return advFlux(gs, s5(rhoB, uB.x, uB.y, uB.z, etB), n);
}

}  // namespace ctbfm
