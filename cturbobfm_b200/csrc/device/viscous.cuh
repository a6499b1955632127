// Laminar viscous terms of the explicit loop (VISCOSITY_ACTIVE with no
// turbulence model): transport properties, the node temperature of the
// solution gradient, the viscous face flux and the stagnation flux of an
// inlet face on a no-slip wall. Every expression keeps the reference's
// operation order (the double instantiation is compiled with --fmad=false).
#pragma once

#include "physics.cuh"

namespace ctbfm {

// Products and sums that are never contracted into a fused multiply-add,
// also in the float instantiation (compiled with contraction on): the
// Green-Gauss sums of a 2-D grid cancel the two K faces' terms exactly, which
// keeps the z-gradients, and so the z-momentum, exactly zero.
CTBFM_DI float mulRn(float a, float b) { return __fmul_rn(a, b); }
CTBFM_DI double mulRn(double a, double b) { return __dmul_rn(a, b); }
CTBFM_DI float addRn(float a, float b) { return __fadd_rn(a, b); }
CTBFM_DI double addRn(double a, double b) { return __dadd_rn(a, b); }

// FluidIdeal::computeMolecularDynamicViscosity (src/fluid_ideal.cpp:224-231):
// a constant or Sutherland's law; FluidReal's (src/fluid_real.cpp:387-393)
// is a constant in both models (the host resolves it into mu_const).
template <typename R>
CTBFM_DI R molecularViscosity(const DevCaseT<R>& c, R T) {
    if (c.visc_const) return R(c.mu_const);
    const R tref = R(c.suth_T), s = R(c.suth_S);
    return R(c.suth_mu) * pow(T / tref, R(1.5)) * ((tref + s) / (T + s));
}

// Node temperature of Solver::computeSolutionGradient (src/solver.cpp:3033-3058)
// from the primitives (rho, u, v, w, et): FluidIdeal::computeTemperature_conservative
// (src/fluid_ideal.cpp:198-207), or FluidBase's (include/fluid_base.hpp:163-177)
// through the (rho, e) table for the real gas.
template <typename R>
CTBFM_DI R gradientTemperature(const DevCaseT<R>& c, Gas<R> gs, const S5<R>& W) {
    const R u = W.v[1], v = W.v[2], w = W.v[3];
    if (gs.lut) {
        const R e = W.v[4] - R(0.5) * (u * u + v * v + w * w);
        return lutInterp(gs.lut->re[kReT], W.v[0], e);
    }
    return (W.v[4] - (u * u + v * v + w * w) * R(0.5)) * R((c.gamma - 1.0) / c.rgas);
}

// TurbulenceModelSA::getEddyViscosity (src/turbulence_model_sa.cpp:843-858):
// fv1 rho nu_hat with the laminar viscosity of the model's last solve (0
// before the first, and 0 without the model: TurbulenceModelNone).
template <typename R>
CTBFM_DI R saEddy(const DevCaseT<R>& c, R rho, long long q) {
    if (!c.sa) return R(0);
    const R nuHat = c.nuhat[q];
    if (nuHat <= R(0)) return R(0);
    const R nuL = c.nul[q];
    if (nuL <= R(0)) return R(0);
    const R chi = nuHat / nuL;
    const R chi3 = chi * chi * chi;
    const R cv1_3 = R(7.1) * R(7.1) * R(7.1);
    const R fv1 = chi3 / (chi3 + cv1_3);
    return fv1 * rho * nuHat;
}

// Solver::computeViscousFlux (src/solver.cpp:2174-2226) with
// computeViscousStressTensor (src/math_utils.cpp:593-608), on the face
// average Ua of the two node states and the averaged gradients; n = S/|S|.
// The eddy conductivity is mu_t cp / Pr_t with SA (getEddyThermalConductivity,
// include/turbulence_model_sa.hpp:73) and 0 without a model. The mass
// component is 0 and not returned: the result holds momentum x, y, z and
// energy.
template <typename R>
CTBFM_DI void viscousFlux(const DevCaseT<R>& c, Gas<R> gs, const S5<R>& Ua, V3<R> gu, V3<R> gv, V3<R> gw, V3<R> gT,
                          V3<R> n, R muEddy, R (&out)[4]) {
    const S5<R> W = primOf(Ua);
    const V3<R> vel = velOf(W);
    const R T = temperature_rho_u_et(gs, W.v[0], vel, W.v[4]);
    const R muL = molecularViscosity(c, T);
    const R kappaL = R(c.vcp) * muL / R(c.vpr);
    const R muT = muL + muEddy;
    const R kappaEddy = c.sa ? muEddy * R(c.vcp) / R(c.sa_prt) : R(0);
    const R kT = kappaL + kappaEddy;
    const R lam = R(-2.0 / 3.0) * muT;
    const R xx = lam * (gu.x + gv.y + gw.z) + R(2) * muT * gu.x;
    const R yy = lam * (gu.x + gv.y + gw.z) + R(2) * muT * gv.y;
    const R zz = lam * (gu.x + gv.y + gw.z) + R(2) * muT * gw.z;
    const R xy = muT * (gu.y + gv.x);
    const R xz = muT * (gu.z + gw.x);
    const R yz = muT * (gv.z + gw.y);
    const V3<R> tX = v3(xx, xy, xz), tY = v3(xy, yy, yz), tZ = v3(xz, yz, zz);
    const R thX = dot(tX, vel) + kT * gT.x;
    const R thY = dot(tY, vel) + kT * gT.y;
    const R thZ = dot(tZ, vel) + kT * gT.z;
    out[0] = dot(tX, n);
    out[1] = dot(tY, n);
    out[2] = dot(tZ, n);
    out[3] = thX * n.x + thY * n.y + thZ * n.z;
}

// BoundaryBase::computeStagnationWallFlux (src/boundary_base.cpp:126-178) for a
// wall at rest: no mass or energy flux, the boundary pressure pB on the
// momentum (n is the outward unit normal).
template <typename R>
CTBFM_DI S5<R> stagnationWallFlux(R pB, V3<R> n) {
    return s5(R(0), pB * n.x, pB * n.y, pB * n.z, R(0));
}

}  // namespace ctbfm
