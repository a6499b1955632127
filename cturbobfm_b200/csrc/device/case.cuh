// Device-side description of one operating point (instance): metric arrays,
// boundary tables, BFM fields, state buffers and the device-resident control
// block that carries the iteration counter, physical time, residual norms,
// turbo performance and plenum state from kernel to kernel without host round
// trips. R is the working precision of the state and the metric arrays
// (double for the plain path, float for the compensated path); reductions,
// integrals, profiles and the control block are always double.
#pragma once

#include <cstdint>

namespace ctbfm {

constexpr int kMaxPatches = 16;
constexpr int kMaxProfiles = 4;

// Boundary types (include/types.hpp:178-194; the 2-D inlet file is not among
// them).
enum DevBc : int {
    kBcInlet = 0,
    kBcOutlet = 1,
    kBcRadialEq = 2,
    kBcInviscidWall = 3,
    kBcWedge = 4,
    kBcPeriodic = 5,
    kBcThrottle = 6,
    kBcEmpty = 7,
    kBcInletSupersonic = 8,
    kBcOutletSupersonic = 9,
    kBcMassFlow = 10,
    kBcTransparent = 11,
    kBcFarfield = 12,
    kBcNoSlipWall = 13
};

struct DevPatch {
    int type;
    int profile;  // radial profile index (throttle / radial equilibrium)
    double v[8];  // patch values from input.ini
};

// One face direction: unit normal n = S/|S| and area |S| per face of the face
// grid (I: (ni+1, nj, nk), J: (ni, nj+1, nk), K: (ni, nj, nk+1)), plus the
// per-face residual contribution flux * |S| written by the face kernel.
template <typename R>
struct DevFacesT {
    const R* nx;
    const R* ny;
    const R* nz;
    const R* area;
    // Roe: the second vector of the face's normal triad, (-ny, nx, 0) over
    // its magnitude ((1, 0, 0) for an axial normal), computed on the host
    // with the device's operations; its z component is 0 (nullptr for JST)
    const R* n2x;
    const R* n2y;
    R* c[5];
};

// One uniform table of the real-gas look-up (Table2D, include/fluid_real.hpp:
// 11-58): values d[i * ny + j] over x_i = xmin + i dx, y_j = ymin + j dy, in
// double and as a float copy for the float path's bulk evaluations.
struct DevTable {
    double xmin, xmax, ymin, ymax, dx, dy;
    float fxmin, fxmax, fymin, fymax, fdx, fdy;
    int nx, ny;
    const double* d;
    const float* f;
};

// The tables of FluidReal (include/fluid_real.hpp:139-160).
enum DevLutRhoE : int { kReP = 0, kReT, kReA, kReS, kReMu, kReKappa, kReDpDrho, kReDpDe };
enum DevLutPT : int { kPtRho = 0, kPtE, kPtA, kPtS };
enum DevLutPS : int { kPsRho = 0, kPsT, kPsE };
struct DevLut {
    DevTable re[8];  // over (rho, e)
    DevTable pt[4];  // over (p, T)
    DevTable ps[3];  // over (p, s)
};

// Iteration state living on the device.
struct Control {
    long long it;       // iterations completed
    long long it_stop;  // kernels of iteration it+1 run only while it < it_stop
    long long hist_base;
    int status;  // 0 running, 1 converged, 2 diverged, 3 stopped by a device error (a grid barrier wait ran out)
    int has_init;
    int has_turbo;
    int pad;
    double t;       // physical time (sum of min dt)
    double dt_min;  // min over the current iteration's dt array
    double hub_p;
    double init_log[5];
    double lognorm[5];
    double massflow[6];
    double turbo[4];  // mass flow, PRtt, TRtt, eta_tt
    double pt_int[2], tt_int[2];
    double gz_p, gz_min, gz_mout, gz_T, gz_t;  // Greitzer plenum
    // progress of the steady convergence test: the largest drop reached so
    // far, min over the tested variables of (initial maximum - log norm);
    // it_best is the last iteration at which it passed drop_mark + 0.05
    // (drop_mark then moves up to it)
    double best_drop;
    double drop_mark;
    long long it_best;
    // real gas: mass-weighted total-enthalpy and entropy integrals over the
    // inlet / outlet planes (enthalpy-based efficiency)
    double ht_int[2], s_int[2];
    // Chima: turning and loss scaling at the iteration's mass flow
    double chima_turn, chima_loss;
};

// A block's share of a batched launch: `count` consecutive elements (nodes,
// faces, periodic pairs, planes or instances) of instance `inst`, starting at
// `start`; `local` numbers the tiles of that instance (reduction partials).
// plane points per block of the boundary integrals (k_bint)
constexpr int kBintChunk = 1024;

struct Tile {
    int inst;
    int local;
    long long start;
    long long count;
};

// History row: log10 norms (5), boundary mass flows (6), turbo performance
// (4), hub static pressure (1), physical time after the iteration (1).
constexpr int kHistWidth = 17;

template <typename R>
struct alignas(16) DevCaseT {
    int ni, nj, nk;
    long long n;
    int topo;  // 0 2D, 1 3D, 2 axisymmetric
    int scheme, muscl, limiter, nstages, dt_method, steady, drop;
    int periodic, bfm, blockage, bfm_model, stalled, perturb, accel, offdesign;
    int need_turbo, greitzer, inlet_cyl, turbo_dir, nprofiles, npatches;
    int le_idx, te_idx;
    int compensated;  // the state carries a Kahan compensation term (float path)
    int force;        // run even when the control block says the run has stopped
    double gamma, rgas, cp, cfl, fixed_dt;
    double coeffs[4];
    double per_cos_p, per_sin_p, per_cos_m, per_sin_m;  // cos/sin of +angle and -angle
    double per_angle_deg, wedge, ramp_iters, init_p, speed_scale;
    double acc_t0, acc_t1, acc_s0, acc_s1;
    double kn, kf, kd, nu;
    double plenum_volume, ambient_p, throttle_kt, inlet_pt;
    double pert_c[3], pert_r, pert_s, pert_t0, pert_dur;

    DevFacesT<R> f[3];
    // per node
    const R* vol;
    const R* cost;  // cos(theta), theta = atan2(z, y) (host glibc)
    const R* sint;
    const R* radius;
    const R* areaK0;    // |S_K(i, j, 0)| (axisymmetric source)
    const R* edge[12];  // dI.xyz, dsI, dJ.xyz, dsJ, dK.xyz, dsK (time step)
    const double* vx;
    const double* vy;
    const double* vz;
    const double* cost64;  // double copies for the FP64 boundary integrals and profiles
    const double* sint64;
    // boundary tables: patch index per boundary face
    const signed char* mapI;  // (2, nj, nk)
    const signed char* mapJ;  // (ni, 2, nk)
    const signed char* mapK;  // (ni, nj, 2)
    DevPatch patch[kMaxPatches];
    // radial profiles
    double* prof_p;        // concatenated pressure profiles
    const double* prof_r;  // concatenated radii
    int prof_off[kMaxProfiles];
    int prof_n[kMaxProfiles];
    int prof_type[kMaxProfiles];
    int prof_i[kMaxProfiles];      // node i of the sampled column
    int prof_j0[kMaxProfiles];     // first j
    double prof_kt[kMaxProfiles];  // throttle coefficient of the profile's patch
    // mass-flow outlets (src/solver.cpp:2734-2770): target mass flow, relaxation,
    // boundary plane of the patch (0..5); a profile without radial
    // equilibrium is filled with the hub value instead of integrated
    double prof_mf[kMaxProfiles];
    double prof_relax[kMaxProfiles];
    int prof_plane[kMaxProfiles];
    int prof_fill[kMaxProfiles];
    double mf_max_change;  // MASS_FLOW_MAX_PRESSURE_CHANGE
    // boundary planes for the surface integrals: raw S vectors
    const double* bsx[6];
    const double* bsy[6];
    const double* bsz[6];
    // the eight boundary integrals (mass flow through planes 0..5, the Pt /
    // Tt / Ht / s integrals over the two turbo planes) are summed in chunks of
    // kBintChunk plane points, one block each, into bint_part (4 sums per
    // chunk), which k_pre adds in chunk order; the chunks of integral b are
    // bint_off[b] .. bint_off[b+1]-1
    double* bint_part;
    int bint_off[9];
    // BFM fields (nullptr when absent)
    const R* blk;
    const R* gbx;
    const R* gby;
    const R* gbz;
    const R* nax;
    const R* nrad;
    const R* ntan;
    const R* rpm;
    // per-node quantities of the blade fields alone, computed once on the
    // host with the operations the force evaluates per stage (bit for bit in
    // FP64): the camber normal over its magnitude (x/0 where the magnitude
    // is 0), the blade pitch 2 pi r / N and the shaft speed rpm 2 pi / 60
    const R* nhat[3];
    const R* pitch;
    const R* omega0;
    const R* stwl;
    const R* bpresent;
    const R* nblades;
    const R* cosmetal;
    const R* metal;  // Correlations: bladeMetalAngle
    const R* devpivot;
    const R* devstall;
    const R* ldbeta0;
    const R* ldkp;
    const R* dangmom;   // Chima: deltaAngularMomentum
    const R* dentropy;  // Chima: deltaEntropy
    const double* chima_mf;    // Chima scaling functions over the mass flow
    const double* chima_turn;
    const double* chima_loss;
    int chima_n;
    // state
    R* U[5];   // U^n
    R* Uc[5];  // Kahan compensation of U^n (compensated path; true state = U - Uc)
    R* S1[5];  // stage buffers
    R* S2[5];
    R* Rp[5];  // periodic-plane residuals (2 * ni * nj)
    R* W[5];   // primitives of the current stage input (k_prim)
    // JST: pressure and spectral radius |u| + a of each node of the current
    // stage input (k_prim; nullptr for Roe), read by the plain face stencils
    R* Wp;
    R* Wr;
    R* dt;
    // per-tile partials: [node_tiles*5 norms of the split stage |
    // per_tiles*5 periodic norms | node_tiles dt minima | nboxes*5 norms of
    // the fused stage kernel]
    double* partial;
    int node_tiles;   // tiles of this instance in the node kernels
    int per_tiles;    // tiles of this instance in the periodic kernel
    // fused stage kernel (k_stage): whether the instance can run it
    // (inviscid, no Chima / Correlations force), its box of nodes per block
    // (extent along i, j, k) and the number of boxes along i, j, k
    int fuse_ok;
    int nboxes;
    int fbox[3];
    int fnb[3];
    const DevLut* lut;  // FLUID_MODEL = real: the look-up tables; nullptr for the ideal gas
    // VISCOSITY_ACTIVE (laminar): viscosity constant (visc_const) or
    // Sutherland's law, conductivity vcp * mu / vpr; nodes of the no-slip
    // walls (at rest); per face of each direction the raw surface vector S
    // and the Green-Gauss interpolation weights of its left and right node;
    // per node the gradients of u, v, w and T (G[3 * field + component]);
    // per face the viscous contribution flux * |S| of the momentum and
    // energy equations
    int viscous, visc_const;
    double mu_const, suth_mu, suth_T, suth_S, vcp, vpr;
    const unsigned char* wall;
    const R* sraw[3][3];
    const R* gwL[3];
    const R* gwR[3];
    R* G[12];
    R* V[3][4];
    // TURBULENCE_MODEL = SA (TurbulenceModelSA): the working variable nu hat,
    // the laminar kinematic viscosity of the model's last solve, the wall
    // distance, the Green-Gauss gradient of nu hat, the node velocities and the
    // work arrays of the implicit update (residual, diagonal, forward and
    // backward increments); per face of each swept direction the distances of
    // the face centre to its left and right node (interpolateScalar); the
    // boundary patches in the boundary file's order as rows of 10 ints (kind:
    // 0 no-slip wall, 1 inlet / farfield, 2 outlet-like; node range [r0, r1) x
    // [r2, r3) x [r4, r5); donor step i, j, k)
    int sa;
    int sa_npatch;
    double sa_init_nu, sa_ff, sa_relax, sa_prt;
    R* nuhat;
    R* nul;
    const R* sa_wd;
    R* sa_res;
    R* sa_diag;
    R* sa_dstar;
    R* sa_dnu;
    R* sa_g[3];
    R* sa_vel[3];
    const R* sa_dL[3];
    const R* sa_dR[3];
    const int* sa_bc;
    Control* ctl;
    double* hist;  // kHistWidth doubles per iteration row
    long long hist_cap;
    long long max_it;  // N_ITERATIONS: no enqueue runs an instance past it
};

using DevCase = DevCaseT<double>;

// The Chima and Correlations body forces run in their own node-kernel
// variant, so the common one carries none of their code.
#ifdef __CUDACC__
#define CTBFM_HD __host__ __device__
#else
#define CTBFM_HD
#endif
template <typename R>
CTBFM_HD inline bool bfmRareModel(const DevCaseT<R>& c) {
    return c.bfm && (c.bfm_model == 5 || c.bfm_model == 6);
}

}  // namespace ctbfm
