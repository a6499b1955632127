// Device-side description of one solver instance: metric arrays, boundary
// tables, BFM fields, state buffers and the device-resident control block that
// carries the iteration counter, physical time, residual norms, turbo
// performance and plenum state from kernel to kernel without host round trips.
#pragma once

#include <cstdint>

namespace ctbfm {

constexpr int kMaxPatches = 16;
constexpr int kMaxProfiles = 4;

// Boundary types on the path (include/types.hpp:178-194 restricted).
enum DevBc : int {
    kBcInlet = 0,
    kBcOutlet = 1,
    kBcRadialEq = 2,
    kBcInviscidWall = 3,
    kBcWedge = 4,
    kBcPeriodic = 5,
    kBcThrottle = 6,
    kBcEmpty = 7
};

struct DevPatch {
    int type;
    int profile;  // radial profile index (throttle / radial equilibrium)
    double v[8];  // patch values from input.ini
};

// One face direction: unit normal n = S/|S| and area |S| per face of the face
// grid (I: (ni+1, nj, nk), J: (ni, nj+1, nk), K: (ni, nj, nk+1)), plus the
// per-face residual contribution flux * |S| written by the face kernel.
struct DevFaces {
    const double* nx;
    const double* ny;
    const double* nz;
    const double* area;
    double* c[5];
};

// Iteration state living on the device.
struct Control {
    long long it;       // iterations completed
    long long it_stop;  // kernels of iteration it+1 run only while it < it_stop
    long long hist_base;
    int status;  // 0 running, 1 converged, 2 diverged
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
};

struct DevCase {
    int ni, nj, nk;
    long long n;
    int topo;  // 0 2D, 1 3D, 2 axisymmetric
    int scheme, muscl, limiter, nstages, dt_method, steady, drop;
    int periodic, bfm, blockage, bfm_model, stalled, perturb, accel, offdesign;
    int need_turbo, greitzer, inlet_cyl, turbo_dir, nprofiles, npatches;
    int le_idx, te_idx;
    int force;  // run even when the control block says the run has stopped
    double gamma, rgas, cp, cfl, fixed_dt;
    double coeffs[4];
    double per_cos_p, per_sin_p, per_cos_m, per_sin_m;  // cos/sin of +angle and -angle
    double per_angle_deg, wedge, ramp_iters, init_p, speed_scale;
    double acc_t0, acc_t1, acc_s0, acc_s1;
    double kn, kf, kd, nu;
    double plenum_volume, ambient_p, throttle_kt, inlet_pt;
    double pert_c[3], pert_r, pert_s, pert_t0, pert_dur;

    DevFaces f[3];
    // per node
    const double* vol;
    const double* cost;  // cos(theta), theta = atan2(z, y) (host glibc)
    const double* sint;
    const double* radius;
    const double* areaK0;  // |S_K(i, j, 0)| (axisymmetric source)
    const double* edge[12];  // dI.xyz, dsI, dJ.xyz, dsJ, dK.xyz, dsK (time step)
    const double* vx;
    const double* vy;
    const double* vz;
    // boundary tables: patch index per boundary face
    const signed char* mapI;  // (2, nj, nk)
    const signed char* mapJ;  // (ni, 2, nk)
    const signed char* mapK;  // (ni, nj, 2)
    DevPatch patch[kMaxPatches];
    // radial profiles
    double* prof_p;          // concatenated pressure profiles
    const double* prof_r;    // concatenated radii
    int prof_off[kMaxProfiles];
    int prof_n[kMaxProfiles];
    int prof_type[kMaxProfiles];
    int prof_i[kMaxProfiles];     // node i of the sampled column
    int prof_j0[kMaxProfiles];    // first j
    double prof_kt[kMaxProfiles]; // throttle coefficient of the profile's patch
    // boundary planes for the surface integrals: raw S vectors
    const double* bsx[6];
    const double* bsy[6];
    const double* bsz[6];
    // BFM fields (nullptr when absent)
    const double* blk;
    const double* gbx;
    const double* gby;
    const double* gbz;
    const double* nax;
    const double* nrad;
    const double* ntan;
    const double* rpm;
    const double* stwl;
    const double* bpresent;
    const double* nblades;
    const double* cosmetal;
    const double* devpivot;
    const double* devstall;
    const double* ldbeta0;
    const double* ldkp;
    // state
    double* U[5];   // U^n
    double* S1[5];  // stage buffers
    double* S2[5];
    double* Rp[5];  // periodic-plane residuals (2 * ni * nj)
    double* W[5];   // primitives of the current stage input (k_prim)
    double* dt;
    double* partial;  // reduction partials
    int node_blocks;  // grid of the node kernel (fixed for deterministic sums)
    int per_blocks;
    int dt_blocks;
    Control* ctl;
    double* hist;  // 16 doubles per iteration row
    long long hist_cap;
};

}  // namespace ctbfm
