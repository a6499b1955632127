/* CPU oracle for the CTurboBFM explicit residual-and-update loop.
 *
 * TEST INFRASTRUCTURE ONLY (see ctbfm_oracle.h). A plain-C restatement of the
 * reference's serial FP64 algorithm; every function cites the reference
 * file:line it follows. Compiled with -ffp-contract=off so that each
 * expression rounds exactly as the reference's does (pinned in tests against
 * oracle/_ref/ref_harness, the reference built from its own sources).
 *
 * Scope: the explicit Runge-Kutta path for 2-D, axisymmetric and 3-D
 * topologies, ideal gas, JST and Roe (+MUSCL) fluxes, inlet / outlet /
 * throttle / radial-equilibrium / inviscid-wall / periodic / wedge boundaries,
 * axisymmetric, blade-row geometric, Gong and BFM (Hall, Hall-Thollet,
 * Lift-Drag, blockage) sources, local / global / fixed time steps, residual
 * norms, convergence test, turbo performance and the Greitzer plenum, and
 * the restart initialisations (standard, axisymmetric, nearest neighbour).
 */
#define _GNU_SOURCE
#include "ctbfm_oracle.h"

#include <ctype.h>
#include <errno.h>
#include <float.h>
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------ errors */

static char g_err[1024];

static int fail(const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof g_err, fmt, ap);
    va_end(ap);
    return 1;
}

const char* oracle_last_error(void) { return g_err; }

/* -------------------------------------------------------------- vector ops */
/* Vector3D (include/types.hpp:15-125). Every operation keeps the reference's
 * left-to-right evaluation order. */

typedef struct { double x, y, z; } vec3;

static vec3 v3(double x, double y, double z) { vec3 r = {x, y, z}; return r; }
static vec3 vadd(vec3 a, vec3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
static vec3 vsub(vec3 a, vec3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
static vec3 vmul(vec3 a, double s) { return v3(a.x * s, a.y * s, a.z * s); }
static vec3 vdiv(vec3 a, double s) { return v3(a.x / s, a.y / s, a.z / s); }
static vec3 vneg(vec3 a) { return v3(-a.x, -a.y, -a.z); }
static double vdot(vec3 a, vec3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static double vmag(vec3 a) { return sqrt(a.x * a.x + a.y * a.y + a.z * a.z); }
static vec3 vnormalized(vec3 a) {
    double m = vmag(a);
    return (m == 0) ? v3(0, 0, 0) : vdiv(a, m);
}
static vec3 vcross(vec3 a, vec3 b) {
    return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}

/* StateVector (include/types.hpp:650-757). */
typedef struct { double v[5]; } sv5;

static sv5 sadd(sv5 a, sv5 b) { sv5 r; for (int i = 0; i < 5; i++) r.v[i] = a.v[i] + b.v[i]; return r; }
static sv5 ssub(sv5 a, sv5 b) { sv5 r; for (int i = 0; i < 5; i++) r.v[i] = a.v[i] - b.v[i]; return r; }
static sv5 smul(sv5 a, double s) { sv5 r; for (int i = 0; i < 5; i++) r.v[i] = a.v[i] * s; return r; }
static sv5 sdiv(sv5 a, double s) { sv5 r; for (int i = 0; i < 5; i++) r.v[i] = a.v[i] / s; return r; }
static sv5 szero(void) { sv5 r = {{0, 0, 0, 0, 0}}; return r; }

static double dmax(double a, double b) { return (a < b) ? b : a; } /* std::max */
static double dmin(double a, double b) { return (b < a) ? b : a; } /* std::min */

/* ------------------------------------------------------------------ config */
/* Config::load (src/config.cpp:15-44): "KEY = value", ';' and '[' lines
 * skipped, keys exact-case, later keys overwrite earlier ones. */

typedef struct { char* key; char* val; } kv;
typedef struct { kv* items; int n, cap; } config;

static void trim(char* s, const char* ws) {
    size_t n = strlen(s), a = 0;
    while (a < n && strchr(ws, s[a])) a++;
    size_t b = n;
    while (b > a && strchr(ws, s[b - 1])) b--;
    memmove(s, s + a, b - a);
    s[b - a] = 0;
}

static const char* cfg_get(const config* c, const char* key) {
    for (int i = 0; i < c->n; i++)
        if (strcmp(c->items[i].key, key) == 0) return c->items[i].val;
    return NULL;
}

static void cfg_set(config* c, const char* key, const char* val) {
    for (int i = 0; i < c->n; i++)
        if (strcmp(c->items[i].key, key) == 0) {
            free(c->items[i].val);
            c->items[i].val = strdup(val);
            return;
        }
    if (c->n == c->cap) {
        c->cap = c->cap ? 2 * c->cap : 64;
        c->items = (kv*)realloc(c->items, sizeof(kv) * c->cap);
    }
    c->items[c->n].key = strdup(key);
    c->items[c->n].val = strdup(val);
    c->n++;
}

static int cfg_load(config* c, const char* path) {
    FILE* f = fopen(path, "r");
    if (!f) return fail("Failed to load configuration file: %s", path);
    char line[4096];
    while (fgets(line, sizeof line, f)) {
        trim(line, " \t\r\n");
        if (!line[0] || line[0] == ';' || line[0] == '[') continue;
        char* eq = strchr(line, '=');
        if (!eq) continue;
        *eq = 0;
        char key[4096], val[4096];
        snprintf(key, sizeof key, "%s", line);
        snprintf(val, sizeof val, "%s", eq + 1);
        trim(key, " \t");
        trim(val, " \t");
        cfg_set(c, key, val);
    }
    fclose(f);
    return 0;
}

static void cfg_free(config* c) {
    for (int i = 0; i < c->n; i++) { free(c->items[i].key); free(c->items[i].val); }
    free(c->items);
    memset(c, 0, sizeof *c);
}

/* std::stod semantics: leading blanks skipped, at least one digit consumed. */
static int parse_double(const char* s, double* out) {
    char* end;
    errno = 0;
    double v = strtod(s, &end);
    if (end == s) return 1;
    *out = v;
    return 0;
}

static int cfg_float(const config* c, const char* key, double* out) {
    const char* v = cfg_get(c, key);
    if (!v) return fail("Not found value for key \"%s\" in configuration.", key);
    if (parse_double(v, out)) return fail("Invalid float format for key \"%s\": \"%s\"", key, v);
    return 0;
}

static int cfg_float_def(const config* c, const char* key, double def, double* out) {
    if (!cfg_get(c, key)) { *out = def; return 0; }
    return cfg_float(c, key, out);
}

static int cfg_int_def(const config* c, const char* key, int def, int* out) {
    double d;
    if (!cfg_get(c, key)) { *out = def; return 0; }
    if (cfg_float(c, key, &d)) return 1;
    *out = (int)d;
    return 0;
}

/* Config::parseBool (src/config.cpp:141-159). */
static int cfg_bool(const config* c, const char* key, int def, int* out) {
    const char* v = cfg_get(c, key);
    if (!v) { *out = def; return 0; }
    char low[256];
    snprintf(low, sizeof low, "%s", v);
    for (char* p = low; *p; p++) *p = (char)tolower((unsigned char)*p);
    if (!strcmp(low, "true") || !strcmp(low, "yes") || !strcmp(low, "1")) { *out = 1; return 0; }
    if (!strcmp(low, "false") || !strcmp(low, "no") || !strcmp(low, "0")) { *out = 0; return 0; }
    return fail("Invalid value for key \"%s\" in configuration.", key);
}

/* Config::parseVector<std::string> (include/config.hpp:29-51): comma
 * separated, items trimmed, empty items dropped. */
static int cfg_list(const config* c, const char* key, char items[][128], int max_items) {
    const char* v = cfg_get(c, key);
    if (!v) return -1;
    int n = 0;
    char buf[4096];
    snprintf(buf, sizeof buf, "%s", v);
    char* save = NULL;
    /* strtok_r would merge empty fields; the reference drops empty items too. */
    for (char* tok = strtok_r(buf, ",", &save); tok; tok = strtok_r(NULL, ",", &save)) {
        char item[1024];
        snprintf(item, sizeof item, "%s", tok);
        trim(item, " \t\r\n");
        if (!item[0]) continue;
        if (n < max_items) snprintf(items[n], 128, "%s", item);
        n++;
    }
    return n;
}

/* ------------------------------------------------------------------- enums */

enum { TOPO_2D = 0, TOPO_3D = 1, TOPO_AXI = 2, TOPO_1D = 3 };
enum { SCHEME_JST = 0, SCHEME_ROE = 1 };
enum { LIM_NONE = 0, LIM_VAN_ALBADA, LIM_VAN_LEER, LIM_MIN_MOD };
enum { DT_LOCAL = 0, DT_GLOBAL, DT_FIXED };
enum { BFM_NONE = 0, BFM_HALL, BFM_THOLLET, BFM_LIFT_DRAG, BFM_BLOCKAGE, BFM_CHIMA, BFM_CORRELATIONS };
/* BoundaryType (include/types.hpp:178-194), restricted to the types on the path. */
enum {
    BC_INLET = 0, BC_OUTLET, BC_RADIAL_EQ, BC_INVISCID_WALL, BC_WEDGE, BC_PERIODIC, BC_THROTTLE,
    BC_EMPTY, BC_INLET_SUPERSONIC, BC_OUTLET_SUPERSONIC, BC_MASS_FLOW, BC_TRANSPARENT, BC_FARFIELD,
    BC_NO_SLIP_WALL
};
enum { BI_ISTART = 0, BI_IEND, BI_JSTART, BI_JEND, BI_KSTART, BI_KEND };

/* ---------------------------------------------------------------- solver */

typedef struct {
    char name[128];
    int type;
    double values[16];
    int nvalues;
    long i_min, i_max, j_min, j_max, k_min, k_max;
    int orientation;
    int profile; /* index into the radial profiles for throttle / radial equilibrium */
} patch;

typedef struct {
    double* pressure; /* size n */
    double* radius;   /* size n or 0 */
    int n, nradius;
    int patch;
} radial_profile;

enum {
    F_BLOCKAGE = 0, F_NAX, F_NRAD, F_NTAN, F_RPM, F_STWL, F_BLADE_PRESENT, F_NBLADES, F_METAL,
    F_GASPATH, F_LEAN, F_DEV_PIVOT, F_DEV_STALL, F_LD_BETA0, F_LD_KP, F_DANGMOM, F_DENTROPY, F_CAMBER_CURV, F_COUNT
};
static const char* FIELD_NAMES[F_COUNT] = {
    "blockage", "normalAxial", "normalRadial", "normalTangential", "rpm", "streamwiseLength",
    "bladePresent", "numberBlades", "bladeMetalAngle", "bladeGasPathAngle", "bladeLeanAngle",
    "deviationAnglePivot", "deviationAngleStall", "liftDragBeta0", "liftDragKpEtamax",
    "deltaAngularMomentum", "deltaEntropy", "bladeCamberCurvature"};

struct oracle_solver {
    config cfg;
    long ni, nj, nk, n;
    int topology, ndim;
    /* settings */
    int scheme, muscl, limiter, nstages, dt_method, steady, drop;
    double coeffs[4], cfl, fixed_dt, gamma, rgas, cp;
    int bfm_active, blockage_active, bfm_model, stalled, perturb;
    double kn, kf, kd, nu;
    int offdesign, has_nu;
    double speed_scale;
    int accel; double acc_t0, acc_t1, acc_s0, acc_s1;
    double pert_center[3], pert_radius, pert_scale, pert_t0, pert_dur;
    long le_idx, te_idx;
    double *chima_mf, *chima_turn, *chima_loss; /* Chima scaling functions */
    int chima_n;
    int inlet_cyl;
    double ramp_iters, init_p;
    double mf_relax, mf_max_change; /* mass-flow outlet controller */
    int need_turbo;
    int turbo_dir; /* bcIndices pair */
    int greitzer;
    double plenum_volume, ambient_p, gz_p, gz_min, gz_mout, gz_T, gz_t, throttle_kt;
    /* FLUID_MODEL = real: the look-up table of FluidReal */
    int real;
    struct lut_s* lut;
    /* mesh */
    vec3* vert;  /* n */
    vec3* dual;  /* (ni+1)(nj+1)(nk+1) */
    vec3 *sI, *sJ, *sK, *cI, *cJ, *cK;
    double* vol;
    double wedge;
    double* field[F_COUNT];
    vec3* gradb;
    int periodic;
    double per_angle_rad, per_angle_deg, per_transl;
    /* boundaries */
    patch* patches;
    int npatches;
    int* mapI; /* 2 x nj x nk */
    int* mapJ; /* ni x 2 x nk */
    int* mapK; /* ni x nj x 2 */
    radial_profile* profiles;
    int nprofiles;
    double hub_p;
    /* VISCOSITY_ACTIVE: laminar transport (constant or Sutherland viscosity,
     * conductivity cp mu / Pr), stationary no-slip walls, Green-Gauss
     * gradients of u, v, w and T per node */
    int viscous, visc_const;
    double mu_const, suth_mu, suth_T, suth_S, vcp, vpr;
    unsigned char* wall;
    vec3* grad[4];
    double* gfield[4];
    /* TURBULENCE_ACTIVE with TURBULENCE_MODEL = SA (TurbulenceModelSA): the
     * working variable nu hat, the laminar kinematic viscosity of its last
     * solve, the wall distance and the work arrays of its implicit update */
    int sa;
    double sa_init_nu, sa_ff_scale, sa_init_scale, sa_relax, sa_prt;
    double *nuhat, *nul, *wdist, *sa_res, *sa_diag, *sa_dstar, *sa_dnu;
    vec3 *nuhat_grad, *sa_vel;
    /* state */
    double *U[5], *Utmp[5], *R[5], *dt;
    double t;
    double massflow[6];
    double turbo[4];
    int has_turbo;
    double init_log[5];
    int has_init_log;
    long iter; /* iterations performed so far (the reference's loop counter) */
    /* history of the last run */
    double* hist;
    long nhist, hist_cap;
};

static long idx3(const oracle_solver* s, long i, long j, long k) { return (i * s->nj + j) * s->nk + k; }
static long didx(const oracle_solver* s, long i, long j, long k) {
    return (i * (s->nj + 1) + j) * (s->nk + 1) + k;
}
/* surfaces/centres I: (ni+1, nj, nk); J: (ni, nj+1, nk); K: (ni, nj, nk+1) */
static long sIi(const oracle_solver* s, long i, long j, long k) { return (i * s->nj + j) * s->nk + k; }
static long sJi(const oracle_solver* s, long i, long j, long k) { return (i * (s->nj + 1) + j) * s->nk + k; }
static long sKi(const oracle_solver* s, long i, long j, long k) { return (i * s->nj + j) * (s->nk + 1) + k; }

static sv5 state_at(const oracle_solver* s, double* const* U, long i, long j, long k) {
    long q = idx3(s, i, j, k);
    sv5 r = {{U[0][q], U[1][q], U[2][q], U[3][q], U[4][q]}};
    return r;
}
static void state_set(const oracle_solver* s, double** U, long i, long j, long k, sv5 v) {
    long q = idx3(s, i, j, k);
    for (int c = 0; c < 5; c++) U[c][q] = v.v[c];
}
static void res_add(oracle_solver* s, long i, long j, long k, sv5 d) {
    long q = idx3(s, i, j, k);
    for (int c = 0; c < 5; c++) s->R[c][q] += d.v[c];
}
static void res_sub(oracle_solver* s, long i, long j, long k, sv5 d) {
    long q = idx3(s, i, j, k);
    for (int c = 0; c < 5; c++) s->R[c][q] -= d.v[c];
}

/* ------------------------------------------------------- real-gas tables */
/* Table2D (include/fluid_real.hpp:11-58): uniform grid, clamped bilinear
 * interpolation, data[i * ny + j]. */
typedef struct {
    long nx, ny;
    double xmin, xmax, ymin, ymax, dx, dy;
    double* d;
} table2d;

static void table_init(table2d* t, long nx, long ny, double x0, double x1, double y0, double y1) {
    t->nx = nx; t->ny = ny; t->xmin = x0; t->xmax = x1; t->ymin = y0; t->ymax = y1;
    t->dx = (nx > 1) ? (x1 - x0) / (double)(nx - 1) : 1.0;
    t->dy = (ny > 1) ? (y1 - y0) / (double)(ny - 1) : 1.0;
    free(t->d);
    t->d = (double*)calloc((size_t)(nx * ny > 0 ? nx * ny : 1), sizeof(double));
}

static double clampd(double v, double lo, double hi) { return (v < lo) ? lo : ((hi < v) ? hi : v); } /* std::clamp */

static double table_interp(const table2d* t, double x, double y) {
    double xc = clampd(x, t->xmin, t->xmax);
    double yc = clampd(y, t->ymin, t->ymax);
    double rx = (xc - t->xmin) / t->dx;
    double ry = (yc - t->ymin) / t->dy;
    /* size_t conversion; a NaN coordinate lands on the last cell either way */
    unsigned long i = (rx >= 0.0 && rx < 1e18) ? (unsigned long)rx : (unsigned long)t->nx;
    unsigned long j = (ry >= 0.0 && ry < 1e18) ? (unsigned long)ry : (unsigned long)t->ny;
    if (i >= (unsigned long)(t->nx - 1)) i = (t->nx >= 2) ? (unsigned long)(t->nx - 2) : 0;
    if (j >= (unsigned long)(t->ny - 1)) j = (t->ny >= 2) ? (unsigned long)(t->ny - 2) : 0;
    double wx = rx - (double)i;
    double wy = ry - (double)j;
    double f00 = t->d[i * t->ny + j];
    double f10 = t->d[(i + 1) * t->ny + j];
    double f01 = t->d[i * t->ny + (j + 1)];
    double f11 = t->d[(i + 1) * t->ny + (j + 1)];
    return (1.0 - wx) * (1.0 - wy) * f00 + wx * (1.0 - wy) * f10 + (1.0 - wx) * wy * f01 + wx * wy * f11;
}

typedef struct lut_s {
    double molar, R, pcrit, Tcrit, rhocrit, gnom;
    table2d p, T, a, s, mu, kappa, dpdrho, dpde; /* (rho, e) */
    table2d rho_pt, e_pt, a_pt, s_pt;           /* (p, T) */
    table2d rho_ps, T_ps, e_ps;                 /* (p, s) */
} lut;

static void lut_free(lut* L) {
    if (!L) return;
    table2d* all[15] = {&L->p, &L->T, &L->a, &L->s, &L->mu, &L->kappa, &L->dpdrho, &L->dpde,
                        &L->rho_pt, &L->e_pt, &L->a_pt, &L->s_pt, &L->rho_ps, &L->T_ps, &L->e_ps};
    for (int q = 0; q < 15; q++) free(all[q]->d);
    free(L);
}

/* splits "KEY: value" with the reference's trimming; returns 0 without ':' */
static int lut_keyval(const char* line, char* key, size_t nk, char* val, size_t nv) {
    const char* colon = strchr(line, ':');
    if (!colon) return 0;
    size_t kl = (size_t)(colon - line);
    if (kl >= nk) kl = nk - 1;
    memcpy(key, line, kl);
    key[kl] = 0;
    trim(key, " \t\r\n");
    snprintf(val, nv, "%s", colon + 1);
    trim(val, " \t\r\n");
    return 1;
}

/* reads the next data line (skipping empty, '#' and '\r' lines) into v[n] */
static int lut_row(FILE* f, char* line, size_t cap, double* v, int n) {
    do {
        if (!fgets(line, (int)cap, f)) return 1;
    } while (line[0] == '\n' || line[0] == '#' || line[0] == '\r' || line[0] == 0);
    char* p = line;
    for (int q = 0; q < n; q++) {
        char* e = NULL;
        v[q] = strtod(p, &e);
        if (e == p) v[q] = 0.0;
        p = e;
    }
    return 0;
}

/* FluidReal::loadTable (src/fluid_real.cpp:12-208). */
static int lut_load(lut* L, const char* path) {
    FILE* f = fopen(path, "r");
    if (!f) return fail("FluidReal: Could not open table file at: %s", path);
    L->R = 287.0; L->gnom = 1.3;
    char line[4096], key[256], val[1024];
    int sec = 0; /* 1 RHO_E, 2 P_T, 3 P_S */
    long n1 = 0, n2 = 0;
    double x0 = 0, x1 = 0, y0 = 0, y1 = 0;
    while (fgets(line, sizeof line, f)) {
        size_t len = strlen(line);
        if (len && line[len - 1] == '\n') line[--len] = 0;
        if (len == 0 || line[0] == '\r') continue;
        if (strstr(line, "# SECTION: RHO_E")) { sec = 1; continue; }
        if (strstr(line, "# SECTION: P_T")) { sec = 2; continue; }
        if (strstr(line, "# SECTION: P_S")) { sec = 3; continue; }
        if (line[0] == '#') continue;
        if (!lut_keyval(line, key, sizeof key, val, sizeof val)) continue;
        if (sec == 0) {
            if (!strcmp(key, "MOLAR_MASS")) L->molar = strtod(val, NULL);
            else if (!strcmp(key, "GAS_CONSTANT")) L->R = strtod(val, NULL);
            else if (!strcmp(key, "CRITICAL_PRESSURE")) L->pcrit = strtod(val, NULL);
            else if (!strcmp(key, "CRITICAL_TEMPERATURE")) L->Tcrit = strtod(val, NULL);
            else if (!strcmp(key, "CRITICAL_DENSITY")) L->rhocrit = strtod(val, NULL);
            else if (!strcmp(key, "NOMINAL_GAMMA")) L->gnom = strtod(val, NULL);
            continue;
        }
        const char* kn1 = sec == 1 ? "N_RHO" : "N_P";
        const char* kn2 = sec == 1 ? "N_E" : (sec == 2 ? "N_T" : "N_S");
        const char* kx0 = sec == 1 ? "RHO_MIN" : "P_MIN";
        const char* kx1 = sec == 1 ? "RHO_MAX" : "P_MAX";
        const char* ky0 = sec == 1 ? "E_MIN" : (sec == 2 ? "T_MIN" : "S_MIN");
        const char* ky1 = sec == 1 ? "E_MAX" : (sec == 2 ? "T_MAX" : "S_MAX");
        if (!strcmp(key, kn1)) n1 = strtol(val, NULL, 10);
        else if (!strcmp(key, kn2)) n2 = strtol(val, NULL, 10);
        else if (!strcmp(key, kx0)) x0 = strtod(val, NULL);
        else if (!strcmp(key, kx1)) x1 = strtod(val, NULL);
        else if (!strcmp(key, ky0)) y0 = strtod(val, NULL);
        else if (!strcmp(key, ky1)) {
            y1 = strtod(val, NULL);
            table2d* t[8];
            int nt;
            if (sec == 1) {
                table2d* q[8] = {&L->p, &L->T, &L->a, &L->s, &L->mu, &L->kappa, &L->dpdrho, &L->dpde};
                memcpy(t, q, sizeof q); nt = 8;
            } else if (sec == 2) {
                table2d* q[4] = {&L->rho_pt, &L->e_pt, &L->a_pt, &L->s_pt};
                memcpy(t, q, sizeof q); nt = 4;
            } else {
                table2d* q[3] = {&L->rho_ps, &L->T_ps, &L->e_ps};
                memcpy(t, q, sizeof q); nt = 3;
            }
            for (int q = 0; q < nt; q++) table_init(t[q], n1, n2, x0, x1, y0, y1);
            double v[8];
            int stop = 0;
            for (long i = 0; i < n1 && !stop; i++)
                for (long j = 0; j < n2; j++) {
                    if (lut_row(f, line, sizeof line, v, nt)) { stop = 1; break; }
                    for (int q = 0; q < nt; q++) t[q]->d[i * n2 + j] = v[q];
                }
        }
    }
    fclose(f);
    return 0;
}

/* FluidReal inversions (src/fluid_real.cpp:211-320). */
static double lut_e_p_rho(const lut* L, double p, double rho) { /* computeStaticEnergy_p_rho :227-250 */
    double eLo = L->p.ymin, eHi = L->p.ymax;
    double pLo = table_interp(&L->p, rho, eLo);
    double pHi = table_interp(&L->p, rho, eHi);
    if (p <= pLo) return eLo;
    if (p >= pHi) return eHi;
    for (int it = 0; it < 30; ++it) {
        double eMid = 0.5 * (eLo + eHi);
        double pMid = table_interp(&L->p, rho, eMid);
        if (fabs(pMid - p) <= 1e-4 * p) return eMid;
        if (pMid < p) eLo = eMid; else eHi = eMid;
    }
    return 0.5 * (eLo + eHi);
}
static double lut_h_p_s(const lut* L, double p, double s) { /* FluidBase::computeEnthalpy_p_s */
    return table_interp(&L->e_ps, p, s) + p / table_interp(&L->rho_ps, p, s);
}
static double lut_pt_rho_e_et(const lut* L, double rho, double e, double et) { /* :299-321 */
    double p = table_interp(&L->p, rho, e);
    double sv = table_interp(&L->s, rho, e);
    double ht = et + p / rho;
    double pLo = p, pHi = L->rho_ps.xmax;
    for (int it = 0; it < 25; ++it) {
        double pMid = 0.5 * (pLo + pHi);
        double rhoMid = table_interp(&L->rho_ps, pMid, sv);
        double eMid = table_interp(&L->e_ps, pMid, sv);
        double hMid = eMid + pMid / rhoMid;
        if (hMid < ht) pLo = pMid; else pHi = pMid;
    }
    return 0.5 * (pLo + pHi);
}

/* ------------------------------------------------------- fluid (ideal gas) */
/* FluidIdeal (src/fluid_ideal.cpp). */

static double f_pressure_rho_e(const oracle_solver* s, double rho, double e) { /* :14-16 */
    if (s->real) return table_interp(&s->lut->p, rho, e); /* FluidReal :211-213 */
    return (s->gamma - 1) * rho * e;
}
static double f_static_energy_u_et(vec3 u, double et) { /* :74-77, pow(|u|,2) == |u|*|u| */
    double m = vmag(u);
    double m2 = m * m;
    return et - 0.5 * m2;
}
/* FluidBase::computeStaticEnergy_u_et (include/fluid_base.hpp:78-80), used by
 * FluidReal: et - 0.5 u.u */
static double fb_static_energy_u_et(vec3 u, double et) { return et - 0.5 * vdot(u, u); }
static double f_pressure_rho_u_et(const oracle_solver* s, double rho, vec3 u, double et) { /* :89-92 */
    if (s->real) return table_interp(&s->lut->p, rho, fb_static_energy_u_et(u, et)); /* fluid_base.hpp:91-94 */
    double e = f_static_energy_u_et(u, et);
    return f_pressure_rho_e(s, rho, e);
}
static double f_sound_speed_p_rho(const oracle_solver* s, double p, double rho) { /* :70-72 */
    if (s->real) return table_interp(&s->lut->a, rho, lut_e_p_rho(s->lut, p, rho)); /* FluidReal :252-255 */
    return sqrt(s->gamma * p / rho);
}
static double f_sound_speed_rho_u_et(const oracle_solver* s, double rho, vec3 u, double et) { /* :83-87 */
    if (s->real) return table_interp(&s->lut->a, rho, fb_static_energy_u_et(u, et)); /* fluid_base.hpp:86-89 */
    double e = f_static_energy_u_et(u, et);
    double p = f_pressure_rho_e(s, rho, e);
    return f_sound_speed_p_rho(s, p, rho);
}
static double f_sound_speed_rho_e(const oracle_solver* s, double rho, double e) { /* :22-24 */
    if (s->real) return table_interp(&s->lut->a, rho, e); /* FluidReal :219-221 */
    return sqrt(s->gamma * (s->gamma - 1.0) * e);
}
static double f_total_enthalpy_rho_u_et(const oracle_solver* s, double rho, vec3 u, double et) { /* :114-118 */
    if (s->real) return et + f_pressure_rho_u_et(s, rho, u, et) / rho; /* fluid_base.hpp:106-109 */
    double e = f_static_energy_u_et(u, et);
    double p = f_pressure_rho_e(s, rho, e);
    return et + p / rho;
}
static double f_temperature_rho_u_et(const oracle_solver* s, double rho, vec3 u, double et) { /* :109-112 */
    if (s->real) return table_interp(&s->lut->T, rho, fb_static_energy_u_et(u, et)); /* fluid_base.hpp:96-99 */
    double p = f_pressure_rho_u_et(s, rho, u, et);
    return p / (rho * s->rgas);
}
static double f_static_energy_p_rho(const oracle_solver* s, double p, double rho) { /* :10-12 */
    if (s->real) return lut_e_p_rho(s->lut, p, rho);
    return p / ((s->gamma - 1) * rho);
}
static double f_mach_rho_u_et(const oracle_solver* s, double rho, vec3 u, double et) { /* :137-141 */
    double a = f_sound_speed_rho_u_et(s, rho, u, et);
    double um = vmag(u);
    return um / a;
}
static double f_total_pressure_rho_u_et(const oracle_solver* s, double rho, vec3 u, double et) { /* :94-98 */
    if (s->real) return lut_pt_rho_e_et(s->lut, rho, fb_static_energy_u_et(u, et), et);
    double p = f_pressure_rho_u_et(s, rho, u, et);
    double M = f_mach_rho_u_et(s, rho, u, et);
    return p * pow(1.0 + (s->gamma - 1.0) / 2.0 * M * M, s->gamma / (s->gamma - 1));
}
static double f_total_temperature_rho_u_et(const oracle_solver* s, double rho, vec3 u, double et) { /* :100-104 */
    if (s->real) { /* FluidReal :323-328 */
        double pt = lut_pt_rho_e_et(s->lut, rho, fb_static_energy_u_et(u, et), et);
        double e = fb_static_energy_u_et(u, et);
        double sv = table_interp(&s->lut->s, rho, e);
        return table_interp(&s->lut->T_ps, pt, sv);
    }
    double T = f_temperature_rho_u_et(s, rho, u, et);
    double M = f_mach_rho_u_et(s, rho, u, et);
    return T * (1.0 + (s->gamma - 1.0) / 2.0 * M * M);
}
static double f_entropy_p_T(const oracle_solver* s, double p, double T) { /* :195-198 */
    return s->cp * log(T / 288.15) - s->rgas * log(p / 101325);
}
static double f_entropy_rho_u_et(const oracle_solver* s, double rho, vec3 u, double et) { /* :128-135 */
    if (s->real) return table_interp(&s->lut->s, rho, fb_static_energy_u_et(u, et)); /* fluid_base.hpp:101-104 */
    double p = f_pressure_rho_u_et(s, rho, u, et);
    double T = f_temperature_rho_u_et(s, rho, u, et);
    return f_entropy_p_T(s, p, T);
}
static double f_efficiency(const oracle_solver* s, double pr, double tr) { /* :179-191 */
    double dT = tr - 1.0;
    double dTs = pow(pr, (s->gamma - 1.0) / s->gamma) - 1.0;
    if (fabs(dT) < 1e-12) return 1.0;
    if (dT >= 0.0) return dTs / dT;
    if (fabs(dTs) < 1e-12) return 1.0;
    return dT / dTs;
}

/* getPrimitiveVariablesFromConservative (src/math_utils.cpp:49-57). */
static sv5 prim_of(sv5 U) {
    sv5 W;
    W.v[0] = U.v[0];
    W.v[1] = U.v[1] / U.v[0];
    W.v[2] = U.v[2] / U.v[0];
    W.v[3] = U.v[3] / U.v[0];
    W.v[4] = U.v[4] / U.v[0];
    return W;
}
static vec3 vel_of(sv5 W) { return v3(W.v[1], W.v[2], W.v[3]); }
static double pressure_prim(const oracle_solver* s, sv5 W) { /* fluid_ideal.cpp:172-176 */
    return f_pressure_rho_u_et(s, W.v[0], vel_of(W), W.v[4]);
}

/* computeAdvectionFluxFromPrimitive (src/math_utils.cpp:71-86). */
static sv5 adv_flux(const oracle_solver* s, sv5 W, vec3 S) {
    vec3 n = vdiv(S, vmag(S));
    vec3 u = vel_of(W);
    double un = vdot(u, n);
    double p = f_pressure_rho_u_et(s, W.v[0], u, W.v[4]);
    double ht = f_total_enthalpy_rho_u_et(s, W.v[0], u, W.v[4]);
    sv5 F;
    F.v[0] = W.v[0] * un;
    F.v[1] = W.v[0] * un * u.x + p * n.x;
    F.v[2] = W.v[0] * un * u.y + p * n.y;
    F.v[3] = W.v[0] * un * u.z + p * n.z;
    F.v[4] = W.v[0] * un * ht;
    return F;
}

/* --------------------------------------------------------------- cylinder */
/* src/math_utils.cpp:109-138; theta rotations about the x axis. */
static vec3 rot_x(vec3 v, double th) {
    vec3 r;
    r.x = v.x;
    r.y = v.y * cos(th) - v.z * sin(th);
    r.z = v.y * sin(th) + v.z * cos(th);
    return r;
}
static sv5 rot_state(sv5 a, double th) {
    vec3 r = rot_x(v3(a.v[1], a.v[2], a.v[3]), th);
    sv5 o = {{a.v[0], r.x, r.y, r.z, a.v[4]}};
    return o;
}
static vec3 cyl_of_cart(vec3 v, double th) {
    vec3 r;
    r.x = v.x;
    r.y = v.y * cos(th) + v.z * sin(th);
    r.z = -v.y * sin(th) + v.z * cos(th);
    return r;
}
static vec3 cart_of_cyl(vec3 v, double th) {
    vec3 r;
    r.x = v.x;
    r.y = v.y * cos(th) - v.z * sin(th);
    r.z = v.y * sin(th) + v.z * cos(th);
    return r;
}
static double node_radius(const oracle_solver* s, long i, long j, long k) { /* mesh.hpp:64-66 */
    vec3 p = s->vert[idx3(s, i, j, k)];
    return sqrt(p.y * p.y + p.z * p.z);
}
static double node_theta(const oracle_solver* s, long i, long j, long k) { /* mesh.hpp:68-70 */
    vec3 p = s->vert[idx3(s, i, j, k)];
    return atan2(p.z, p.y);
}

/* ------------------------------------------------------------- advection */

/* AdvectionJst::computeFlux (src/advection_jst.cpp:4-57), constants
 * include/advection_jst.hpp:23. */
static double jst_r(const oracle_solver* s, sv5 W) {
    vec3 u = vel_of(W);
    double vm = vmag(u);
    double a = f_sound_speed_rho_u_et(s, W.v[0], u, W.v[4]);
    return vm + a;
}
static double jst_s(const oracle_solver* s, sv5 W1, sv5 W2, sv5 W3) {
    double p1 = pressure_prim(s, W1), p2 = pressure_prim(s, W2), p3 = pressure_prim(s, W3);
    return fabs((p1 - 2 * p2 + p3) / (p1 + 2 * p2 + p3));
}
static sv5 flux_jst(const oracle_solver* s, sv5 Ull, sv5 Ul, sv5 Ur, sv5 Urr, vec3 S) {
    sv5 Wll = prim_of(Ull), Wl = prim_of(Ul), Wr = prim_of(Ur), Wrr = prim_of(Urr);
    sv5 Wavg = smul(sadd(Wl, Wr), 0.5);
    double rL = jst_r(s, Wl), rR = jst_r(s, Wr);
    double sL = jst_s(s, Wll, Wl, Wr), sR = jst_s(s, Wl, Wr, Wrr);
    double r = dmax(rL, rR);
    double sf = dmax(sL, sR);
    double psi2 = 0.5 * sf * r;
    double psi4 = dmax(0.0, 0.02 * r - 2.0 * psi2);
    sv5 F = adv_flux(s, Wavg, S);
    sv5 d = ssub(smul(ssub(Ur, Ul), psi2),
                 smul(sadd(ssub(ssub(Urr, Ur), smul(ssub(Ur, Ul), 2)), ssub(Ul, Ull)), psi4));
    return ssub(F, d);
}

/* AdvectionBase MUSCL helpers (src/advection_base.cpp:10-64). */
static sv5 muscl_smooth(sv5 Wl, sv5 Wc, sv5 Wr) {
    sv5 r;
    for (int i = 0; i < 5; i++) {
        double dR = Wr.v[i] - Wc.v[i];
        double dL = Wc.v[i] - Wl.v[i];
        r.v[i] = (fabs(dR) < 1E-12) ? 0.0 : dL / dR;
    }
    return r;
}
static sv5 muscl_limiter(const oracle_solver* s, sv5 sm) {
    sv5 l = szero();
    for (int i = 0; i < 5; i++) {
        double x = sm.v[i];
        switch (s->limiter) {
            case LIM_NONE: l.v[i] = 0.0; break;
            case LIM_VAN_ALBADA: l.v[i] = (x <= 0.0) ? 0.0 : (x * x + x) / (1.0 + x * x); break;
            case LIM_VAN_LEER: l.v[i] = (x + fabs(x)) / (1.0 + fabs(x)); break;
            case LIM_MIN_MOD: l.v[i] = dmax(0.0, dmin(1.0, x)); break;
        }
    }
    return l;
}

/* AdvectionRoe (src/advection_roe.cpp:6-220, include/advection_roe.hpp:63). */
static double roe_avg(double rl, double rr, double pl, double pr) {
    return (sqrt(rl) * pl + sqrt(rr) * pr) / (sqrt(rl) + sqrt(rr));
}
static sv5 flux_roe(const oracle_solver* s, sv5 Ull, sv5 Ul, sv5 Ur, sv5 Urr, vec3 S) {
    sv5 Wl = prim_of(Ul), Wr = prim_of(Ur), Wrr = prim_of(Urr), Wll = prim_of(Ull);
    if (s->muscl) {
        sv5 smL = muscl_smooth(Wll, Wl, Wr);
        sv5 smR = muscl_smooth(Wl, Wr, Wrr);
        sv5 limL = muscl_limiter(s, smL);
        sv5 limR = muscl_limiter(s, smR);
        for (int i = 0; i < 5; i++) Wl.v[i] += limL.v[i] * (Wr.v[i] - Wl.v[i]) * 0.5;
        for (int i = 0; i < 5; i++) Wr.v[i] -= limR.v[i] * (Wrr.v[i] - Wr.v[i]) * 0.5;
    }
    /* normal triad :41-58 */
    vec3 n1 = vnormalized(S), n2;
    if (n1.x == 0 && n1.y == 0) n2 = v3(1, 0, 0);
    else n2 = v3(-n1.y, n1.x, 0);
    n2 = vnormalized(n2);
    vec3 n3 = vcross(n1, n2);
    /* rotated primitives :61-65 */
    vec3 uL = vel_of(Wl), uR = vel_of(Wr);
    sv5 L = {{Wl.v[0], vdot(uL, n1), vdot(uL, n2), vdot(uL, n3), Wl.v[4]}};
    sv5 Rr = {{Wr.v[0], vdot(uR, n1), vdot(uR, n2), vdot(uR, n3), Wr.v[4]}};
    /* Roe averages :68-143 */
    double rhoL = L.v[0], rhoR = Rr.v[0];
    double u1L = L.v[1], u1R = Rr.v[1], u2L = L.v[2], u2R = Rr.v[2], u3L = L.v[3], u3R = Rr.v[3];
    double etL = L.v[4], etR = Rr.v[4];
    double htL = f_total_enthalpy_rho_u_et(s, rhoL, v3(u1L, u2L, u3L), etL);
    double htR = f_total_enthalpy_rho_u_et(s, rhoR, v3(u1R, u2R, u3R), etR);
    double rhoA = sqrt(rhoL * rhoR);
    double u1A = roe_avg(rhoL, rhoR, u1L, u1R);
    double u2A = roe_avg(rhoL, rhoR, u2L, u2R);
    double u3A = roe_avg(rhoL, rhoR, u3L, u3R);
    double htA = roe_avg(rhoL, rhoR, htL, htR);
    double eL = etL - 0.5 * (u1L * u1L + u2L * u2L + u3L * u3L);
    double eR = etR - 0.5 * (u1R * u1R + u2R * u2R + u3R * u3R);
    double pL = f_pressure_rho_e(s, rhoL, eL);
    double pR = f_pressure_rho_e(s, rhoR, eR);
    double chiL, kapL, chiR, kapR;
    if (s->real) { /* FluidReal :410-416 */
        chiL = table_interp(&s->lut->dpdrho, rhoL, eL); kapL = table_interp(&s->lut->dpde, rhoL, eL);
        chiR = table_interp(&s->lut->dpdrho, rhoR, eR); kapR = table_interp(&s->lut->dpde, rhoR, eR);
    } else {
        chiL = (s->gamma - 1.0) * eL; kapL = (s->gamma - 1.0) * rhoL;
        chiR = (s->gamma - 1.0) * eR; kapR = (s->gamma - 1.0) * rhoR;
    }
    double barChi = 0.5 * (chiL + chiR);
    double barKap = 0.5 * (kapL + kapR);
    double barRho = 0.5 * (rhoL + rhoR);
    double barE = 0.5 * (eL + eR);
    double dP = pR - pL, dRho = rhoR - rhoL, dE = eR - eL;
    double dRhoHat = (barRho > 1e-12) ? dRho / barRho : 0.0;
    double dEHat = (fabs(barE) > 1e-12) ? dE / fabs(barE) : 0.0;
    double dNorm2 = dRhoHat * dRhoHat + dEHat * dEHat;
    double chiT = barChi, kapT = barKap;
    if (dNorm2 > 1e-12) {
        double res = dP - (barChi * dRho + barKap * dE);
        chiT += (res * dRhoHat) / (dNorm2 * barRho);
        kapT += (res * dEHat) / (dNorm2 * fabs(barE));
    }
    if (barKap > 0.0 && kapT <= 0.0) kapT = 0.01 * barKap;
    double kapP = (rhoA > 1e-12) ? kapT / rhoA : 0.4;
    double eA = roe_avg(rhoL, rhoR, eL, eR);
    double chiP = chiT - kapP * eA;
    double q2 = u1A * u1A + u2A * u2A + u3A * u3A;
    double hA = htA - 0.5 * q2;
    double a2 = chiP + kapP * hA;
    if (a2 <= 0.0) {
        double aL = f_sound_speed_rho_e(s, rhoL, eL);
        double aR = f_sound_speed_rho_e(s, rhoR, eR);
        a2 = 0.5 * (aL * aL + aR * aR);
    }
    double aA = sqrt(a2);
    /* eigenvalues / eigenvectors :146-169 */
    double lam[5] = {u1A - aA, u1A, u1A, u1A, u1A + aA};
    double cE5 = htA - (aA * aA) / kapP;
    double ev[5][5] = {
        {1.0, u1A - aA, u2A, u3A, htA - aA * u1A},
        {1.0, u1A, u2A, u3A, cE5},
        {0.0, 0.0, 1.0, 0.0, u2A},
        {0.0, 0.0, 0.0, 1.0, u3A},
        {1.0, u1A + aA, u2A, u3A, htA + aA * u1A}};
    /* wave strengths :172-185 */
    double ddRho = Rr.v[0] - L.v[0];
    double du1 = Rr.v[1] - L.v[1], du2 = Rr.v[2] - L.v[2], du3 = Rr.v[3] - L.v[3];
    double ppL = f_pressure_rho_u_et(s, L.v[0], v3(L.v[1], L.v[2], L.v[3]), L.v[4]);
    double ppR = f_pressure_rho_u_et(s, Rr.v[0], v3(Rr.v[1], Rr.v[2], Rr.v[3]), Rr.v[4]);
    double ddP = ppR - ppL;
    double ws[5];
    ws[0] = 1.0 / (2.0 * aA * aA) * (ddP - rhoA * aA * du1);
    ws[1] = ddRho - ddP / (aA * aA);
    ws[2] = rhoA * du2;
    ws[3] = rhoA * du3;
    ws[4] = 1.0 / (2.0 * aA * aA) * (ddP + rhoA * aA * du1);
    /* assembly :188-220 */
    sv5 FL = adv_flux(s, L, v3(1.0, 0.0, 0.0));
    sv5 FR = adv_flux(s, Rr, v3(1.0, 0.0, 0.0));
    double fix[5];
    for (int i = 0; i < 5; i++) fix[i] = (fabs(lam[i]) < 0.01) ? 0.01 : fabs(lam[i]);
    sv5 Fr = smul(sadd(FL, FR), 0.5);
    for (int i = 0; i < 5; i++)
        for (int j = 0; j < 5; j++) Fr.v[i] -= 0.5 * ws[j] * fix[j] * ev[j][i];
    vec3 ex = v3(1.0, 0.0, 0.0), ey = v3(0.0, 1.0, 0.0), ez = v3(0.0, 0.0, 1.0);
    sv5 F;
    F.v[0] = Fr.v[0];
    F.v[1] = Fr.v[1] * (vdot(n1, ex)) + Fr.v[2] * (vdot(n2, ex)) + Fr.v[3] * (vdot(n3, ex));
    F.v[2] = Fr.v[1] * (vdot(n1, ey)) + Fr.v[2] * (vdot(n2, ey)) + Fr.v[3] * (vdot(n3, ey));
    F.v[3] = Fr.v[1] * (vdot(n1, ez)) + Fr.v[2] * (vdot(n2, ez)) + Fr.v[3] * (vdot(n3, ez));
    F.v[4] = Fr.v[4];
    return F;
}

static sv5 flux_interior(const oracle_solver* s, sv5 Ull, sv5 Ul, sv5 Ur, sv5 Urr, vec3 S) {
    return (s->scheme == SCHEME_JST) ? flux_jst(s, Ull, Ul, Ur, Urr, S)
                                     : flux_roe(s, Ull, Ul, Ur, Urr, S);
}

/* ------------------------------------------------------------- boundaries */

/* Config::computeRampedOutletPressure (src/config.cpp:430-439). */
static double ramped_outlet_pressure(const oracle_solver* s, long it, double p_out) {
    double maxIter = s->ramp_iters;
    double ratio = (double)it / maxIter;
    if (ratio >= 1.0) return p_out;
    return s->init_p + (p_out - s->init_p) * ratio;
}

/* BoundaryBase::computeOutletFlux (src/boundary_base.cpp:181-224). */
static sv5 bc_outlet(const oracle_solver* s, sv5 Uint, vec3 S, double p_b, long it) {
    sv5 W = prim_of(Uint);
    vec3 u = vel_of(W);
    double rho = W.v[0];
    double p = f_pressure_rho_u_et(s, rho, u, W.v[4]);
    double a = f_sound_speed_p_rho(s, p, W.v[0]);
    if (vmag(u) >= a) return adv_flux(s, W, S);
    double pb = ramped_outlet_pressure(s, it, p_b);
    double rhob, eb;
    if (s->real) { /* isentropic extrapolation, src/boundary_base.cpp:206-211 */
        double eInt = W.v[4] - 0.5 * vdot(u, u);
        double sInt = table_interp(&s->lut->s, rho, eInt);
        rhob = table_interp(&s->lut->rho_ps, pb, sInt);
        eb = table_interp(&s->lut->e_ps, pb, sInt);
    } else {
        rhob = pb * rho / p;
        eb = f_static_energy_p_rho(s, pb, rhob);
    }
    double etb = eb + 0.5 * vdot(u, u);
    sv5 Wb = {{rhob, u.x, u.y, u.z, etb}};
    return adv_flux(s, Wb, S);
}

/* BoundaryInviscidWall::computeBoundaryFlux (src/boundary_inviscid_wall.cpp:5-30). */
static sv5 bc_wall(const oracle_solver* s, sv5 Uint, vec3 S) {
    sv5 W = prim_of(Uint);
    vec3 u = vel_of(W);
    double p = f_pressure_rho_u_et(s, W.v[0], u, W.v[4]);
    vec3 d = vdiv(S, vmag(S));
    double un = vdot(u, d);
    double a = f_sound_speed_p_rho(s, p, W.v[0]);
    double pw = p + W.v[0] * un * a;
    if (pw < 0.01 * p) pw = 0.01 * p;
    sv5 F = {{0.0, pw * d.x, pw * d.y, pw * d.z, 0.0}};
    return F;
}

/* BoundaryInlet::computeBoundaryFlux (src/boundary_inlet.cpp:4-43) and
 * BoundaryBase::computeSubsonicInletFlux (src/boundary_base.cpp:7-124). */
static sv5 bc_inlet(const oracle_solver* s, const patch* pt, sv5 Uint, vec3 S, long fi, long fj,
                    long fk) {
    double Pt = pt->values[0], Tt = pt->values[1];
    vec3 dir = v3(pt->values[2], pt->values[3], pt->values[4]);
    if (s->inlet_cyl) dir = cart_of_cyl(dir, node_theta(s, fi, fj, fk));
    if (dir.x == 1.0 && dir.y == 1.0 && dir.z == 1.0) dir = vneg(S);
    dir = vdiv(dir, vmag(dir));

    sv5 W = prim_of(Uint);
    vec3 u = vel_of(W);
    double aInt = f_sound_speed_rho_u_et(s, W.v[0], u, W.v[4]);
    vec3 n = vdiv(S, vmag(S));
    double unInt = vdot(u, n);
    double Z = W.v[0] * aInt;
    double pInt = f_pressure_rho_u_et(s, W.v[0], u, W.v[4]);
    double Cg = vdot(dir, n);
    if (Cg >= 0.0) Cg = -1.0;
    double Rout = pInt + Z * unInt;
    if (s->real) { /* src/boundary_base.cpp:78-111 */
        const lut* L = s->lut;
        double sIn = table_interp(&L->s_pt, Pt, Tt);
        double htIn = lut_h_p_s(L, Pt, sIn);
        double pLow = 0.05 * Pt, pHigh = 0.999999 * Pt;
        double pB = 0.5 * (pLow + pHigh);
        for (int iter = 0; iter < 30; ++iter) {
            double pMid = 0.5 * (pLow + pHigh);
            double hMid = lut_h_p_s(L, pMid, sIn);
            double VMid = sqrt(2.0 * dmax(0.0, htIn - hMid));
            double res = pMid + Z * Cg * VMid - Rout;
            if (fabs(res) < 1e-4 * Pt) { pB = pMid; break; }
            if (res < 0.0) pLow = pMid; else pHigh = pMid;
            pB = pMid;
        }
        double hB = lut_h_p_s(L, pB, sIn);
        double VB = sqrt(2.0 * dmax(0.0, htIn - hB));
        vec3 uB = vmul(dir, VB);
        double rhoB = table_interp(&L->rho_ps, pB, sIn);
        double eB = table_interp(&L->e_ps, pB, sIn);
        double etB = eB + 0.5 * vdot(uB, uB);
        sv5 Wb = {{rhoB, uB.x, uB.y, uB.z, etB}};
        return adv_flux(s, Wb, S);
    }
    double g = s->gamma, Rg = s->rgas;
    double cp = g * Rg / (g - 1.0);
    double htIn = cp * Tt;
    double pLow = 0.05 * Pt, pHigh = 0.999999 * Pt;
    double pB = 0.5 * (pLow + pHigh);
    for (int iter = 0; iter < 30; ++iter) {
        double pMid = 0.5 * (pLow + pHigh);
        double TMid = Tt * pow(pMid / Pt, (g - 1.0) / g);
        double hMid = cp * TMid;
        double VMid = sqrt(2.0 * dmax(0.0, htIn - hMid));
        double res = pMid + Z * Cg * VMid - Rout;
        if (fabs(res) < 1e-4 * Pt) { pB = pMid; break; }
        if (res < 0.0) pLow = pMid; else pHigh = pMid;
        pB = pMid;
    }
    double TB = Tt * pow(pB / Pt, (g - 1.0) / g);
    double hB = cp * TB;
    double VB = sqrt(2.0 * dmax(0.0, htIn - hB));
    vec3 uB = vmul(dir, VB);
    double rhoB = pB / (Rg * TB);
    double eB = f_static_energy_p_rho(s, pB, rhoB);
    double etB = eB + 0.5 * vdot(uB, uB);
    sv5 Wb = {{rhoB, uB.x, uB.y, uB.z, etB}};
    return adv_flux(s, Wb, S);
}

/* FluidIdeal::computeDensity_p_T (src/fluid_ideal.cpp:134-136),
 * FluidReal::computeDensity_p_T (src/fluid_real.cpp:279-281). */
static double f_density_p_T(const oracle_solver* s, double p, double T) {
    if (s->real) return table_interp(&s->lut->rho_pt, p, T);
    return p / (s->rgas * T);
}

/* BoundaryInletSupersonic::computeBoundaryFlux (src/boundary_inlet_supersonic.cpp:4-34). */
static sv5 bc_inlet_supersonic(const oracle_solver* s, const patch* pt, vec3 S) {
    double p = pt->values[0], T = pt->values[1];
    vec3 u = v3(pt->values[2], pt->values[3], pt->values[4]);
    double rho = f_density_p_T(s, p, T);
    double e = f_static_energy_p_rho(s, p, rho);
    double et = e + 0.5 * vdot(u, u);
    sv5 W = {{rho, u.x, u.y, u.z, et}};
    return adv_flux(s, W, S);
}

/* BoundaryFarfield::computeBoundaryFlux (src/boundary_farfield.cpp:5-144). */
static sv5 bc_farfield(const oracle_solver* s, const patch* pt, sv5 Uint, vec3 S) {
    double g = s->gamma;
    double machInf = pt->values[0], pInf = pt->values[1], TInf = pt->values[2];
    vec3 dir = v3(pt->values[3], pt->values[4], pt->values[5]);
    dir = vdiv(dir, vmag(dir));
    double rhoInf = f_density_p_T(s, pInf, TInf);
    double aInf = f_sound_speed_p_rho(s, pInf, rhoInf);
    vec3 uInf = vmul(dir, machInf * aInf);
    sv5 W = prim_of(Uint);
    double rhoI = W.v[0];
    vec3 uI = vel_of(W);
    double pI = f_pressure_rho_u_et(s, rhoI, uI, W.v[4]);
    double aI = f_sound_speed_p_rho(s, pI, rhoI);
    vec3 n = vdiv(S, vmag(S));
    double unI = vdot(uI, n), unInf = vdot(uInf, n);
    sv5 Wb;
    if (unI >= aI) {
        Wb = W;
    } else if (unI <= -aI) {
        double eInf = f_static_energy_p_rho(s, pInf, rhoInf);
        double etInf = eInf + 0.5 * vdot(uInf, uInf);
        sv5 t = {{rhoInf, uInf.x, uInf.y, uInf.z, etInf}};
        Wb = t;
    } else {
        double rhoB, eB, unB;
        vec3 uRef;
        if (!s->real) {
            double Rp = unI + 2.0 * aI / (g - 1.0);
            double Rm = unInf - 2.0 * aInf / (g - 1.0);
            unB = 0.5 * (Rp + Rm);
            double aB = 0.25 * (g - 1.0) * (Rp - Rm);
            double rhoRef, pRef;
            if (unB > 0.0) { rhoRef = rhoI; pRef = pI; uRef = uI; }
            else { rhoRef = rhoInf; pRef = pInf; uRef = uInf; }
            double ent = pRef / pow(rhoRef, g);
            rhoB = pow(aB * aB / (g * ent), 1.0 / (g - 1.0));
            double pB = rhoB * aB * aB / g;
            eB = f_static_energy_p_rho(s, pB, rhoB);
        } else {
            double rhoAvg = 0.5 * (rhoI + rhoInf);
            double aAvg = 0.5 * (aI + aInf);
            double Z = rhoAvg * aAvg;
            double Rp = unI + pI / Z;
            double Rm = unInf - pInf / Z;
            unB = 0.5 * (Rp + Rm);
            double pB = 0.5 * (Rp - Rm) * Z;
            double sRef;
            if (unB > 0.0) {
                double eI = W.v[4] - 0.5 * vdot(uI, uI);
                sRef = table_interp(&s->lut->s, rhoI, eI);
                uRef = uI;
            } else {
                sRef = table_interp(&s->lut->s_pt, pInf, TInf);
                uRef = uInf;
            }
            rhoB = table_interp(&s->lut->rho_ps, pB, sRef);
            eB = table_interp(&s->lut->e_ps, pB, sRef);
        }
        vec3 ut = vsub(uRef, vmul(n, vdot(uRef, n)));
        vec3 uB = vadd(ut, vmul(n, unB));
        double etB = eB + 0.5 * vdot(uB, uB);
        sv5 t = {{rhoB, uB.x, uB.y, uB.z, etB}};
        Wb = t;
    }
    return adv_flux(s, Wb, S);
}

/* BoundaryBase::isNodeOnNoSlipWall (include/boundary_base.hpp:44-49): the
 * boundary face's own indices read as node indices, so the end faces of a
 * direction (index n) never count. */
static int node_on_wall(const oracle_solver* s, long i, long j, long k) {
    if (!s->viscous || !s->wall) return 0;
    if (i >= s->ni || j >= s->nj || k >= s->nk) return 0;
    return s->wall[idx3(s, i, j, k)] != 0;
}

/* BoundaryBase::computeStagnationWallFlux (src/boundary_base.cpp:126-178) for
 * a wall at rest: the boundary pressure is the patch's first value. */
static sv5 stagnation_wall_flux(double pB, vec3 S) {
    vec3 n = vdiv(S, vmag(S));
    sv5 F = {{0.0, pB * n.x, pB * n.y, pB * n.z, 0.0}};
    return F;
}

static sv5 boundary_flux(oracle_solver* s, int pidx, sv5 Uint, vec3 S, long fi, long fj, long fk,
                         long it) {
    const patch* p = &s->patches[pidx];
    if ((p->type == BC_INLET || p->type == BC_INLET_SUPERSONIC) && node_on_wall(s, fi, fj, fk))
        return stagnation_wall_flux(p->values[0], S);
    switch (p->type) {
        case BC_INLET: return bc_inlet(s, p, Uint, S, fi, fj, fk);
        case BC_OUTLET: return bc_outlet(s, Uint, S, p->values[0], it);
        case BC_INLET_SUPERSONIC: return bc_inlet_supersonic(s, p, S);
        case BC_OUTLET_SUPERSONIC: /* src/boundary_outlet_supersonic.cpp:4-14 */
            return adv_flux(s, prim_of(Uint), S);
        case BC_FARFIELD: return bc_farfield(s, p, Uint, S);
        case BC_TRANSPARENT: /* src/boundary_transparent.cpp:5-16 */
            return flux_interior(s, Uint, Uint, Uint, Uint, S);
        case BC_MASS_FLOW: { /* src/boundary_outlet_mass_flow.cpp:4-19 */
            const radial_profile* rp = &s->profiles[p->profile];
            long idx = fj < rp->n ? fj : rp->n - 1;
            return bc_outlet(s, Uint, S, rp->pressure[idx], it);
        }
        case BC_RADIAL_EQ:
        case BC_THROTTLE: /* src/boundary_outlet_throttle.cpp:5-16, radial_equilibrium.cpp:5-16 */
            return bc_outlet(s, Uint, S, s->profiles[p->profile].pressure[fj], it);
        case BC_INVISCID_WALL:
        case BC_NO_SLIP_WALL: return bc_wall(s, Uint, S); /* src/solver.cpp:393-398 */
        default: return szero(); /* BoundaryFake (src/boundary_fake.cpp:4-13) */
    }
}

/* ------------------------------------------------------------ residuals */

/* Solver::computeAdvectionFluxResidualsImpl (src/solver.cpp:1865-2040). */
static void advection_residuals(oracle_solver* s, int dir, double* const* U, long it) {
    long nfi, nfj, nfk;
    const vec3* surf;
    const int* map;
    if (dir == 0) { nfi = s->ni + 1; nfj = s->nj; nfk = s->nk; surf = s->sI; map = s->mapI; }
    else if (dir == 1) { nfi = s->ni; nfj = s->nj + 1; nfk = s->nk; surf = s->sJ; map = s->mapJ; }
    else { nfi = s->ni; nfj = s->nj; nfk = s->nk + 1; surf = s->sK; map = s->mapK; }
    const long st[3] = {dir == 0, dir == 1, dir == 2};
    const long nface[3] = {nfi, nfj, nfk};
    const long stop = nface[dir] - 1;

    for (long a = 0; a < (dir == 0 ? nfj : nfi); a++) {
        for (long b = 0; b < (dir == 2 ? nfj : nfk); b++) {
            for (long c = 0; c < nface[dir]; c++) {
                long fi, fj, fk;
                if (dir == 0) { fj = a; fk = b; fi = c; }
                else if (dir == 1) { fi = a; fk = b; fj = c; }
                else { fi = a; fj = b; fk = c; }
                long sidx = (dir == 0) ? sIi(s, fi, fj, fk) : (dir == 1) ? sJi(s, fi, fj, fk) : sKi(s, fi, fj, fk);
                long dface = (dir == 0) ? fi : (dir == 1) ? fj : fk;
                if (dir == 2 && s->bfm_active) {
                    if (s->field[F_BLADE_PRESENT][idx3(s, fi, fj, 0)] > 0.0) continue;
                }
                if (dface == 0) {
                    sv5 Ui = state_at(s, U, fi, fj, fk);
                    vec3 S = vneg(surf[sidx]);
                    long mi = (dir == 0) ? (0 * s->nj + fj) * s->nk + fk
                            : (dir == 1) ? (fi * 2 + 0) * s->nk + fk
                                         : (fi * s->nj + fj) * 2 + 0;
                    sv5 F = boundary_flux(s, map[mi], Ui, S, fi, fj, fk, it);
                    res_add(s, fi, fj, fk, smul(F, vmag(S)));
                } else if (dface == stop) {
                    long ii = fi - st[0], jj = fj - st[1], kk = fk - st[2];
                    sv5 Ui = state_at(s, U, ii, jj, kk);
                    vec3 S = surf[sidx];
                    long mi = (dir == 0) ? (1 * s->nj + fj) * s->nk + fk
                            : (dir == 1) ? (fi * 2 + 1) * s->nk + fk
                                         : (fi * s->nj + fj) * 2 + 1;
                    sv5 F = boundary_flux(s, map[mi], Ui, S, fi, fj, fk, it);
                    res_add(s, ii, jj, kk, smul(F, vmag(S)));
                } else {
                    sv5 Ul = state_at(s, U, fi - st[0], fj - st[1], fk - st[2]);
                    sv5 Ur = state_at(s, U, fi, fj, fk);
                    sv5 Ull, Urr;
                    if (dir == 2 && s->periodic) {
                        if (dface == 1) {
                            Ull = state_at(s, U, fi, fj, nfk - 3);
                            Ull = rot_state(Ull, -s->per_angle_rad);
                            Urr = state_at(s, U, fi, fj, fk + 1);
                        } else if (dface == stop - 1) {
                            Ull = state_at(s, U, fi, fj, fk - 2);
                            Urr = state_at(s, U, fi, fj, 1);
                            Urr = rot_state(Urr, s->per_angle_rad);
                        } else {
                            Ull = state_at(s, U, fi - 2 * st[0], fj - 2 * st[1], fk - 2 * st[2]);
                            Urr = state_at(s, U, fi + st[0], fj + st[1], fk + st[2]);
                        }
                    } else {
                        if (dface == 1) {
                            Ull = ssub(Ul, ssub(Ur, Ul));
                            Urr = state_at(s, U, fi + st[0], fj + st[1], fk + st[2]);
                        } else if (dface == stop - 1) {
                            Ull = state_at(s, U, fi - 2 * st[0], fj - 2 * st[1], fk - 2 * st[2]);
                            Urr = sadd(Ur, ssub(Ur, Ul));
                        } else {
                            Ull = state_at(s, U, fi - 2 * st[0], fj - 2 * st[1], fk - 2 * st[2]);
                            Urr = state_at(s, U, fi + st[0], fj + st[1], fk + st[2]);
                        }
                    }
                    vec3 S = surf[sidx];
                    sv5 F = flux_interior(s, Ull, Ul, Ur, Urr, S);
                    res_add(s, fi - st[0], fj - st[1], fk - st[2], smul(F, vmag(S)));
                    res_sub(s, fi, fj, fk, smul(F, vmag(S)));
                }
            }
        }
    }
}

/* Solver::getRotationalSpeedScalingFactor (src/config.cpp:695-718). */
static double speed_scaling(const oracle_solver* s, double t) {
    if (!s->accel) return s->speed_scale;
    if (t < s->acc_t0 || t > s->acc_t1) return s->speed_scale;
    return s->acc_s0 + (s->acc_s1 - s->acc_s0) * (t - s->acc_t0) / (s->acc_t1 - s->acc_t0);
}

/* Solver::computeGongSource (src/solver.cpp:3074-3145). */
static sv5 gong_source(const oracle_solver* s, double* const* U, double omega, long i, long j,
                       long k, double vol) {
    if (fabs(omega) < 1E-3) return szero();
    sv5 U0, U1, U2;
    long nk = s->nk;
    if (omega > 0) {
        if (k == 0) { U0 = state_at(s, U, i, j, k); U1 = state_at(s, U, i, j, nk - 2); U2 = state_at(s, U, i, j, nk - 3); }
        else if (k == 1) { U0 = state_at(s, U, i, j, k); U1 = state_at(s, U, i, j, 0); U2 = state_at(s, U, i, j, nk - 2); }
        else { U0 = state_at(s, U, i, j, k); U1 = state_at(s, U, i, j, k - 1); U2 = state_at(s, U, i, j, k - 2); }
    } else {
        if (k == nk - 1) { U0 = state_at(s, U, i, j, 0); U1 = state_at(s, U, i, j, 1); U2 = state_at(s, U, i, j, 2); }
        else if (k == nk - 2) { U0 = state_at(s, U, i, j, k); U1 = state_at(s, U, i, j, 0); U2 = state_at(s, U, i, j, 1); }
        else { U0 = state_at(s, U, i, j, k); U1 = state_at(s, U, i, j, k + 1); U2 = state_at(s, U, i, j, k + 2); }
    }
    double dth = (2 * M_PI / (double)(nk - 1));
    sv5 d;
    if (omega > 0.0) d = sdiv(sadd(ssub(smul(U0, 3.0), smul(U1, 4.0)), U2), 2 * dth);
    else d = sdiv(ssub(sadd(smul(U0, -3.0), smul(U1, 4.0)), U2), 2 * dth);
    sv5 src;
    for (int c = 0; c < 5; c++) src.v[c] = -d.v[c] * omega;
    return smul(src, vol);
}

/* SourceBFMBase flow state (src/source_bfm_base.cpp:104-199). */
typedef struct {
    double radius, theta, omega, pitch, staggered, nblades, blockage, flow_angle, dev;
    vec3 velCyl, relCyl, relCart, nCyl, invDirCyl, viscDirCyl;
} bfm_state;

static double bfm_deviation(vec3 rel, vec3 ncam) { /* :152-166 */
    vec3 n = vdiv(ncam, vmag(ncam));
    vec3 vm = v3(rel.x, rel.y, 0.0);
    vec3 span = v3(-vm.y, vm.x, 0.0);
    span = vdiv(span, vmag(span));
    vec3 vin = vsub(rel, vmul(span, vdot(rel, span)));
    double nv = vdot(vin, n);
    return -asin(nv / vmag(vin));
}

static vec3 bfm_inviscid_dir(const oracle_solver* s, vec3 rel, vec3 ncam, double dev, long q) { /* :168-199 */
    vec3 rd = vnormalized(rel);
    vec3 nd = vnormalized(ncam);
    vec3 ver;
    if (s->stalled && dev > s->field[F_DEV_STALL][q]) ver = nd;
    else ver = vnormalized(vsub(nd, vmul(rd, vdot(nd, rd))));
    vec3 vm = v3(rel.x, rel.y, 0.0);
    vec3 sd = vnormalized(v3(vm.y, -vm.x, 0.0));
    return vnormalized(vsub(ver, vmul(sd, vdot(ver, sd))));
}

static void bfm_flow_state(const oracle_solver* s, long i, long j, long k, sv5 W, double t,
                           bfm_state* b) {
    long q = idx3(s, i, j, k);
    b->radius = node_radius(s, i, j, k);
    b->theta = node_theta(s, i, j, k);
    vec3 vc = vel_of(W);
    b->velCyl = cyl_of_cart(vc, b->theta);
    b->omega = s->field[F_RPM][q] * 2 * M_PI / 60;
    b->omega *= speed_scaling(s, t);
    vec3 drag = v3(0, 0, b->omega * b->radius);
    b->relCyl = vsub(b->velCyl, drag);
    b->relCart = cart_of_cyl(b->relCyl, b->theta);
    double vmer = sqrt(b->velCyl.x * b->velCyl.x + b->velCyl.y * b->velCyl.y);
    b->nblades = s->field[F_NBLADES][q];
    b->pitch = 2.0 * M_PI * b->radius / b->nblades;
    b->nCyl = v3(s->field[F_NAX][q], s->field[F_NRAD][q], s->field[F_NTAN][q]);
    b->blockage = s->field[F_BLOCKAGE][q];
    double metal = s->field[F_METAL] ? s->field[F_METAL][q] : 0.0;
    b->staggered = b->pitch * cos(metal);
    b->flow_angle = atan2(b->relCyl.z, vmer);
    b->dev = bfm_deviation(b->relCyl, b->nCyl);
    b->invDirCyl = bfm_inviscid_dir(s, b->relCyl, b->nCyl, b->dev, q);
    b->viscDirCyl = vneg(vnormalized(b->relCyl));
}

static sv5 force_source(vec3 fcyl, const bfm_state* b, double vol, double rho) {
    vec3 fc = cart_of_cyl(fcyl, b->theta);
    sv5 src = {{0, fc.x, fc.y, fc.z, fcyl.z * b->omega * b->radius}};
    return smul(smul(src, vol), rho);
}

/* SourceBFMThollet::computeCompressibilityCorrection (src/source_bfm_thollet.cpp:48-70). */
static double thollet_kmach(const oracle_solver* s, vec3 rel, sv5 W) {
    double a = f_sound_speed_rho_u_et(s, W.v[0], vel_of(W), W.v[4]);
    double M = vmag(rel) / a;
    if (fabs(M - 1.0) < 1E-03) M = 0.999;
    double kp;
    if (M < 1.0) kp = 1.0 / sqrt(1.0 - M * M);
    else kp = 2.0 / M_PI / sqrt(M * M - 1.0);
    return dmin(3.0, kp);
}

/* InputTable::readCsvFile (src/input_table.cpp:14-55) for the Chima scaling
 * functions: a header line of field names, then rows of values appended
 * column by column; the MassFlow, PhiTurn and PhiLoss columns. */
static int read_chima_table(oracle_solver* s, const char* path) {
    FILE* f = fopen(path, "r");
    if (!f) return fail("Error opening file: %s", path);
    char* line = NULL;
    size_t cap = 0;
    char names[64][64];
    int nh = 0;
    if (getline(&line, &cap, f) >= 0) {
        size_t L = strlen(line);
        if (L && line[L - 1] == '\n') line[--L] = 0;
        char* p = line;
        while (nh < 64) {
            char* c = strchr(p, ',');
            if (c) *c = 0;
            snprintf(names[nh++], 64, "%s", p);
            if (!c) break;
            p = c + 1;
        }
    }
    int im = -1, it = -1, il = -1;
    for (int h = 0; h < nh; h++) {
        if (!strcmp(names[h], "MassFlow")) im = h;
        if (!strcmp(names[h], "PhiTurn")) it = h;
        if (!strcmp(names[h], "PhiLoss")) il = h;
    }
    if (im < 0 || it < 0 || il < 0) { free(line); fclose(f); return fail("Chima scaling functions file %s lacks a column", path); }
    int cap_rows = 16;
    s->chima_mf = (double*)malloc(cap_rows * sizeof(double));
    s->chima_turn = (double*)malloc(cap_rows * sizeof(double));
    s->chima_loss = (double*)malloc(cap_rows * sizeof(double));
    s->chima_n = 0;
    while (getline(&line, &cap, f) >= 0) {
        double v[64];
        int nv = 0;
        char* save = NULL;
        for (char* t = strtok_r(line, ",\n", &save); t && nv < 64; t = strtok_r(NULL, ",\n", &save)) v[nv++] = strtod(t, NULL);
        if (nv <= im || nv <= it || nv <= il) continue;
        if (s->chima_n == cap_rows) {
            cap_rows *= 2;
            s->chima_mf = (double*)realloc(s->chima_mf, cap_rows * sizeof(double));
            s->chima_turn = (double*)realloc(s->chima_turn, cap_rows * sizeof(double));
            s->chima_loss = (double*)realloc(s->chima_loss, cap_rows * sizeof(double));
        }
        s->chima_mf[s->chima_n] = v[im];
        s->chima_turn[s->chima_n] = v[it];
        s->chima_loss[s->chima_n] = v[il];
        s->chima_n++;
    }
    free(line);
    fclose(f);
    if (s->chima_n == 0) return fail("Chima scaling functions file %s has no data rows", path);
    return 0;
}

/* SourceBFMCorrelations::computeCorrelationParameters and
 * computeInviscidComponent (src/source_bfm_correlations.cpp:33-210); the
 * viscous component is zero (:213-236). */
static sv5 correlations_force(const oracle_solver* s, double* const* U, long j, long k, long q, sv5 W,
                              const bfm_state* b, double vol) {
    long qle = idx3(s, s->le_idx, j, k), qte = idx3(s, s->te_idx, j, k);
    const double* stwl = s->field[F_STWL];
    const double* metal = s->field[F_METAL];
    double sol = (stwl[qte] - stwl[qle]) / b->pitch;
    sv5 Wi = prim_of(state_at(s, U, s->le_idx, j, k)), Wo = prim_of(state_at(s, U, s->te_idx, j, k));
    vec3 vic = cyl_of_cart(vel_of(Wi), b->theta), voc = cyl_of_cart(vel_of(Wo), b->theta);
    double rIn = node_radius(s, s->le_idx, j, k), rOut = node_radius(s, s->te_idx, j, k);
    vec3 relIn = vsub(vic, v3(0.0, 0.0, b->omega * rIn));
    vec3 relOut = vsub(voc, v3(0.0, 0.0, b->omega * rOut));
    double vmIn = sqrt(relIn.x * relIn.x + relIn.y * relIn.y);
    double flowInDeg = atan2(relIn.z, vmIn) * 180.0 / M_PI;
    double chordM = stwl[qte] - stwl[qle];
    double camberAbs = fabs(metal[qte] - metal[qle]) * 180 / M_PI;
    double k1 = metal[qle] * 180 / M_PI, k2 = metal[qte] * 180 / M_PI;
    double inc = flowInDeg - k1;
    double aAbs = fabs(flowInDeg);
    double n = 0.025 * sol - 0.06 - (pow(aAbs / 90.0, 1.0 + 1.2 * sol)) / (1.5 + 0.43 * sol);
    double p = 0.914 + sol * sol * sol / 160.0;
    double i0 = pow(aAbs, p) / (5.0 + 46.0 * exp(-2.3 * sol)) - 0.1 * pow(sol, 3.0) * exp((aAbs - 70.0) / 4.0);
    double thk = 0.0;
    for (long st = s->le_idx; st <= s->te_idx; ++st) {
        double r = node_radius(s, st, j, k);
        double pitch = 2.0 * M_PI * r / b->nblades;
        double t = pitch * (1.0 - s->field[F_BLOCKAGE][idx3(s, st, j, k)]);
        if (t > thk) thk = t;
    }
    double tc = thk / chordM;
    double Kti = pow(10.0 * tc, 0.28 / (0.1 + pow(tc, 0.3)));
    double Ksh = 0.8;
    double istar = Ksh * Kti * i0 + n * camberAbs;
    double a = f_sound_speed_rho_u_et(s, W.v[0], vel_of(W), W.v[4]);
    double mach = vmag(b->relCart) / a;
    double istarC = istar + 1.3026 * mach + 5.7380;
    double dev10 = 0.01 * sol * aAbs + (0.74 * pow(sol, 1.9) + 3.0 * sol) * pow(aAbs / 90.0, 1.67 + 1.09 * sol);
    double Ktd = 6.25 * tc + 37.5 * tc * tc;
    double ac = 0.3;
    double devStar = (0.92 * ac * ac + 0.002 * fabs(k2)) / (1 - 0.002 * camberAbs / sqrt(sol)) * camberAbs / sqrt(sol) +
                     (Ksh * Ktd - 1.0) * dev10;
    double devStarC = -1.099379 + 3.0186 * devStar - 0.1988 * devStar * devStar;
    double ddi = (1.0 + (sol + 0.25 * pow(sol, 4.0)) * pow((aAbs / 53.0), 2.5)) / exp(3.1 * sol);
    double umIn = sqrt(relIn.x * relIn.x + relIn.y * relIn.y);
    double umOut = sqrt(relOut.x * relOut.x + relOut.y * relOut.y);
    double incMag = b->omega > 0.0 ? inc * (-1.0) : inc;
    double devOut = devStarC + ddi * (incMag - istarC) + 10.0 * (1.0 - umOut / umIn);
    double loc = (stwl[q] - stwl[qle]) / (stwl[qte] - stwl[qle]);
    double devExpDeg = incMag + loc * (devOut - incMag);
    double devExp = devExpDeg * M_PI / 180.0;
    double uth = b->relCyl.z, kappa = metal[q];
    double vmer = sqrt(b->velCyl.x * b->velCyl.x + b->velCyl.y * b->velCyl.y);
    double Wn;
    if (b->omega > 0.0) Wn = vmer * tan(-devExp + kappa) - uth;
    else Wn = -(vmer * tan(devExp + kappa)) + uth;
    double fn = s->kn * vmer * Wn / (b->pitch * fabs(cos(metal[q])));
    vec3 dirCart = cart_of_cyl(b->invDirCyl, b->theta);
    vec3 fc = vmul(dirCart, fn), fy = vmul(b->invDirCyl, fn);
    sv5 inv = {{0.0, fc.x, fc.y, fc.z, fy.z * b->omega * b->radius}};
    sv5 visc = {{0.0, 0.0, 0.0, 0.0, 0.0 * b->omega * b->radius}};
    return sadd(smul(smul(inv, vol), W.v[0]), smul(smul(visc, vol), W.v[0]));
}

/* linearInterpolation (src/math_utils.cpp:487-514). */
static double linear_interp(const double* x, const double* y, int n, double xp) {
    if (xp <= x[0]) return y[0];
    if (xp >= x[n - 1]) return y[n - 1];
    int i = 0;
    while (i + 1 < n && x[i + 1] <= xp) i++;
    double t = (xp - x[i]) / (x[i + 1] - x[i]);
    return (1.0 - t) * y[i] + t * y[i + 1];
}

/* SourceBFMChima::computeDerivativeFunction (src/source_bfm_chima.cpp:180-190). */
static double chima_derivative(double yF, double xL, double xF) {
    return -2.0 * yF * xL / (xF * xF) + 2.0 * yF / xF;
}

static sv5 bfm_body_force(const oracle_solver* s, double* const* U, long i, long j, long k, sv5 W, double t) {
    long q = idx3(s, i, j, k);
    bfm_state b;
    bfm_flow_state(s, i, j, k, W, t, &b);
    double vol = s->vol[q];
    double w2 = vdot(b.relCyl, b.relCyl);
    if (s->bfm_model == BFM_CORRELATIONS) return correlations_force(s, U, j, k, q, W, &b, vol);
    if (s->bfm_model == BFM_CHIMA) { /* src/source_bfm_chima.cpp:16-190 */
        double mf = s->turbo[0];
        double scTurn = linear_interp(s->chima_mf, s->chima_turn, s->chima_n, mf);
        double scLoss = linear_interp(s->chima_mf, s->chima_loss, s->chima_n, mf);
        double sLoc = s->field[F_STWL][q];
        double sTe = s->field[F_STWL][idx3(s, s->te_idx, j, k)];
        double dSdM = chima_derivative(s->field[F_DENTROPY][q], sLoc, sTe);
        dSdM *= scLoss;
        double T = f_temperature_rho_u_et(s, W.v[0], vel_of(W), W.v[4]);
        double vmer = sqrt(b.velCyl.x * b.velCyl.x + b.velCyl.y * b.velCyl.y);
        double fv = T * vmer / vmag(b.relCyl) * dSdM;
        vec3 fvCyl = vmul(b.viscDirCyl, fv);
        sv5 visc = force_source(fvCyl, &b, vol, W.v[0]);
        double dLdM = chima_derivative(s->field[F_DANGMOM][q], sLoc, sTe);
        dLdM *= scTurn;
        double ftan = dLdM * vmer / b.radius;
        double fi = (ftan - fvCyl.z) / b.invDirCyl.z;
        sv5 inv = force_source(vmul(b.invDirCyl, fi), &b, vol, W.v[0]);
        return sadd(inv, visc);
    }
    if (s->bfm_model == BFM_HALL) { /* src/source_bfm_hall.cpp:3-34 */
        double fm = w2 * M_PI * b.dev / b.pitch / fabs(b.nCyl.z);
        return force_source(vmul(b.invDirCyl, fm), &b, vol, W.v[0]);
    }
    if (s->bfm_model == BFM_THOLLET) { /* src/source_bfm_thollet.cpp:3-138 */
        double km = thollet_kmach(s, b.relCyl, W);
        double fm = s->kn * km * w2 * M_PI * b.dev / b.pitch / fabs(b.nCyl.z) / b.blockage;
        sv5 inv = force_source(vmul(b.invDirCyl, fm), &b, vol, W.v[0]);
        sv5 visc;
        if (s->stalled && b.dev > s->field[F_DEV_STALL][q]) {
            visc = szero();
        } else {
            double nu = s->nu;
            double stwl = s->field[F_STWL][q];
            if (stwl < 1E-06) {
                if (i + 1 < s->ni) stwl = (s->field[F_STWL][idx3(s, i + 1, j, k)] + s->field[F_STWL][q]) / 2.0;
                if (stwl < 1E-06) stwl = 1E-06;
            }
            double rex = vmag(b.relCyl) * stwl / nu;
            double cf = 0.0592 * pow(rex, -0.2);
            double fmv;
            if (!s->offdesign) {
                fmv = w2 / (b.pitch * b.blockage * fabs(b.nCyl.z)) * (s->kf * cf);
            } else {
                double piv = s->field[F_DEV_PIVOT][q];
                double km2 = thollet_kmach(s, b.relCyl, W);
                fmv = w2 / (b.pitch * b.blockage * fabs(b.nCyl.z)) *
                      (s->kf * cf + M_PI * km2 * pow(fabs(b.dev - piv), 2.0 * s->kd));
            }
            visc = force_source(vmul(b.viscDirCyl, fmv), &b, vol, W.v[0]);
        }
        return sadd(inv, visc);
    }
    if (s->bfm_model == BFM_LIFT_DRAG) { /* src/source_bfm_lift_drag.cpp:3-88 */
        double chord = s->field[F_STWL][idx3(s, s->te_idx, j, k)] - s->field[F_STWL][idx3(s, s->le_idx, j, k)];
        double sol = chord / b.pitch;
        double w = vmag(b.relCart);
        double beta0 = s->field[F_LD_BETA0][q];
        double sgn = (b.nCyl.z >= 0.0) ? 1.0 : -1.0;
        double fm = 0.5 * w * w * 2.0 * M_PI / b.staggered * sgn * (-b.flow_angle + beta0);
        sv5 inv = force_source(vmul(b.invDirCyl, fm), &b, vol, W.v[0]);
        double kp0 = s->field[F_LD_KP][q];
        double d = b.flow_angle - beta0;
        double kp = kp0 + 2.0 * M_PI * sol * (d * d);
        double fmv = kp * w * w / b.staggered;
        sv5 visc = force_source(vmul(b.viscDirCyl, fmv), &b, vol, W.v[0]);
        return sadd(inv, visc);
    }
    return szero();
}

/* SourceBFMBase::computePerturbationFactor (src/source_bfm_base.cpp:215-243). */
static double bfm_perturbation(const oracle_solver* s, long i, long j, long k, double t) {
    if (!s->perturb) return 0.0;
    if (t < s->pert_t0 || t > s->pert_t0 + s->pert_dur) return 0.0;
    vec3 p = s->vert[idx3(s, i, j, k)];
    double dist = vmag(vsub(p, v3(s->pert_center[0], s->pert_center[1], s->pert_center[2])));
    if (dist > 3.0 * s->pert_radius) return 0.0;
    double sm = exp(-(dist * dist) / (s->pert_radius * s->pert_radius));
    double peak = s->pert_t0 + s->pert_dur / 2.0;
    double sig = s->pert_dur / 3.0;
    double dtp = t - peak;
    double tm = exp(-(dtp * dtp) / (sig * sig));
    return s->pert_scale * sm * tm;
}

/* SourceBFMBase::computeTotalSource (src/source_bfm_base.cpp:25-84). */
static sv5 bfm_total_source(const oracle_solver* s, double* const* U, long i, long j, long k, sv5 W, double t) {
    long q = idx3(s, i, j, k);
    sv5 blk = szero();
    if (s->blockage_active) {
        vec3 u = vel_of(W);
        double ht = f_total_enthalpy_rho_u_et(s, W.v[0], u, W.v[4]);
        double bb = s->field[F_BLOCKAGE][q];
        vec3 gb = s->gradb[q];
        double vol = s->vol[q];
        double ct = -1.0 / bb * W.v[0] * vdot(u, gb);
        sv5 src = {{ct, ct * u.x, ct * u.y, ct * u.z, ct * ht}};
        blk = smul(src, vol);
    }
    if (s->field[F_NBLADES][q] == 0) return blk;
    sv5 bf = bfm_body_force(s, U, i, j, k, W, t);
    double pf = bfm_perturbation(s, i, j, k, t);
    return sadd(blk, smul(bf, 1.0 + pf));
}

/* Solver::computeSourceResiduals (src/solver.cpp:2790-2924). */
static void source_residuals(oracle_solver* s, double* const* U) {
    if (s->topology == TOPO_3D && !s->bfm_active) return;
    for (long i = 0; i < s->ni; i++)
        for (long j = 0; j < s->nj; j++)
            for (long k = 0; k < s->nk; k++) {
                long q = idx3(s, i, j, k);
                sv5 W = prim_of(state_at(s, U, i, j, k));
                double vol = s->vol[q];
                double p = f_pressure_rho_u_et(s, W.v[0], vel_of(W), W.v[4]);
                double r = node_radius(s, i, j, k);
                double th = node_theta(s, i, j, k);
                int geo = 0, gong = 0;
                if (s->topology == TOPO_3D && s->bfm_active) {
                    geo = gong = (s->field[F_BLADE_PRESENT][q] > 0.0);
                } else if (s->topology == TOPO_AXI) {
                    geo = 1;
                }
                if (geo) {
                    vec3 vc = cyl_of_cart(vel_of(W), th);
                    vec3 sc, sCart;
                    if (s->topology == TOPO_AXI) {
                        double aK = vmag(s->sK[sKi(s, i, j, 0)]);
                        double gf = aK * s->wedge;
                        sc.x = 0.0;
                        sc.y = (+W.v[0] * vc.z * vc.z + p) * gf;
                        sc.z = -W.v[0] * vc.y * vc.z * gf;
                        sCart = cart_of_cyl(sc, th);
                        sv5 g = {{0.0, sCart.x, sCart.y, sCart.z, 0.0}};
                        res_sub(s, i, j, k, g);
                    } else {
                        sc.x = 0.0;
                        sc.y = (+W.v[0] * vc.z * vc.z + p) / r;
                        sc.z = -W.v[0] * vc.y * vc.z / r;
                        sCart = cart_of_cyl(sc, th);
                        sv5 g = {{0.0, sCart.x, sCart.y, sCart.z, 0.0}};
                        res_sub(s, i, j, k, smul(g, vol));
                    }
                }
                if (gong) {
                    double om = s->field[F_RPM][q] * 2 * M_PI / 60;
                    om *= speed_scaling(s, s->t);
                    res_sub(s, i, j, k, gong_source(s, U, om, i, j, k, vol));
                }
                if (s->bfm_active) {
                    if (vmag(s->gradb[q]) > 1E-10) res_sub(s, i, j, k, bfm_total_source(s, U, i, j, k, W, s->t));
                }
            }
}

/* Solver::enforcePeriodicityOnResiduals (src/solver.cpp:1836-1853). */
static void periodic_residuals(oracle_solver* s) {
    for (long i = 0; i < s->ni; i++)
        for (long j = 0; j < s->nj; j++) {
            sv5 R1 = state_at(s, s->R, i, j, 0);
            sv5 R2 = state_at(s, s->R, i, j, s->nk - 1);
            sv5 R2f = rot_state(R2, -s->per_angle_rad);
            sv5 Ra = smul(sadd(R1, R2f), 0.5);
            state_set(s, s->R, i, j, 0, Ra);
            state_set(s, s->R, i, j, s->nk - 1, rot_state(Ra, +s->per_angle_rad));
        }
}

/* ------------------------------------------------------- viscous path */

/* FluidIdeal::computeMolecularDynamicViscosity (src/fluid_ideal.cpp:224-231);
 * FluidReal's (src/fluid_real.cpp:387-393) is a constant in both models. */
static double f_mu(const oracle_solver* s, double T) {
    if (s->visc_const) return s->mu_const;
    return s->suth_mu * pow(T / s->suth_T, 1.5) * ((s->suth_T + s->suth_S) / (T + s->suth_S));
}

/* SA constants (include/turbulence_model_sa.hpp:80-93). */
static const double SA_CB1 = 0.1355, SA_CB2 = 0.622, SA_SIGMA = 2.0 / 3.0, SA_KAPPA = 0.41, SA_CW2 = 0.3,
                    SA_CW3 = 2.0, SA_CV1 = 7.1, SA_CT3 = 0.0, SA_CT4 = 0.5, SA_CN1 = 16.0, SA_C2 = 0.7, SA_C3 = 0.9;
static double sa_cw1(void) { return SA_CB1 / (SA_KAPPA * SA_KAPPA) + (1.0 + SA_CB2) / SA_SIGMA; }

/* TurbulenceModelSA::getEddyViscosity (src/turbulence_model_sa.cpp:843-858),
 * with the laminar viscosity of the model's last solve (0 before the first:
 * no eddy viscosity). TurbulenceModelNone's is 0. */
static double sa_mut(const oracle_solver* s, double rho, long q) {
    if (!s->sa) return 0.0;
    double nuHat = s->nuhat[q];
    if (nuHat <= 0.0) return 0.0;
    double nuL = s->nul[q];
    if (nuL <= 0.0) return 0.0;
    double chi = nuHat / nuL;
    double chi3 = chi * chi * chi;
    double cv1_3 = SA_CV1 * SA_CV1 * SA_CV1;
    double fv1 = chi3 / (chi3 + cv1_3);
    return fv1 * rho * nuHat;
}

/* Solver::computeSolutionGradient (src/solver.cpp:3033-3058): node
 * temperature of FluidIdeal::computeTemperature_conservative
 * (src/fluid_ideal.cpp:198-207) or FluidBase's (include/fluid_base.hpp:163-177),
 * then computeGradientsGreenGauss4 (src/math_utils.cpp:237-392): face values
 * interpolated by the distances of the face centre to the two nodes, the
 * node value on boundary faces, summed W, E, N, S, B, T and scaled by 1/V. */
static void solution_gradient(oracle_solver* s, double* const* U) {
    if (!s->viscous) return;
    for (long q = 0; q < s->n; q++) {
        double rho = U[0][q];
        double ux = U[1][q] / rho, uy = U[2][q] / rho, uz = U[3][q] / rho, et = U[4][q] / rho;
        double T;
        if (s->real) {
            double e = et - 0.5 * (ux * ux + uy * uy + uz * uz);
            T = table_interp(&s->lut->T, rho, e);
        } else {
            T = (et - (ux * ux + uy * uy + uz * uz) * 0.5) * ((s->gamma - 1.0) / s->rgas);
        }
        s->gfield[0][q] = ux;
        s->gfield[1][q] = uy;
        s->gfield[2][q] = uz;
        s->gfield[3][q] = T;
    }
    for (long i = 0; i < s->ni; i++)
        for (long j = 0; j < s->nj; j++)
            for (long k = 0; k < s->nk; k++) {
                long q = idx3(s, i, j, k);
                vec3 p0 = s->vert[q];
                long nb[6];
                vec3 mid[6];
                int has[6];
                has[0] = i > 0;          nb[0] = has[0] ? idx3(s, i - 1, j, k) : q; mid[0] = s->cI[sIi(s, i, j, k)];
                has[1] = i < s->ni - 1;  nb[1] = has[1] ? idx3(s, i + 1, j, k) : q; mid[1] = has[1] ? s->cI[sIi(s, i + 1, j, k)] : p0;
                has[2] = j < s->nj - 1;  nb[2] = has[2] ? idx3(s, i, j + 1, k) : q; mid[2] = has[2] ? s->cJ[sJi(s, i, j + 1, k)] : p0;
                has[3] = j > 0;          nb[3] = has[3] ? idx3(s, i, j - 1, k) : q; mid[3] = s->cJ[sJi(s, i, j, k)];
                has[4] = k > 0;          nb[4] = has[4] ? idx3(s, i, j, k - 1) : q; mid[4] = s->cK[sKi(s, i, j, k)];
                has[5] = k < s->nk - 1;  nb[5] = has[5] ? idx3(s, i, j, k + 1) : q; mid[5] = has[5] ? s->cK[sKi(s, i, j, k + 1)] : p0;
                vec3 sf[6] = {vneg(s->sI[sIi(s, i, j, k)]), s->sI[sIi(s, i + 1, j, k)], s->sJ[sJi(s, i, j + 1, k)],
                              vneg(s->sJ[sJi(s, i, j, k)]), vneg(s->sK[sKi(s, i, j, k)]), s->sK[sKi(s, i, j, k + 1)]};
                for (int v = 0; v < 4; v++) {
                    double fc = s->gfield[v][q];
                    vec3 g = v3(0.0, 0.0, 0.0);
                    for (int f = 0; f < 6; f++) {
                        double sv = fc;
                        if (has[f]) {
                            double d0 = vmag(vsub(mid[f], p0));
                            double d1 = vmag(vsub(mid[f], s->vert[nb[f]]));
                            double w = d0 / (d0 + d1);
                            sv = fc + (s->gfield[v][nb[f]] - fc) * w;
                        }
                        g = vadd(g, vmul(sf[f], sv));
                    }
                    double inv = 1.0 / s->vol[q];
                    s->grad[v][q] = vmul(g, inv);
                }
            }
}

/* Solver::computeViscousFlux (src/solver.cpp:2174-2226) with
 * computeViscousStressTensor (src/math_utils.cpp:593-608); the eddy
 * conductivity is mu_t cp / Pr_t with SA (getEddyThermalConductivity,
 * include/turbulence_model_sa.hpp:73) and 0 with TurbulenceModelNone. */
static sv5 viscous_flux(const oracle_solver* s, sv5 Uc, vec3 gu, vec3 gv, vec3 gw, vec3 gT, vec3 S,
                        double muEddy) {
    sv5 W = prim_of(Uc);
    vec3 vel = vel_of(W);
    double T = f_temperature_rho_u_et(s, W.v[0], vel, W.v[4]);
    double muL = f_mu(s, T);
    double kappaL = s->vcp * muL / s->vpr;
    double kappaEddy = s->sa ? muEddy * s->vcp / s->sa_prt : 0.0;
    double muT = muL + muEddy;
    double kT = kappaL + kappaEddy;
    double lam = -2.0 / 3.0 * muT;
    double xx = lam * (gu.x + gv.y + gw.z) + 2.0 * muT * gu.x;
    double yy = lam * (gu.x + gv.y + gw.z) + 2.0 * muT * gv.y;
    double zz = lam * (gu.x + gv.y + gw.z) + 2.0 * muT * gw.z;
    double xy = muT * (gu.y + gv.x);
    double xz = muT * (gu.z + gw.x);
    double yz = muT * (gv.z + gw.y);
    vec3 tX = v3(xx, xy, xz), tY = v3(xy, yy, yz), tZ = v3(xz, yz, zz);
    double thX = vdot(tX, vel) + kT * gT.x;
    double thY = vdot(tY, vel) + kT * gT.y;
    double thZ = vdot(tZ, vel) + kT * gT.z;
    vec3 n = vdiv(S, vmag(S));
    sv5 F = {{0.0, vdot(tX, n), vdot(tY, n), vdot(tZ, n), thX * n.x + thY * n.y + thZ * n.z}};
    return F;
}

/* Solver::computeViscousFluxResiduals (src/solver.cpp:2060-2171): interior
 * faces only, states and gradients averaged over the two nodes. */
static void viscous_residuals(oracle_solver* s, int dir, double* const* U) {
    long nf[3] = {s->ni, s->nj, s->nk};
    nf[dir] += 1;
    const vec3* surf = dir == 0 ? s->sI : (dir == 1 ? s->sJ : s->sK);
    const long st[3] = {dir == 0, dir == 1, dir == 2};
    for (long fi = 0; fi < nf[0]; fi++)
        for (long fj = 0; fj < nf[1]; fj++)
            for (long fk = 0; fk < nf[2]; fk++) {
                long dface = dir == 0 ? fi : (dir == 1 ? fj : fk);
                if (dface == 0 || dface == nf[dir] - 1) continue;
                long ql = idx3(s, fi - st[0], fj - st[1], fk - st[2]);
                long qr = idx3(s, fi, fj, fk);
                vec3 S = surf[dir == 0 ? sIi(s, fi, fj, fk) : (dir == 1 ? sJi(s, fi, fj, fk) : sKi(s, fi, fj, fk))];
                sv5 Ua = smul(sadd(state_at(s, U, fi - st[0], fj - st[1], fk - st[2]), state_at(s, U, fi, fj, fk)), 0.5);
                vec3 g[4];
                for (int v = 0; v < 4; v++) g[v] = vmul(vadd(s->grad[v][ql], s->grad[v][qr]), 0.5);
                double muEddy = (sa_mut(s, U[0][ql], ql) + sa_mut(s, U[0][qr], qr)) * 0.5;
                sv5 F = viscous_flux(s, Ua, g[0], g[1], g[2], g[3], S, muEddy);
                sv5 c = smul(smul(F, vmag(S)), -1.0);
                res_add(s, fi - st[0], fj - st[1], fk - st[2], c);
                res_sub(s, fi, fj, fk, c);
            }
}

/* Solver::setMomentumSolutionOnViscousWalls (src/solver.cpp:3147-3186) for a
 * wall at rest: the momentum of every wall node becomes density * 0, on the
 * state (preprocessSolution, :3189-3203) and on the residuals
 * (enforceNoSlipWallsOnResiduals, :1856-1863). */
static void no_slip_momentum(const oracle_solver* s, double* const* X) {
    if (!s->viscous) return;
    for (long q = 0; q < s->n; q++)
        if (s->wall[q])
            for (int c = 1; c <= 3; c++) X[c][q] = X[0][q] * 0.0;
}

/* ------------------------------------------------------ Spalart-Allmaras */
/* fetchBoundaryNodesIndexRange (src/boundary_base.cpp:227-267) and
 * Boundary::computeOrientation (include/boundary_base.hpp:109-119): the
 * patch's node range [r0, r1) x [r2, r3) x [r4, r5) and the step from a
 * boundary node to its interior donor. */
static void patch_nodes(const oracle_solver* s, const patch* p, long r[6], long step[3]) {
    r[0] = p->i_min; r[1] = p->i_max; r[2] = p->j_min; r[3] = p->j_max; r[4] = p->k_min; r[5] = p->k_max;
    if (r[0] == r[1] && r[0] == 0) r[1] = 1;
    else if (r[0] == r[1] && r[0] == s->ni) { r[0] = s->ni - 1; r[1] = r[0] + 1; }
    else if (r[2] == r[3] && r[2] == 0) r[3] = 1;
    else if (r[2] == r[3] && r[2] == s->nj) { r[2] = s->nj - 1; r[3] = r[2] + 1; }
    else if (r[4] == r[5] && r[4] == 0) r[5] = 1;
    else if (r[4] == r[5] && r[4] == s->nk) { r[4] = s->nk - 1; r[5] = r[4] + 1; }
    step[0] = step[1] = step[2] = 0;
    if (p->i_min == p->i_max) step[0] = p->i_min == 0 ? 1 : -1;
    else if (p->j_min == p->j_max) step[1] = p->j_min == 0 ? 1 : -1;
    else if (p->k_min == p->k_max) step[2] = p->k_min == 0 ? 1 : -1;
}

/* TurbulenceModelSA::updateBoundaryValues (src/turbulence_model_sa.cpp:250-345):
 * patch by patch in the boundary file's order, nu hat 0 on no-slip walls,
 * the free-stream value on inlets and farfields, the interior donor's value
 * on outlets, inviscid walls and transparent patches. */
static void sa_boundary_values(oracle_solver* s) {
    for (int m = 0; m < s->npatches; m++) {
        const patch* p = &s->patches[m];
        int kind;
        if (p->type == BC_NO_SLIP_WALL) kind = 0;
        else if (p->type == BC_INLET || p->type == BC_INLET_SUPERSONIC || p->type == BC_FARFIELD) kind = 1;
        else if (p->type == BC_OUTLET || p->type == BC_RADIAL_EQ || p->type == BC_THROTTLE || p->type == BC_MASS_FLOW ||
                 p->type == BC_OUTLET_SUPERSONIC || p->type == BC_INVISCID_WALL || p->type == BC_TRANSPARENT)
            kind = 2;
        else continue;
        long r[6], st[3];
        patch_nodes(s, p, r, st);
        for (long i = r[0]; i < r[1]; i++)
            for (long j = r[2]; j < r[3]; j++)
                for (long k = r[4]; k < r[5]; k++) {
                    long q = idx3(s, i, j, k);
                    if (kind == 0) s->nuhat[q] = 0.0;
                    else if (kind == 1) s->nuhat[q] = s->sa_init_nu * s->sa_ff_scale;
                    else s->nuhat[q] = s->nuhat[idx3(s, i + st[0], j + st[1], k + st[2])];
                }
    }
}

/* computeGradientGreenGauss (src/math_utils.cpp:173-234) of nu hat with
 * interpolateScalar (:395-466) and computeGreenGaussDivergence
 * (include/math_utils.hpp:95-106): face values (f1 - f0) d0 / (d0 + d1) from
 * the node, the node's own value on boundary faces, W E N S B T, divided by
 * the volume. */
static void sa_gradient(oracle_solver* s) {
    for (long i = 0; i < s->ni; i++)
        for (long j = 0; j < s->nj; j++)
            for (long k = 0; k < s->nk; k++) {
                long q = idx3(s, i, j, k);
                vec3 p0 = s->vert[q];
                double f0 = s->nuhat[q];
                long nb[6];
                int has[6];
                vec3 mid[6];
                has[0] = i > 0;         nb[0] = has[0] ? idx3(s, i - 1, j, k) : q; mid[0] = s->cI[sIi(s, i, j, k)];
                has[1] = i < s->ni - 1; nb[1] = has[1] ? idx3(s, i + 1, j, k) : q; mid[1] = s->cI[sIi(s, i + 1, j, k)];
                has[2] = j < s->nj - 1; nb[2] = has[2] ? idx3(s, i, j + 1, k) : q; mid[2] = s->cJ[sJi(s, i, j + 1, k)];
                has[3] = j > 0;         nb[3] = has[3] ? idx3(s, i, j - 1, k) : q; mid[3] = s->cJ[sJi(s, i, j, k)];
                has[4] = k > 0;         nb[4] = has[4] ? idx3(s, i, j, k - 1) : q; mid[4] = s->cK[sKi(s, i, j, k)];
                has[5] = k < s->nk - 1; nb[5] = has[5] ? idx3(s, i, j, k + 1) : q; mid[5] = s->cK[sKi(s, i, j, k + 1)];
                vec3 sf[6] = {vneg(s->sI[sIi(s, i, j, k)]), s->sI[sIi(s, i + 1, j, k)], s->sJ[sJi(s, i, j + 1, k)],
                              vneg(s->sJ[sJi(s, i, j, k)]), vneg(s->sK[sKi(s, i, j, k)]), s->sK[sKi(s, i, j, k + 1)]};
                vec3 g = v3(0.0, 0.0, 0.0);
                for (int f = 0; f < 6; f++) {
                    double sc = f0;
                    if (has[f]) {
                        double d0 = vmag(vsub(mid[f], p0));
                        double d1 = vmag(vsub(mid[f], s->vert[nb[f]]));
                        sc = f0 + (s->nuhat[nb[f]] - f0) * d0 / (d0 + d1);
                    }
                    g = vadd(g, vmul(sf[f], sc));
                }
                s->nuhat_grad[q] = vdiv(g, s->vol[q]);
            }
}

/* TurbulenceModelSA::updateMeanFlowTerms (src/turbulence_model_sa.cpp:370-390):
 * laminar kinematic viscosity mu(T) / rho from rho, rho u / rho, rho E / rho. */
static void sa_mean_flow(oracle_solver* s, double* const* U) {
    for (long q = 0; q < s->n; q++) {
        double rho = U[0][q];
        vec3 u = v3(U[1][q] / rho, U[2][q] / rho, U[3][q] / rho);
        double T = f_temperature_rho_u_et(s, rho, u, U[4][q] / rho);
        s->nul[q] = f_mu(s, T) / rho;
    }
}

/* nu + nu hat fn of one node (computeViscousFlux, :513-545). */
static double sa_nu_total(const oracle_solver* s, long q) {
    double nuL = s->nul[q], nuHat = s->nuhat[q];
    if (nuHat >= 0.0) return nuL + nuHat;
    double chi = (nuL > 0.0) ? (nuHat / nuL) : 0.0;
    double chi3 = chi * chi * chi;
    double fn = (SA_CN1 + chi3) / (SA_CN1 - chi3);
    return nuL + nuHat * fn;
}

/* TurbulenceModelSA::computeFluxContribution / computeAdvectionFlux /
 * computeViscousFlux (src/turbulence_model_sa.cpp:406-558): interior faces of
 * direction dir in storage order, first-order upwind advection of nu hat by
 * the mean face-normal velocity, diffusion (nu + nu hat fn) grad nu hat /
 * sigma averaged over the two nodes; the left node gains and the right node
 * loses (adv - visc) |S|. */
static void sa_flux_dir(oracle_solver* s, int dir, double* const* U) {
    long nf[3] = {s->ni, s->nj, s->nk};
    nf[dir] += 1;
    const vec3* surf = dir == 0 ? s->sI : (dir == 1 ? s->sJ : s->sK);
    const long st[3] = {dir == 0, dir == 1, dir == 2};
    for (long fi = 0; fi < nf[0]; fi++)
        for (long fj = 0; fj < nf[1]; fj++)
            for (long fk = 0; fk < nf[2]; fk++) {
                long dface = dir == 0 ? fi : (dir == 1 ? fj : fk);
                if (dface == 0 || dface == nf[dir] - 1) continue;
                long ql = idx3(s, fi - st[0], fj - st[1], fk - st[2]);
                long qr = idx3(s, fi, fj, fk);
                vec3 S = surf[dir == 0 ? sIi(s, fi, fj, fk) : (dir == 1 ? sJi(s, fi, fj, fk) : sKi(s, fi, fj, fk))];
                vec3 n = vnormalized(S);
                sv5 Wl = prim_of(state_at(s, U, fi - st[0], fj - st[1], fk - st[2]));
                sv5 Wr = prim_of(state_at(s, U, fi, fj, fk));
                double un = 0.5 * vdot(vadd(vel_of(Wl), vel_of(Wr)), n);
                double phi = (un >= 0.0) ? s->nuhat[ql] : s->nuhat[qr];
                double adv = phi * un;
                vec3 tl = vmul(vdiv(s->nuhat_grad[ql], SA_SIGMA), sa_nu_total(s, ql));
                vec3 tr = vmul(vdiv(s->nuhat_grad[qr], SA_SIGMA), sa_nu_total(s, qr));
                double visc = 0.5 * vdot(vadd(tl, tr), n);
                double c = (adv - visc) * vmag(S);
                s->sa_res[ql] += c;
                s->sa_res[qr] -= c;
            }
}

/* TurbulenceModelSA::computeSource (src/turbulence_model_sa.cpp:578-647):
 * production, destruction and cross diffusion of one node (SA-neg branch
 * for negative nu hat), with the rotation-rate magnitude of
 * computeRotationRateMagnitude (src/math_utils.cpp:620-639) from the
 * velocity gradients of the solution gradient. */
static double sa_source(const oracle_solver* s, long q) {
    double d = s->wdist[q];
    if (d <= 0.0) return 0.0;
    double nuHat = s->nuhat[q];
    double nuL = s->nul[q];
    if (nuL <= 0.0) nuL = 1e-14;
    vec3 gu = s->grad[0][q], gv = s->grad[1][q], gw = s->grad[2][q];
    double o12 = 0.5 * (gu.y - gv.x), o13 = 0.5 * (gu.z - gw.x), o23 = 0.5 * (gv.z - gw.y);
    double Sv = 2.0 * sqrt(o12 * o12 + o13 * o13 + o23 * o23);
    vec3 gn = s->nuhat_grad[q];
    double gsq = gn.x * gn.x + gn.y * gn.y + gn.z * gn.z;
    double cross = (SA_CB2 / SA_SIGMA) * gsq;
    double cw1 = sa_cw1();
    if (nuHat >= 0.0) {
        double chi = nuHat / nuL;
        double chi3 = chi * chi * chi;
        double cv1_3 = SA_CV1 * SA_CV1 * SA_CV1;
        double fv1 = chi3 / (chi3 + cv1_3);
        double fv2 = 1.0 - chi / (1.0 + chi * fv1);
        double dSq = d * d;
        double kd = SA_KAPPA * SA_KAPPA * dSq;
        double Sbar = (nuHat / kd) * fv2;
        double Shat;
        if (Sbar >= -SA_C2 * Sv) Shat = Sv + Sbar;
        else Shat = Sv + (Sv * (SA_C2 * SA_C2 * Sv + SA_C3 * Sbar)) / ((SA_C3 - 2.0 * SA_C2) * Sv - Sbar);
        double r;
        if (Shat * kd <= 0.0) r = 10.0;
        else r = dmin(nuHat / (Shat * kd), 10.0);
        double r2 = r * r;
        double r6 = r2 * r2 * r2;
        double g = r + SA_CW2 * (r6 - r);
        double g6 = pow(g, 6.0);
        double cw3_6 = pow(SA_CW3, 6.0);
        double fw = g * pow((1.0 + cw3_6) / (g6 + cw3_6), 1.0 / 6.0);
        double ft2 = SA_CT3 * exp(-SA_CT4 * chi * chi);
        double P = SA_CB1 * (1.0 - ft2) * Shat * nuHat;
        double D = (cw1 * fw - (SA_CB1 / (SA_KAPPA * SA_KAPPA)) * ft2) * (nuHat * nuHat / dSq);
        return P - D + cross;
    }
    double dSq = d * d;
    double Pn = SA_CB1 * (1.0 - SA_CT3) * Sv * nuHat;
    double Dn = cw1 * (nuHat * nuHat / dSq);
    return Pn + Dn + cross;
}

/* TurbulenceModelSA::updateSolution (src/turbulence_model_sa.cpp:649-841):
 * diagonal (time term, convective and diffusive spectral radii, destruction
 * Jacobian), a forward and a backward Gauss-Seidel sweep over the nodes in
 * storage order with upwind face couplings, under-relaxed update clamped to
 * +-1e5 nu. Returns 1 when an increment is NaN/Inf (the reference's
 * "Turbulence model diverged"). */
static int sa_update(oracle_solver* s, double* const* U) {
    const int is1D = s->topology == TOPO_1D, is3D = s->topology == TOPO_3D;
    const double cw1 = sa_cw1();
    for (long q = 0; q < s->n; q++) {
        double inv = 1.0 / U[0][q];
        s->sa_vel[q] = v3(U[1][q] * inv, U[2][q] * inv, U[3][q] * inv);
    }
    for (long i = 0; i < s->ni; i++)
        for (long j = 0; j < s->nj; j++)
            for (long k = 0; k < s->nk; k++) {
                long q = idx3(s, i, j, k);
                vec3 v = s->sa_vel[q];
                double vol = s->vol[q], nuHat = s->nuhat[q];
                vec3 sW = s->sI[sIi(s, i, j, k)], sE = s->sI[sIi(s, i + 1, j, k)];
                vec3 sS = s->sJ[sJi(s, i, j, k)], sN = s->sJ[sJi(s, i, j + 1, k)];
                vec3 sB = s->sK[sKi(s, i, j, k)], sT = s->sK[sKi(s, i, j, k + 1)];
                double lamW = fabs(vdot(v, sW)), lamE = fabs(vdot(v, sE));
                double lamS = 0.0, lamN = 0.0, lamB = 0.0, lamT = 0.0;
                if (!is1D) { lamS = fabs(vdot(v, sS)); lamN = fabs(vdot(v, sN)); }
                if (is3D) { lamB = fabs(vdot(v, sB)); lamT = fabs(vdot(v, sT)); }
                double sigC = 0.5 * (lamW + lamE + lamS + lamN + lamB + lamT);
                double nuDiff = (s->nul[q] + dmax(0.0, nuHat)) / SA_SIGMA;
                double sq = vdot(sW, sW) + vdot(sE, sE);
                if (!is1D) sq += vdot(sS, sS) + vdot(sN, sN);
                if (is3D) sq += vdot(sB, sB) + vdot(sT, sT);
                double sigV = (nuDiff / vol) * sq;
                double d = s->wdist[q];
                double dSq = dmax(d * d, 1e-16);
                double sigD = vol * (2.0 * cw1 * fabs(nuHat) / dSq);
                s->sa_diag[q] = (vol / s->dt[q]) + sigC + sigV + sigD;
            }
    for (long q = 0; q < s->n; q++) s->sa_dstar[q] = s->sa_dnu[q] = 0.0;
    for (long i = 0; i < s->ni; i++)
        for (long j = 0; j < s->nj; j++)
            for (long k = 0; k < s->nk; k++) {
                long q = idx3(s, i, j, k);
                double rhs = -s->sa_res[q];
                if (i > 0) {
                    double Vn = vdot(s->sa_vel[idx3(s, i - 1, j, k)], s->sI[sIi(s, i, j, k)]);
                    rhs += 0.5 * (Vn + fabs(Vn)) * s->sa_dstar[idx3(s, i - 1, j, k)];
                }
                if (!is1D && j > 0) {
                    double Vn = vdot(s->sa_vel[idx3(s, i, j - 1, k)], s->sJ[sJi(s, i, j, k)]);
                    rhs += 0.5 * (Vn + fabs(Vn)) * s->sa_dstar[idx3(s, i, j - 1, k)];
                }
                if (is3D && k > 0) {
                    double Vn = vdot(s->sa_vel[idx3(s, i, j, k - 1)], s->sK[sKi(s, i, j, k)]);
                    rhs += 0.5 * (Vn + fabs(Vn)) * s->sa_dstar[idx3(s, i, j, k - 1)];
                }
                s->sa_dstar[q] = rhs / s->sa_diag[q];
            }
    for (long i = s->ni - 1; i >= 0; i--)
        for (long j = s->nj - 1; j >= 0; j--)
            for (long k = s->nk - 1; k >= 0; k--) {
                long q = idx3(s, i, j, k);
                double sum = 0.0;
                if (i + 1 < s->ni) {
                    double Vn = vdot(s->sa_vel[idx3(s, i + 1, j, k)], s->sI[sIi(s, i + 1, j, k)]);
                    sum += 0.5 * (fabs(Vn) - Vn) * s->sa_dnu[idx3(s, i + 1, j, k)];
                }
                if (!is1D && j + 1 < s->nj) {
                    double Vn = vdot(s->sa_vel[idx3(s, i, j + 1, k)], s->sJ[sJi(s, i, j + 1, k)]);
                    sum += 0.5 * (fabs(Vn) - Vn) * s->sa_dnu[idx3(s, i, j + 1, k)];
                }
                if (is3D && k + 1 < s->nk) {
                    double Vn = vdot(s->sa_vel[idx3(s, i, j, k + 1)], s->sK[sKi(s, i, j, k + 1)]);
                    sum += 0.5 * (fabs(Vn) - Vn) * s->sa_dnu[idx3(s, i, j, k + 1)];
                }
                s->sa_dnu[q] = s->sa_dstar[q] + sum / s->sa_diag[q];
            }
    int diverged = 0;
    for (long q = 0; q < s->n; q++) {
        double dNu = s->sa_dnu[q] * s->sa_relax;
        if (isnan(dNu) || isinf(dNu)) diverged = 1;
        double nn = s->nuhat[q] + dNu;
        double mx = 1.0e5 * dmax(s->nul[q], 1e-12);
        nn = dmax(-mx, dmin(nn, mx));
        s->nuhat[q] = nn;
    }
    return diverged;
}

/* TurbulenceModelSA::solve (src/turbulence_model_sa.cpp:347-368), called once
 * per iteration before the Runge-Kutta stages with the iteration's time
 * step (Solver::updateTurbulenceSolution, src/solver.cpp:3061-3071). */
static int sa_solve(oracle_solver* s, double* const* U) {
    sa_boundary_values(s);
    sa_gradient(s);
    sa_mean_flow(s, U);
    memset(s->sa_res, 0, sizeof(double) * s->n);
    sa_flux_dir(s, 0, U);
    if (s->topology != TOPO_1D) sa_flux_dir(s, 1, U);
    if (s->topology == TOPO_3D) sa_flux_dir(s, 2, U);
    for (long i = 0; i < s->ni; i++)
        for (long j = 0; j < s->nj; j++)
            for (long k = 0; k < s->nk; k++) {
                long q = idx3(s, i, j, k);
                double Qt = sa_source(s, q);
                s->sa_res[q] -= Qt * s->vol[q];
            }
    int div = sa_update(s, U);
    sa_boundary_values(s);
    return div;
}

/* Solver::computeResiduals (src/solver.cpp:1783-1833). */
static void compute_residuals(oracle_solver* s, double* const* U, long it) {
    for (int c = 0; c < 5; c++) memset(s->R[c], 0, sizeof(double) * s->n);
    advection_residuals(s, 0, U, it);
    if (s->topology != TOPO_1D) advection_residuals(s, 1, U, it);
    if (s->topology == TOPO_3D) advection_residuals(s, 2, U, it);
    if (s->viscous) {
        viscous_residuals(s, 0, U);
        viscous_residuals(s, 1, U);
        if (s->topology == TOPO_3D) viscous_residuals(s, 2, U);
    }
    source_residuals(s, U);
    if (s->periodic) periodic_residuals(s);
    no_slip_momentum(s, s->R);
}

/* Solver::computeTimestepArray (src/solver.cpp:1531-1630). */
static void compute_timestep(oracle_solver* s, double* const* U) {
    if (s->dt_method == DT_FIXED) {
        for (long q = 0; q < s->n; q++) s->dt[q] = s->fixed_dt;
        return;
    }
    for (long i = 0; i < s->ni; i++)
        for (long j = 0; j < s->nj; j++)
            for (long k = 0; k < s->nk; k++) {
                vec3 p0 = s->dual[didx(s, i, j, k)];
                vec3 eI = vsub(s->dual[didx(s, i + 1, j, k)], p0);
                vec3 eJ = vsub(s->dual[didx(s, i, j + 1, k)], p0);
                vec3 eK = vsub(s->dual[didx(s, i, j, k + 1)], p0);
                double dsI = vmag(eI), dsJ = vmag(eJ), dsK = vmag(eK);
                vec3 dI = vdiv(eI, dsI), dJ = vdiv(eJ, dsJ), dK = vdiv(eK, dsK);
                sv5 W = prim_of(state_at(s, U, i, j, k));
                vec3 u = vel_of(W);
                double rho = W.v[0];
                double a = f_sound_speed_rho_u_et(s, W.v[0], u, W.v[4]);
                double mu = 0.0, mut = 0.0;
                if (s->viscous) {
                    mu = f_mu(s, f_temperature_rho_u_et(s, W.v[0], u, W.v[4]));
                    mut = sa_mut(s, rho, idx3(s, i, j, k));
                }
                double nu = mu / rho, nut = mut / rho;
                double ui = fabs(vdot(u, dI)), uj = fabs(vdot(u, dJ)), uk = fabs(vdot(u, dK));
                double lc = (ui + a) / dsI;
                double ih2 = 1.0 / (dsI * dsI);
                if (s->topology != TOPO_1D) { lc += (uj + a) / dsJ; ih2 += 1.0 / (dsJ * dsJ); }
                if (s->topology == TOPO_3D) { lc += (uk + a) / dsK; ih2 += 1.0 / (dsK * dsK); }
                double lv = 4.0 * (nu + nut) * ih2;
                s->dt[idx3(s, i, j, k)] = s->cfl / (lc + lv);
            }
    if (s->dt_method == DT_GLOBAL) {
        double m = s->dt[0];
        for (long q = 1; q < s->n; q++) if (s->dt[q] < m) m = s->dt[q];
        for (long q = 0; q < s->n; q++) s->dt[q] = m;
    }
}

/* Solver::updateSolution (src/solver.cpp:2230-2249). */
static void update_solution(oracle_solver* s, double alpha) {
    for (long q = 0; q < s->n; q++) {
        double f = alpha * s->dt[q] / s->vol[q];
        for (int c = 0; c < 5; c++) s->Utmp[c][q] = s->U[c][q] - s->R[c][q] * f;
    }
}

/* Solver::enforcePeriodicityOnSolution (src/solver.cpp:2308-2327). */
static void periodic_solution(oracle_solver* s) {
    if (!s->periodic) return;
    double ang = s->per_angle_rad, inv = -ang;
    for (long i = 0; i < s->ni; i++)
        for (long j = 0; j < s->nj; j++) {
            sv5 U1 = state_at(s, s->Utmp, i, j, 0);
            sv5 U2 = state_at(s, s->Utmp, i, j, s->nk - 1);
            sv5 Ua = smul(sadd(U1, rot_state(U2, inv)), 0.5);
            state_set(s, s->Utmp, i, j, 0, Ua);
            state_set(s, s->Utmp, i, j, s->nk - 1, rot_state(Ua, ang));
        }
}

/* ---------------------------------------------------- mass flow and turbo */

static vec3 boundary_surface(const oracle_solver* s, int bi, long a, long b) {
    switch (bi) {
        case BI_ISTART: return s->sI[sIi(s, 0, a, b)];
        case BI_IEND: return s->sI[sIi(s, s->ni, a, b)];
        case BI_JSTART: return s->sJ[sJi(s, a, 0, b)];
        case BI_JEND: return s->sJ[sJi(s, a, s->nj, b)];
        case BI_KSTART: return s->sK[sKi(s, a, b, 0)];
        default: return s->sK[sKi(s, a, b, s->nk)];
    }
}
static void boundary_extent(const oracle_solver* s, int bi, long* na, long* nb) {
    if (bi <= BI_IEND) { *na = s->nj; *nb = s->nk; }
    else if (bi <= BI_JEND) { *na = s->ni; *nb = s->nk; }
    else { *na = s->ni; *nb = s->nj; }
}
static long boundary_node(const oracle_solver* s, int bi, long a, long b) {
    switch (bi) {
        case BI_ISTART: return idx3(s, 0, a, b);
        case BI_IEND: return idx3(s, s->ni - 1, a, b);
        case BI_JSTART: return idx3(s, a, 0, b);
        case BI_JEND: return idx3(s, a, s->nj - 1, b);
        case BI_KSTART: return idx3(s, a, b, 0);
        default: return idx3(s, a, b, s->nk - 1);
    }
}

/* Solver::updateMassFlows (src/solver.cpp:1633-1649) with computeSurfaceIntegral
 * (src/math_utils.cpp:18-33). */
static void update_mass_flows(oracle_solver* s, double* const* U) {
    for (int bi = 0; bi < 6; bi++) {
        long na, nb;
        boundary_extent(s, bi, &na, &nb);
        double sum = 0.0;
        for (long a = 0; a < na; a++)
            for (long b = 0; b < nb; b++) {
                vec3 S = boundary_surface(s, bi, a, b);
                long q = boundary_node(s, bi, a, b);
                sum += S.x * U[1][q] + S.y * U[2][q] + S.z * U[3][q];
            }
        s->massflow[bi] = sum;
    }
}

/* Solver::updateTurboPerformance (src/solver.cpp:1652-1781). */
static void update_turbo(oracle_solver* s, double* const* U) {
    int bci[2];
    switch (s->turbo_dir) {
        case 1: bci[0] = BI_IEND; bci[1] = BI_ISTART; break;
        case 2: bci[0] = BI_JSTART; bci[1] = BI_JEND; break;
        case 3: bci[0] = BI_JEND; bci[1] = BI_JSTART; break;
        default: bci[0] = BI_ISTART; bci[1] = BI_IEND; break;
    }
    double mflow = 0.5 * (fabs(s->massflow[bci[0]]) + fabs(s->massflow[bci[1]]));
    if (s->topology == TOPO_AXI) mflow *= 2.0 * M_PI / s->wedge;
    else if (s->per_angle_deg != 0.0) mflow *= 360.0 / s->per_angle_deg;
    double pt[2], tt[2], htot[2], ent[2];
    for (int m = 0; m < 2; m++) {
        int bi = bci[m];
        long na, nb;
        boundary_extent(s, bi, &na, &nb);
        double sp = 0.0, stt = 0.0, sht = 0.0, ss = 0.0;
        for (long a = 0; a < na; a++)
            for (long b = 0; b < nb; b++) {
                long q;
                /* getPrimitiveAtBoundary: K planes fall back to (0, a, b). */
                if (bi <= BI_JEND) q = boundary_node(s, bi, a, b);
                else q = idx3(s, 0, a, b);
                sv5 Uc = {{U[0][q], U[1][q], U[2][q], U[3][q], U[4][q]}};
                sv5 W = prim_of(Uc);
                double rho = W.v[0];
                vec3 u = vel_of(W);
                double et = W.v[4];
                double P = f_total_pressure_rho_u_et(s, rho, u, et);
                double T = f_total_temperature_rho_u_et(s, rho, u, et);
                vec3 S = boundary_surface(s, bi, a, b);
                sp += S.x * (rho * u.x * P) + S.y * (rho * u.y * P) + S.z * (rho * u.z * P);
                stt += S.x * (rho * u.x * T) + S.y * (rho * u.y * T) + S.z * (rho * u.z * T);
                if (s->real) { /* total enthalpy and entropy integrals, src/solver.cpp:1732-1749 */
                    double H = f_total_enthalpy_rho_u_et(s, rho, u, et);
                    double Sv = f_entropy_rho_u_et(s, rho, u, et);
                    sht += S.x * (rho * u.x * H) + S.y * (rho * u.y * H) + S.z * (rho * u.z * H);
                    ss += S.x * (rho * u.x * Sv) + S.y * (rho * u.y * Sv) + S.z * (rho * u.z * Sv);
                }
            }
        double mf = s->massflow[bi];
        if (fabs(mf) < 1e-12) mf = (mf >= 0.0 ? 1e-12 : -1e-12);
        pt[m] = sp / mf;
        tt[m] = stt / mf;
        htot[m] = sht / mf;
        ent[m] = ss / mf;
    }
    double pr = (fabs(pt[0]) > 1e-12) ? pt[1] / pt[0] : 1.0;
    double tr = (fabs(tt[0]) > 1e-12) ? tt[1] / tt[0] : 1.0;
    s->turbo[0] = mflow;
    s->turbo[1] = pr;
    s->turbo[2] = tr;
    if (s->real) { /* src/solver.cpp:1768-1776, FluidBase::computeTotalEfficiency_h */
        double hIn = htot[0], sIn = ent[0], ptOut = pt[1], hOut = htot[1];
        double hOutS = lut_h_p_s(s->lut, ptOut, sIn);
        double dh = hOut - hIn, dhs = hOutS - hIn;
        double eta;
        if (fabs(dh) < 1e-12) eta = 1.0;
        else if (dh >= 0.0) eta = dhs / dh;
        else eta = (fabs(dhs) < 1e-12) ? 1.0 : dh / dhs;
        s->turbo[3] = eta;
    } else {
        s->turbo[3] = f_efficiency(s, pr, tr);
    }
    s->has_turbo = 1;
}

/* integrateRadialEquilibrium (src/math_utils.cpp:141-170). */
static void integrate_radial_eq(const double* rho, const double* ut, const double* r, double* p,
                                int n, double hub) {
    p[0] = hub;
    for (int i = 1; i < n; ++i) {
        double r1 = r[i - 1], r2 = r[i];
        double dr = r2 - r1;
        double d1 = rho[i - 1] * ut[i - 1] * ut[i - 1] / r1;
        double d2 = rho[i] * ut[i] * ut[i] / r2;
        p[i] = p[i - 1] + 0.5 * (d1 + d2) * dr;
    }
}

/* GreitzerModel::computePlenumPressure (src/greitzer_model.cpp:36-56). */
static double greitzer_step(oracle_solver* s, double mflow) {
    s->gz_min = mflow;
    s->gz_t += s->fixed_dt;
    /* computeSoundSpeed_p_T: FluidIdeal sqrt(gamma R T), FluidReal the (p, T) table */
    double a = s->real ? table_interp(&s->lut->a_pt, s->gz_p, s->gz_T) : sqrt(s->gamma * s->rgas * s->gz_T);
    double np = s->gz_p + s->fixed_dt * a * a / s->plenum_volume * (s->gz_min - s->gz_mout);
    s->gz_p = np;
    double dp = s->gz_p - s->ambient_p;
    s->gz_mout = (dp > 0.0) ? sqrt(dp / s->throttle_kt) : 0.0;
    return s->gz_p;
}

/* Solver::updateRadialProfiles (src/solver.cpp:2688-2787). */
static void update_radial_profiles(oracle_solver* s, double* const* U) {
    if (!s->has_turbo) {
        update_mass_flows(s, U);
        update_turbo(s, U);
    }
    if (s->greitzer) s->hub_p = greitzer_step(s, s->turbo[0]);
    for (int m = 0; m < s->nprofiles; m++) {
        radial_profile* rp = &s->profiles[m];
        const patch* bp = &s->patches[rp->patch];
        double* dens = (double*)calloc(rp->n, sizeof(double));
        double* vt = (double*)calloc(rp->n, sizeof(double));
        long i = (bp->i_min > 0) ? (bp->i_min - 1) : 0;
        int kk = 0;
        for (long j = bp->j_min; j < bp->j_max && kk < rp->n; j++) {
            sv5 W = prim_of(state_at(s, U, i, j, 0));
            double th = node_theta(s, i, j, 0);
            vec3 vcyl = cyl_of_cart(vel_of(W), th);
            dens[kk] = W.v[0];
            vt[kk] = fabs(vcyl.z);
            kk++;
        }
        if (s->greitzer) {
        } else if (bp->type == BC_THROTTLE) {
            double kt = bp->values[0];
            double mf = s->turbo[0];
            double ptin = 0.0;
            for (int b = 0; b < s->npatches; b++)
                if (s->patches[b].type == BC_INLET) { ptin = s->patches[b].values[0]; break; }
            s->hub_p = ptin + kt * mf * mf;
        } else if (bp->type == BC_MASS_FLOW) { /* src/solver.cpp:2734-2770 */
            double target = bp->values[0];
            double cur = fabs(s->massflow[bp->orientation]);
            if (s->topology == TOPO_AXI) cur *= 2.0 * M_PI / s->wedge;
            else if (s->per_angle_deg != 0.0) cur *= 360.0 / s->per_angle_deg;
            double relax = s->mf_relax;
            if (bp->nvalues >= 3 && bp->values[2] > 0.0) relax = bp->values[2];
            double err = (cur - target) / target;
            double dp = relax * err;
            if (dp < -s->mf_max_change) dp = -s->mf_max_change;
            else if (s->mf_max_change < dp) dp = s->mf_max_change;
            double p0 = rp->pressure[0];
            if (p0 <= 0.0) p0 = s->init_p > 0.0 ? s->init_p : 101325.0;
            s->hub_p = p0 * (1.0 + dp);
            if (s->hub_p < 100.0) s->hub_p = 100.0;
        } else if (bp->type == BC_RADIAL_EQ) {
            s->hub_p = rp->pressure[0];
        }
        if (rp->nradius == rp->n && rp->nradius > 1)
            integrate_radial_eq(dens, vt, rp->radius, rp->pressure, rp->n, s->hub_p);
        else
            for (int q = 0; q < rp->n; q++) rp->pressure[q] = s->hub_p;
        free(dens);
        free(vt);
    }
}

/* Solver::computeLogResidualNorm (src/solver.cpp:1488-1508), Matrix3D::norm
 * (include/types.hpp:441-448). */
static int log_residual_norm(const oracle_solver* s, double out[5]) {
    for (int v = 0; v < 5; v++) {
        double sum = 0;
        for (long q = 0; q < s->n; q++) sum += s->R[v][q] * s->R[v][q];
        double nrm = sqrt(sum);
        if (isnan(nrm) || isinf(nrm)) return fail("Solver diverged: NaN or Inf detected in residual variable %d", v);
        if (nrm >= DBL_MIN) out[v] = log10(nrm / (double)(s->ni * s->nj * s->nk));
        else out[v] = -16.0;
        if (out[v] < -16.0) out[v] = -16.0;
    }
    return 0;
}

/* Solver::checkConvergence (src/solver.cpp:2985-3015). */
static int check_convergence(const oracle_solver* s, const double cur[5]) {
    if (!s->steady) return 0;
    for (int v = 0; v < 5; ++v) {
        if (v == 3 && s->topology != TOPO_3D && s->topology != TOPO_AXI) continue;
        if (v == 2 && s->topology == TOPO_1D) continue;
        if (s->init_log[v] <= -15.99) continue;
        if (cur[v] <= -15.0) continue;
        if (cur[v] >= s->init_log[v] - (double)s->drop) return 0;
    }
    return 1;
}

/* -------------------------------------------------------------- set-up */

static int read_grid(oracle_solver* s, const char* path) { /* src/input.cpp:14-82 */
    FILE* f = fopen(path, "r");
    if (!f) return fail("Error opening coordinates CSV file '%s'", path);
    char* line = NULL;
    size_t cap = 0;
    long ni = 0, nj = 0, nk = 0;
    char names[64][64];
    int nh = 0;
    while (getline(&line, &cap, f) > 0) {
        if (!strncmp(line, "NI=", 3)) ni = atol(line + 3);
        else if (!strncmp(line, "NJ=", 3)) nj = atol(line + 3);
        else if (!strncmp(line, "NK=", 3)) nk = atol(line + 3);
        else if (!strncmp(line, "x,y,z", 5)) {
            char* save = NULL;
            trim(line, "\r\n");
            for (char* t = strtok_r(line, ",", &save); t && nh < 64; t = strtok_r(NULL, ",", &save))
                snprintf(names[nh++], 64, "%s", t);
            break;
        }
    }
    s->ni = ni; s->nj = nj; s->nk = nk; s->n = ni * nj * nk;
    if (s->n <= 0) { fclose(f); free(line); return fail("bad grid header in %s", path); }
    double** cols = (double**)calloc(nh, sizeof(double*));
    for (int h = 0; h < nh; h++) cols[h] = (double*)calloc(s->n, sizeof(double));
    long np = 0;
    while (getline(&line, &cap, f) > 0 && np < s->n) {
        double vals[64];
        int nv = 0;
        char* p = line;
        while (*p && nv < 64) {
            char* end;
            double v = strtod(p, &end);
            if (end == p) break;
            vals[nv++] = v;
            p = end;
            while (*p == ',' || *p == ' ') p++;
            if (*p == '\r' || *p == '\n') break;
        }
        if (nv != nh) continue;
        for (int h = 0; h < nh; h++) cols[h][np] = vals[h];
        np++;
    }
    fclose(f);
    free(line);
    if (np != s->n) return fail("grid %s: read %ld points, expected %ld", path, np, s->n);
    s->vert = (vec3*)calloc(s->n, sizeof(vec3));
    for (int h = 0; h < nh; h++) {
        int used = 0;
        if (!strcmp(names[h], "x")) { for (long q = 0; q < s->n; q++) s->vert[q].x = cols[h][q]; used = 1; }
        if (!strcmp(names[h], "y")) { for (long q = 0; q < s->n; q++) s->vert[q].y = cols[h][q]; used = 1; }
        if (!strcmp(names[h], "z")) { for (long q = 0; q < s->n; q++) s->vert[q].z = cols[h][q]; used = 1; }
        for (int fdx = 0; fdx < F_COUNT && !used; fdx++)
            if (!strcmp(names[h], FIELD_NAMES[fdx])) { s->field[fdx] = cols[h]; cols[h] = NULL; used = 1; }
        free(cols[h]);
    }
    free(cols);
    if (nj == 1 && nk == 1) s->ndim = 1;
    else if (nk == 1) s->ndim = 2;
    else s->ndim = 3;
    return 0;
}

/* Mesh::computeSurfaceVectorAndCenter (src/mesh.cpp:165-190). */
static void surface_and_center(vec3 p1, vec3 p2, vec3 p3, vec3 p4, vec3* nrm, vec3* ctr) {
    vec3 a1 = vsub(p2, p1), b1 = vsub(p3, p2), a2 = vsub(p3, p1), b2 = vsub(p4, p3);
    vec3 s1 = vdiv(vcross(a1, b1), 2.0);
    vec3 s2 = vdiv(vcross(a2, b2), 2.0);
    *nrm = vadd(s1, s2);
    vec3 c1 = vdiv(vadd(vadd(p1, p2), p3), 3.0);
    vec3 c2 = vdiv(vadd(vadd(p1, p3), p4), 3.0);
    *ctr = vdiv(vadd(vmul(c1, vmag(s1)), vmul(c2, vmag(s2))), vmag(s1) + vmag(s2));
}

static void build_dual_2d(oracle_solver* s) { /* src/mesh.cpp:373-435 */
    long NI = s->ni, NJ = s->nj, DI = NI + 1, DJ = NJ + 1;
    vec3* nodes = (vec3*)calloc(DI * DJ, sizeof(vec3));
#define ND(i, j) nodes[(i) * DJ + (j)]
#define VX(i, j) s->vert[idx3(s, (i), (j), 0)]
    for (long i = 1; i < DI - 1; i++)
        for (long j = 1; j < DJ - 1; j++)
            ND(i, j) = vdiv(vadd(vadd(vadd(VX(i - 1, j - 1), VX(i, j - 1)), VX(i, j)), VX(i - 1, j)), 4.0);
    ND(0, 0) = VX(0, 0);
    ND(0, DJ - 1) = VX(0, NJ - 1);
    ND(DI - 1, 0) = VX(NI - 1, 0);
    ND(DI - 1, DJ - 1) = VX(NI - 1, NJ - 1);
    for (long i = 1; i < DI - 1; i++) {
        ND(i, 0) = vdiv(vadd(VX(i - 1, 0), VX(i, 0)), 2.0);
        ND(i, DJ - 1) = vdiv(vadd(VX(i - 1, NJ - 1), VX(i, NJ - 1)), 2.0);
    }
    for (long j = 1; j < DJ - 1; j++) {
        ND(0, j) = vdiv(vadd(VX(0, j - 1), VX(0, j)), 2.0);
        ND(DI - 1, j) = vdiv(vadd(VX(NI - 1, j - 1), VX(NI - 1, j)), 2.0);
    }
    if (s->topology == TOPO_AXI) {
        s->wedge = 1.0 * M_PI / 180.0;
        for (long i = 0; i < DI; i++)
            for (long j = 0; j < DJ; j++) {
                vec3* d0 = &s->dual[didx(s, i, j, 0)];
                vec3* d1 = &s->dual[didx(s, i, j, 1)];
                d0->x = ND(i, j).x; d1->x = ND(i, j).x;
                d0->y = ND(i, j).y * cos(-s->wedge / 2.0);
                d1->y = ND(i, j).y * cos(+s->wedge / 2.0);
                d0->z = ND(i, j).y * sin(-s->wedge / 2.0);
                d1->z = ND(i, j).y * sin(+s->wedge / 2.0);
            }
    } else {
        double th = 1.0;
        for (long i = 0; i < DI; i++)
            for (long j = 0; j < DJ; j++) {
                vec3* d0 = &s->dual[didx(s, i, j, 0)];
                vec3* d1 = &s->dual[didx(s, i, j, 1)];
                d0->x = ND(i, j).x; d1->x = ND(i, j).x;
                d0->y = ND(i, j).y; d1->y = ND(i, j).y;
                d0->z = -th / 2.0; d1->z = +th / 2.0;
            }
    }
#undef ND
#undef VX
    free(nodes);
}

static void build_dual_3d(oracle_solver* s) { /* src/mesh.cpp:478-557 */
    long NI = s->ni, NJ = s->nj, NK = s->nk, DI = NI + 1, DJ = NJ + 1, DK = NK + 1;
#define D(i, j, k) s->dual[didx(s, (i), (j), (k))]
#define V(i, j, k) s->vert[idx3(s, (i), (j), (k))]
    for (long i = 1; i < DI - 1; i++)
        for (long j = 1; j < DJ - 1; j++)
            for (long k = 1; k < DK - 1; k++) {
                vec3 a = vadd(vadd(vadd(V(i - 1, j - 1, k - 1), V(i, j - 1, k - 1)), V(i - 1, j, k - 1)), V(i - 1, j - 1, k));
                a = vadd(vadd(vadd(vadd(a, V(i, j, k - 1)), V(i, j - 1, k)), V(i - 1, j, k)), V(i, j, k));
                D(i, j, k) = vdiv(a, 8.0);
            }
    D(0, 0, 0) = V(0, 0, 0);
    D(DI - 1, 0, 0) = V(NI - 1, 0, 0);
    D(0, DJ - 1, 0) = V(0, NJ - 1, 0);
    D(0, 0, DK - 1) = V(0, 0, NK - 1);
    D(DI - 1, DJ - 1, 0) = V(NI - 1, NJ - 1, 0);
    D(DI - 1, 0, DK - 1) = V(NI - 1, 0, NK - 1);
    D(0, DJ - 1, DK - 1) = V(0, NJ - 1, NK - 1);
    D(DI - 1, DJ - 1, DK - 1) = V(NI - 1, NJ - 1, NK - 1);
    for (long i = 1; i < DI - 1; i++) {
        D(i, 0, 0) = vdiv(vadd(V(i - 1, 0, 0), V(i, 0, 0)), 2.0);
        D(i, DJ - 1, 0) = vdiv(vadd(V(i - 1, NJ - 1, 0), V(i, NJ - 1, 0)), 2.0);
        D(i, 0, DK - 1) = vdiv(vadd(V(i - 1, 0, NK - 1), V(i, 0, NK - 1)), 2.0);
        D(i, DJ - 1, DK - 1) = vdiv(vadd(V(i - 1, NJ - 1, NK - 1), V(i, NJ - 1, NK - 1)), 2.0);
    }
    for (long j = 1; j < DJ - 1; j++) {
        D(0, j, 0) = vdiv(vadd(V(0, j - 1, 0), V(0, j, 0)), 2.0);
        D(DI - 1, j, 0) = vdiv(vadd(V(NI - 1, j - 1, 0), V(NI - 1, j, 0)), 2.0);
        D(0, j, DK - 1) = vdiv(vadd(V(0, j - 1, NK - 1), V(0, j, NK - 1)), 2.0);
        D(DI - 1, j, DK - 1) = vdiv(vadd(V(NI - 1, j - 1, NK - 1), V(NI - 1, j, NK - 1)), 2.0);
    }
    for (long k = 1; k < DK - 1; k++) {
        D(0, 0, k) = vdiv(vadd(V(0, 0, k - 1), V(0, 0, k)), 2.0);
        D(DI - 1, 0, k) = vdiv(vadd(V(NI - 1, 0, k - 1), V(NI - 1, 0, k)), 2.0);
        D(0, DJ - 1, k) = vdiv(vadd(V(0, NJ - 1, k - 1), V(0, NJ - 1, k)), 2.0);
        D(DI - 1, DJ - 1, k) = vdiv(vadd(V(NI - 1, NJ - 1, k - 1), V(NI - 1, NJ - 1, k)), 2.0);
    }
    for (long j = 1; j < DJ - 1; j++)
        for (long k = 1; k < DK - 1; k++) {
            D(0, j, k) = vdiv(vadd(vadd(vadd(V(0, j - 1, k - 1), V(0, j, k - 1)), V(0, j - 1, k)), V(0, j, k)), 4.0);
            D(DI - 1, j, k) = vdiv(vadd(vadd(vadd(V(NI - 1, j - 1, k - 1), V(NI - 1, j, k - 1)), V(NI - 1, j - 1, k)), V(NI - 1, j, k)), 4.0);
        }
    for (long i = 1; i < DI - 1; i++)
        for (long k = 1; k < DK - 1; k++) {
            D(i, 0, k) = vdiv(vadd(vadd(vadd(V(i - 1, 0, k - 1), V(i, 0, k - 1)), V(i - 1, 0, k)), V(i, 0, k)), 4.0);
            D(i, DJ - 1, k) = vdiv(vadd(vadd(vadd(V(i - 1, NJ - 1, k - 1), V(i, NJ - 1, k - 1)), V(i - 1, NJ - 1, k)), V(i, NJ - 1, k)), 4.0);
        }
    for (long i = 1; i < DI - 1; i++)
        for (long j = 1; j < DJ - 1; j++) {
            D(i, j, 0) = vdiv(vadd(vadd(vadd(V(i - 1, j - 1, 0), V(i, j - 1, 0)), V(i - 1, j, 0)), V(i, j, 0)), 4.0);
            D(i, j, DK - 1) = vdiv(vadd(vadd(vadd(V(i - 1, j - 1, NK - 1), V(i, j - 1, NK - 1)), V(i - 1, j, NK - 1)), V(i, j, NK - 1)), 4.0);
        }
#undef D
#undef V
}

static void build_interfaces(oracle_solver* s) { /* src/mesh.cpp:116-163 */
    long DI = s->ni + 1, DJ = s->nj + 1, DK = s->nk + 1;
#define D(i, j, k) s->dual[didx(s, (i), (j), (k))]
    for (long i = 0; i < DI; i++)
        for (long j = 0; j < DJ - 1; j++)
            for (long k = 0; k < DK - 1; k++)
                surface_and_center(D(i, j, k), D(i, j + 1, k), D(i, j + 1, k + 1), D(i, j, k + 1),
                                   &s->sI[sIi(s, i, j, k)], &s->cI[sIi(s, i, j, k)]);
    for (long i = 0; i < DI - 1; i++)
        for (long j = 0; j < DJ; j++)
            for (long k = 0; k < DK - 1; k++)
                surface_and_center(D(i, j, k), D(i, j, k + 1), D(i + 1, j, k + 1), D(i + 1, j, k),
                                   &s->sJ[sJi(s, i, j, k)], &s->cJ[sJi(s, i, j, k)]);
    for (long i = 0; i < DI - 1; i++)
        for (long j = 0; j < DJ - 1; j++)
            for (long k = 0; k < DK; k++)
                surface_and_center(D(i, j, k), D(i + 1, j, k), D(i + 1, j + 1, k), D(i, j + 1, k),
                                   &s->sK[sKi(s, i, j, k)], &s->cK[sKi(s, i, j, k)]);
#undef D
}

static void build_volumes(oracle_solver* s) { /* src/mesh.cpp:192-230 */
    for (long i = 0; i < s->ni; i++)
        for (long j = 0; j < s->nj; j++)
            for (long k = 0; k < s->nk; k++) {
                vec3 sf[6] = {vneg(s->sI[sIi(s, i, j, k)]), vneg(s->sJ[sJi(s, i, j, k)]),
                              vneg(s->sK[sKi(s, i, j, k)]), s->sI[sIi(s, i + 1, j, k)],
                              s->sJ[sJi(s, i, j + 1, k)], s->sK[sKi(s, i, j, k + 1)]};
                vec3 cc[6] = {s->cI[sIi(s, i, j, k)], s->cJ[sJi(s, i, j, k)], s->cK[sKi(s, i, j, k)],
                              s->cI[sIi(s, i + 1, j, k)], s->cJ[sJi(s, i, j + 1, k)], s->cK[sKi(s, i, j, k + 1)]};
                double v = 0.0;
                for (int f = 0; f < 6; f++) v += sf[f].x * cc[f].x;
                s->vol[idx3(s, i, j, k)] = v;
            }
}

/* interpolateScalar (src/math_utils.cpp:395-463), direction codes
 * 0 W, 1 E, 2 N, 3 S, 4 B, 5 T. */
static double interp_scalar(const oracle_solver* s, const double* fld, long i, long j, long k,
                            vec3 pt, int dir) {
    vec3 p0 = s->vert[idx3(s, i, j, k)];
    double f0 = fld[idx3(s, i, j, k)];
    long i1 = i, j1 = j, k1 = k;
    switch (dir) {
        case 0: if (i == 0) return f0; i1 = i - 1; break;
        case 1: if (i == s->ni - 1) return f0; i1 = i + 1; break;
        case 2: if (j == s->nj - 1) return f0; j1 = j + 1; break;
        case 3: if (j == 0) return f0; j1 = j - 1; break;
        case 4: if (k == 0) return f0; k1 = k - 1; break;
        default: if (k == s->nk - 1) return f0; k1 = k + 1; break;
    }
    vec3 p1 = s->vert[idx3(s, i1, j1, k1)];
    double f1 = fld[idx3(s, i1, j1, k1)];
    double d0 = vmag(vsub(pt, p0)), d1 = vmag(vsub(pt, p1));
    return f0 + (f1 - f0) * d0 / (d0 + d1);
}

/* computeGradientGreenGauss (src/math_utils.cpp:173-234) for the blockage
 * (Mesh::computeInputGradients, src/mesh.cpp:571-581). */
static void build_blockage_gradient(oracle_solver* s) {
    s->gradb = (vec3*)calloc(s->n, sizeof(vec3));
    const double* b = s->field[F_BLOCKAGE];
    for (long i = 0; i < s->ni; i++)
        for (long j = 0; j < s->nj; j++)
            for (long k = 0; k < s->nk; k++) {
                vec3 sf[6] = {vneg(s->sI[sIi(s, i, j, k)]), s->sI[sIi(s, i + 1, j, k)],
                              s->sJ[sJi(s, i, j + 1, k)], vneg(s->sJ[sJi(s, i, j, k)]),
                              vneg(s->sK[sKi(s, i, j, k)]), s->sK[sKi(s, i, j, k + 1)]};
                vec3 cc[6] = {s->cI[sIi(s, i, j, k)], s->cI[sIi(s, i + 1, j, k)], s->cJ[sJi(s, i, j + 1, k)],
                              s->cJ[sJi(s, i, j, k)], s->cK[sKi(s, i, j, k)], s->cK[sKi(s, i, j, k + 1)]};
                int dirs[6] = {0, 1, 2, 3, 4, 5};
                vec3 g = v3(0, 0, 0);
                for (int f = 0; f < 6; f++) {
                    double sc = interp_scalar(s, b, i, j, k, cc[f], dirs[f]);
                    g = vadd(g, vmul(sf[f], sc));
                }
                s->gradb[idx3(s, i, j, k)] = vdiv(g, s->vol[idx3(s, i, j, k)]);
            }
}

/* atan2FromZeroTo2pi (src/math_utils.cpp:466-471). */
static double atan2_0_2pi(double y, double x) {
    double a = atan2(y, x);
    if (a < 0) a += 2 * M_PI;
    return a;
}

/* Mesh::checkPeriodicity (src/mesh.cpp:584-619). */
static int check_periodicity(oracle_solver* s, double transl, double angle) {
    vec3 drag = v3(0.0, 0.0, transl);
    for (long i = 0; i < s->ni; i++)
        for (long j = 0; j < s->nj; j++) {
            vec3 a = s->vert[idx3(s, i, j, 0)];
            vec3 b = vsub(s->vert[idx3(s, i, j, s->nk - 1)], drag);
            double ta = atan2_0_2pi(a.z, a.y), tb = atan2_0_2pi(b.z, b.y);
            double dth = fmod(tb - ta, 2.0 * M_PI);
            if (fabs(dth - angle) > 1E-4)
                return fail("Periodicity check failed at (i,j)=(%ld,%ld)", i, j);
            if (fabs(transl) > 1e-6 && angle == 0.0) {
                if (fabs(b.z - a.z) > 1E-4) return fail("Axial translation mismatch at (%ld,%ld)", i, j);
            }
        }
    s->periodic = 1;
    return 0;
}

static int bc_type_of(const char* name, int* out) { /* boundaryTypeFromString, include/types.hpp:202-232 */
    char low[128];
    snprintf(low, sizeof low, "%s", name);
    for (char* p = low; *p; p++) *p = (char)tolower((unsigned char)*p);
    if (!strcmp(low, "inlet")) *out = BC_INLET;
    else if (!strcmp(low, "outlet")) *out = BC_OUTLET;
    else if (!strcmp(low, "radial_equilibrium")) *out = BC_RADIAL_EQ;
    else if (!strcmp(low, "inviscid_wall")) *out = BC_INVISCID_WALL;
    else if (!strcmp(low, "wedge")) *out = BC_WEDGE;
    else if (!strcmp(low, "periodic")) *out = BC_PERIODIC;
    else if (!strcmp(low, "throttle")) *out = BC_THROTTLE;
    else if (!strcmp(low, "empty")) *out = BC_EMPTY;
    else if (!strcmp(low, "inlet_supersonic")) *out = BC_INLET_SUPERSONIC;
    else if (!strcmp(low, "outlet_supersonic")) *out = BC_OUTLET_SUPERSONIC;
    else if (!strcmp(low, "mass_flow") || !strcmp(low, "outlet_mass_flow") || !strcmp(low, "massflow") ||
             !strcmp(low, "mass_flow_rate")) *out = BC_MASS_FLOW;
    else if (!strcmp(low, "transparent")) *out = BC_TRANSPARENT;
    else if (!strcmp(low, "farfield")) *out = BC_FARFIELD;
    else if (!strcmp(low, "no_slip_wall")) *out = BC_NO_SLIP_WALL;
    else return fail("Boundary type '%s' is not supported by the oracle", name);
    return 0;
}

static void dir_join(char* out, size_t n, const char* base_dir, const char* file) {
    if (file[0] == '/') snprintf(out, n, "%s", file);
    else snprintf(out, n, "%s/%s", base_dir, file);
}

/* Solver::readBoundaryFile + buildBoundaryDataStructures + map
 * (src/solver.cpp:224-561). */
static int read_boundaries(oracle_solver* s, const char* path) {
    FILE* f = fopen(path, "r");
    if (!f) return fail("Cannot open file: %s", path);
    char line[4096];
    int in_data = 0;
    while (fgets(line, sizeof line, f)) {
        trim(line, "\r\n");
        if (!line[0]) continue;
        if (strchr(line, '=')) continue;
        if (strstr(line, "PATCH_NAME")) { in_data = 1; continue; }
        if (!in_data) continue;
        patch p;
        memset(&p, 0, sizeof p);
        char* save = NULL;
        char* tok = strtok_r(line, ",", &save);
        if (!tok) continue;
        int w = 0;
        for (char* c = tok; *c; c++) if (*c != ' ') p.name[w++] = *c;
        p.name[w] = 0;
        long v[6];
        for (int q = 0; q < 6; q++) {
            tok = strtok_r(NULL, ",", &save);
            if (!tok) { fclose(f); return fail("bad boundary row for %s", p.name); }
            v[q] = atol(tok);
        }
        p.i_min = v[0]; p.i_max = v[1]; p.j_min = v[2]; p.j_max = v[3]; p.k_min = v[4]; p.k_max = v[5];
        char items[32][128];
        int ni = cfg_list(&s->cfg, p.name, items, 32);
        if (ni < 1) { fclose(f); return fail("Boundary info for %s is missing in configuration.", p.name); }
        if (bc_type_of(items[0], &p.type)) { fclose(f); return 1; }
        p.nvalues = 0;
        for (int q = 1; q < ni && q < 17; q++) {
            if (parse_double(items[q], &p.values[p.nvalues])) { fclose(f); return fail("Invalid float format for boundary value"); }
            p.nvalues++;
        }
        if (p.i_min == p.i_max) p.orientation = p.i_min == 0 ? BI_ISTART : BI_IEND;
        else if (p.j_min == p.j_max) p.orientation = p.j_min == 0 ? BI_JSTART : BI_JEND;
        else p.orientation = p.k_min == 0 ? BI_KSTART : BI_KEND;
        p.profile = -1;
        s->patches = (patch*)realloc(s->patches, sizeof(patch) * (s->npatches + 1));
        s->patches[s->npatches++] = p;
    }
    fclose(f);
    return 0;
}

static int build_boundary_structures(oracle_solver* s) {
    for (int m = 0; m < s->npatches; m++) {
        patch* p = &s->patches[m];
        if (p->type == BC_RADIAL_EQ || p->type == BC_THROTTLE || p->type == BC_MASS_FLOW) {
            /* Solver::buildBoundaryDataStructures (src/solver.cpp:296-345) */
            int radial = 1;
            if (p->type == BC_MASS_FLOW) {
                int can = p->i_min == p->i_max && p->i_min != 0 && p->j_max > p->j_min;
                if (p->nvalues >= 4) radial = p->values[3] > 0.5 && can;
                else radial = can && (s->topology == TOPO_AXI || s->bfm_active);
                if (p->nvalues < 1 || p->values[0] <= 0.0)
                    return fail("Target mass flow for boundary patch %s must be specified and positive.", p->name);
                if (p->i_min != p->i_max || p->i_min == 0)
                    return fail("mass-flow outlets on other than the i-end face are outside the oracle's scope");
            }
            if (p->i_min != p->i_max) return fail("Radial equilibrium only supported on j-k patches");
            if (p->i_min == 0) return fail("Radial equilibrium only supported to the last i-position");
            if (p->j_max <= p->j_min) return fail("Invalid boundary indices for radial equilibrium patch: %s", p->name);
            radial_profile rp;
            memset(&rp, 0, sizeof rp);
            rp.n = (int)(p->j_max - p->j_min);
            rp.nradius = radial ? rp.n : 0;
            rp.pressure = (double*)calloc(rp.n, sizeof(double));
            rp.radius = (double*)calloc(rp.n, sizeof(double));
            for (long j = p->j_min; j < p->j_max; j++) rp.radius[j - p->j_min] = node_radius(s, p->i_max - 1, j, 0);
            rp.patch = m;
            p->profile = s->nprofiles;
            s->profiles = (radial_profile*)realloc(s->profiles, sizeof(radial_profile) * (s->nprofiles + 1));
            s->profiles[s->nprofiles++] = rp;
        } else if (p->type == BC_PERIODIC) {
            double id = p->values[0];
            if (id == 0) {
                s->per_transl = p->values[1];
                s->per_angle_deg = p->values[2];
                if (s->per_angle_deg == 360.0) s->per_angle_deg = 0.0;
                s->per_angle_rad = s->per_angle_deg * M_PI / 180.0;
                if (check_periodicity(s, s->per_transl, s->per_angle_rad)) return 1;
            }
            if (p->k_min != p->k_max) return fail("Periodic boundary only supported on i-j patches");
            if (p->i_min != 0 || p->j_min != 0 || p->i_max != s->ni || p->j_max != s->nj)
                return fail("Periodic boundary only supported on full i-j patches");
            if (p->k_min == 0 && id != 0) return fail("Periodic boundary with i_min=0 must have boundary id 0");
        }
    }
    s->mapI = (int*)malloc(sizeof(int) * 2 * s->nj * s->nk);
    s->mapJ = (int*)malloc(sizeof(int) * s->ni * 2 * s->nk);
    s->mapK = (int*)malloc(sizeof(int) * s->ni * s->nj * 2);
    for (long q = 0; q < 2 * s->nj * s->nk; q++) s->mapI[q] = -1;
    for (long q = 0; q < s->ni * 2 * s->nk; q++) s->mapJ[q] = -1;
    for (long q = 0; q < s->ni * s->nj * 2; q++) s->mapK[q] = -1;
    for (int m = 0; m < s->npatches; m++) {
        const patch* p = &s->patches[m];
        if (p->i_min == p->i_max) {
            long t = p->i_min == 0 ? 0 : 1;
            for (long j = p->j_min; j < p->j_max; j++)
                for (long k = p->k_min; k < p->k_max; k++) s->mapI[(t * s->nj + j) * s->nk + k] = m;
        } else if (p->j_min == p->j_max) {
            long t = p->j_min == 0 ? 0 : 1;
            for (long i = p->i_min; i < p->i_max; i++)
                for (long k = p->k_min; k < p->k_max; k++) s->mapJ[(i * 2 + t) * s->nk + k] = m;
        } else if (p->k_min == p->k_max) {
            long t = p->k_min == 0 ? 0 : 1;
            for (long i = p->i_min; i < p->i_max; i++)
                for (long j = p->j_min; j < p->j_max; j++) s->mapK[(i * s->nj + j) * 2 + t] = m;
        } else {
            return fail("Invalid boundary definition: %s", p->name);
        }
    }
    /* checkBoundaryConditionsMap (src/solver.cpp:565-593) */
    for (long q = 0; q < 2 * s->nj * s->nk; q++) if (s->mapI[q] < 0) return fail("Missing boundary condition (I)");
    if (s->topology != TOPO_1D)
        for (long q = 0; q < s->ni * 2 * s->nk; q++) if (s->mapJ[q] < 0) return fail("Missing boundary condition (J)");
    if (s->topology == TOPO_3D)
        for (long q = 0; q < s->ni * s->nj * 2; q++) if (s->mapK[q] < 0) return fail("Missing boundary condition (K)");
    return 0;
}

/* setTransportProperties of FluidIdeal (src/fluid_ideal.cpp:209-222) and
 * FluidReal (src/fluid_real.cpp:378-385) with Config::getViscosityModel and
 * getFluidMuConstant (src/config.cpp:575-598); FluidReal's viscosity stays at
 * its 2.0e-5 default unless the model is constant. */
static int read_transport(oracle_solver* s) {
    config* c = &s->cfg;
    const char* m = cfg_get(c, "FLUID_VISCOSITY_MODEL");
    int has_mu = cfg_get(c, "FLUID_MU_CONSTANT") || cfg_get(c, "FLUID_CONSTANT_MU");
    if (!m || !strcmp(m, "None")) s->visc_const = has_mu;
    else {
        char low[128];
        snprintf(low, sizeof low, "%s", m);
        for (char* q = low; *q; q++) *q = (char)tolower((unsigned char)*q);
        if (!strcmp(low, "sutherland")) s->visc_const = 0;
        else if (!strcmp(low, "constant")) s->visc_const = 1;
        else return fail("Unknown ViscosityModel: %s. Supported options: Sutherland, Constant.", m);
    }
    if (s->visc_const) {
        const char* k = cfg_get(c, "FLUID_MU_CONSTANT") ? "FLUID_MU_CONSTANT"
                        : cfg_get(c, "FLUID_CONSTANT_MU") ? "FLUID_CONSTANT_MU"
                        : cfg_get(c, "FLUID_SUTHERLAND_MU_REF") ? "FLUID_SUTHERLAND_MU_REF" : NULL;
        if (!k) return fail("Missing constant viscosity value: please specify \"FLUID_MU_CONSTANT\" in configuration.");
        if (cfg_float(c, k, &s->mu_const)) return 1;
    } else if (s->real) {
        s->visc_const = 1;
        s->mu_const = 2.0e-5;
    } else if (cfg_float(c, "FLUID_SUTHERLAND_MU_REF", &s->suth_mu) || cfg_float(c, "FLUID_SUTHERLAND_T_REF", &s->suth_T) ||
               cfg_float(c, "FLUID_SUTHERLAND_S", &s->suth_S)) {
        return 1;
    }
    if (cfg_float(c, "FLUID_CP", &s->vcp) || cfg_float(c, "FLUID_PRANDTL_NUMBER", &s->vpr)) return 1;
    return 0;
}

/* Solver::buildBoundaryFluxes (src/solver.cpp:369-388) with
 * fetchBoundaryNodesIndexRange (src/boundary_base.cpp:227-267): the nodes of
 * every no-slip wall patch; a moving wall is outside the oracle. */
static int build_wall_mask(oracle_solver* s) {
    s->wall = (unsigned char*)calloc(s->n, 1);
    for (int m = 0; m < s->npatches; m++) {
        const patch* p = &s->patches[m];
        if (p->type != BC_NO_SLIP_WALL) continue;
        if (p->nvalues > 0 && (p->nvalues < 3 || p->values[0] != 0.0 || p->values[1] != 0.0 || p->values[2] != 0.0))
            return fail("moving no-slip walls are outside the oracle's scope (patch %s)", p->name);
        long i0 = p->i_min, i1 = p->i_max, j0 = p->j_min, j1 = p->j_max, k0 = p->k_min, k1 = p->k_max;
        if (i0 == i1 && i0 == 0) i1 = 1;
        else if (i0 == i1 && i0 == s->ni) { i0 = s->ni - 1; i1 = i0 + 1; }
        else if (j0 == j1 && j0 == 0) j1 = 1;
        else if (j0 == j1 && j0 == s->nj) { j0 = s->nj - 1; j1 = j0 + 1; }
        else if (k0 == k1 && k0 == 0) k1 = 1;
        else if (k0 == k1 && k0 == s->nk) { k0 = s->nk - 1; k1 = k0 + 1; }
        else return fail("Invalid indexing on boundary condition specs for patch %s", p->name);
        for (long i = i0; i < i1; i++)
            for (long j = j0; j < j1; j++)
                for (long k = k0; k < k1; k++) s->wall[idx3(s, i, j, k)] = 1;
    }
    for (int v = 0; v < 4; v++) {
        s->grad[v] = (vec3*)calloc(s->n, sizeof(vec3));
        s->gfield[v] = (double*)calloc(s->n, sizeof(double));
    }
    return 0;
}

/* Config::isTurbulenceActive / getTurbulenceModel (src/config.cpp:165-207)
 * and the settings TurbulenceModelSA reads (include/config.hpp:126-133, 229,
 * 377). The oracle restates SA for ideal-gas, viscous runs started from the
 * initial field. */
static int read_turbulence(oracle_solver* s) {
    config* c = &s->cfg;
    int turb = 0;
    if (cfg_bool(c, "TURBULENCE_ACTIVE", 0, &turb)) return 1;
    s->sa = 0;
    if (!turb) return 0;
    const char* m = cfg_get(c, "TURBULENCE_MODEL");
    if (!m) return fail("Not found value for key \"TURBULENCE_MODEL\" in configuration.");
    if (!strcmp(m, "None")) return 0;
    if (strcmp(m, "SA")) return fail("Invalid value for key \"TURBULENCE_MODEL\" in configuration.");
    if (!s->viscous) return fail("the Spalart-Allmaras model needs VISCOSITY_ACTIVE in the oracle");
    if (s->real) return fail("the Spalart-Allmaras model with FLUID_MODEL = real is outside the oracle's scope");
    int restart = 0;
    if (cfg_bool(c, "RESTART_SOLUTION", 0, &restart)) return 1;
    if (restart) return fail("a restarted Spalart-Allmaras field is outside the oracle's scope");
    s->sa = 1;
    if (cfg_float_def(c, "TURBULENT_PRANDTL_NUMBER", 0.86, &s->sa_prt)) return 1;
    if (cfg_float_def(c, "IMPLICIT_UNDER_RELAXATION", 1.0, &s->sa_relax)) return 1;
    return 0;
}

/* reconstructNuTildeFromEddyViscosity (src/math_utils.cpp:641-675): nu hat
 * whose fv1 nu hat rho equals mu_t (Newton on chi^4 - y chi^3 - cv1^3 y). */
static double sa_nutilde_of_eddy(double mu_t, double mu_L, double rho) {
    if (mu_t <= 0.0 || mu_L <= 0.0 || rho <= 0.0) return 0.0;
    double nu = mu_L / rho;
    double y = mu_t / mu_L;
    double cv1_3 = SA_CV1 * SA_CV1 * SA_CV1;
    double cv1_3_y = cv1_3 * y;
    double chi = dmax(y, pow(cv1_3_y, 0.25));
    for (int it = 0; it < 12; ++it) {
        double chi2 = chi * chi;
        double chi3 = chi2 * chi;
        double chi4 = chi3 * chi;
        double f = chi4 - y * chi3 - cv1_3_y;
        double df = 4.0 * chi3 - 3.0 * y * chi2;
        if (fabs(df) < 1e-14) break;
        double delta = f / df;
        chi -= delta;
        if (fabs(delta) < 1e-10 * (1.0 + chi)) break;
    }
    return dmax(0.0, chi * nu);
}

/* Solver::computeWallDistance / computeMinimumDistanceToBoundary
 * (src/solver.cpp:657-698): per node the least distance to a node of a
 * no-slip wall patch; TurbulenceModelSA::setupInitialValues /
 * initializeFromZero (src/turbulence_model_sa.cpp:32-71): nu hat = scaling
 * mu(T_init) / rho(p_init, T_init) everywhere. */
static int setup_sa(oracle_solver* s) {
    if (!s->sa) return 0;
    config* c = &s->cfg;
    s->nuhat = (double*)calloc(s->n, sizeof(double));
    s->nul = (double*)calloc(s->n, sizeof(double));
    s->wdist = (double*)calloc(s->n, sizeof(double));
    s->sa_res = (double*)calloc(s->n, sizeof(double));
    s->sa_diag = (double*)calloc(s->n, sizeof(double));
    s->sa_dstar = (double*)calloc(s->n, sizeof(double));
    s->sa_dnu = (double*)calloc(s->n, sizeof(double));
    s->nuhat_grad = (vec3*)calloc(s->n, sizeof(vec3));
    s->sa_vel = (vec3*)calloc(s->n, sizeof(vec3));
    for (long q = 0; q < s->n; q++) {
        double mn = 1.0E9;
        for (int m = 0; m < s->npatches; m++) {
            const patch* p = &s->patches[m];
            if (p->type != BC_NO_SLIP_WALL) continue;
            long r[6], st[3];
            patch_nodes(s, p, r, st);
            double pm = 1.0E9;
            for (long ib = r[0]; ib < r[1]; ib++)
                for (long jb = r[2]; jb < r[3]; jb++)
                    for (long kb = r[4]; kb < r[5]; kb++) {
                        vec3 a = s->vert[q], b = s->vert[idx3(s, ib, jb, kb)];
                        double dx = a.x - b.x, dy = a.y - b.y, dz = a.z - b.z;
                        double dd = sqrt(dx * dx + dy * dy + dz * dz);
                        if (dd < pm) pm = dd;
                    }
            if (pm < mn) mn = pm;
        }
        s->wdist[q] = mn;
    }
    double T, p;
    if (cfg_float(c, "INIT_TEMPERATURE", &T) || cfg_float(c, "INIT_PRESSURE", &p)) return 1;
    double rho = p / (s->rgas * T);
    s->sa_init_nu = f_mu(s, T) / rho;
    if (cfg_get(c, "TURBULENCE_NU_TILDE_RATIO")) {
        if (cfg_float(c, "TURBULENCE_NU_TILDE_RATIO", &s->sa_ff_scale)) return 1;
    } else if (cfg_get(c, "TURBULENCE_EDDY_VISCOSITY_RATIO")) {
        double ratio;
        if (cfg_float(c, "TURBULENCE_EDDY_VISCOSITY_RATIO", &ratio)) return 1;
        s->sa_ff_scale = sa_nutilde_of_eddy(ratio, 1.0, 1.0);
    } else {
        s->sa_ff_scale = 3.0;
    }
    if (cfg_get(c, "TURBULENCE_INIT_NU_TILDE_RATIO")) {
        if (cfg_float(c, "TURBULENCE_INIT_NU_TILDE_RATIO", &s->sa_init_scale)) return 1;
    } else {
        s->sa_init_scale = s->sa_ff_scale;
    }
    for (long q = 0; q < s->n; q++) s->nuhat[q] = s->sa_init_scale * s->sa_init_nu;
    return 0;
}

static int read_settings(oracle_solver* s) {
    config* c = &s->cfg;
    const char* v;
    v = cfg_get(c, "TOPOLOGY");
    if (!v) return fail("Not found value for key \"TOPOLOGY\" in configuration.");
    if (!strcmp(v, "2D") || !strcmp(v, "2d")) s->topology = TOPO_2D;
    else if (!strcmp(v, "3D") || !strcmp(v, "3d")) s->topology = TOPO_3D;
    else if (!strcmp(v, "axisymmetric") || !strcmp(v, "Axisymmetric") || !strcmp(v, "AXISYMMETRIC")) s->topology = TOPO_AXI;
    else if (!strcmp(v, "1D") || !strcmp(v, "1d")) s->topology = TOPO_1D;
    else return fail("Invalid value for key \"TOPOLOGY\" in configuration.");
    if (s->topology == TOPO_1D) return fail("1-D topology is outside the oracle's scope");

    v = cfg_get(c, "CONVECTION_SCHEME");
    if (!v) return fail("Not found value for key \"CONVECTION_SCHEME\" in configuration.");
    if (!strcmp(v, "JST")) s->scheme = SCHEME_JST;
    else if (!strcmp(v, "ROE") || !strcmp(v, "roe") || !strcmp(v, "Roe")) s->scheme = SCHEME_ROE;
    else return fail("Invalid value for key \"CONVECTION_SCHEME\" in configuration.");
    if (cfg_bool(c, "MUSCL_RECONSTRUCTION", 0, &s->muscl)) return 1;
    v = cfg_get(c, "FLUX_LIMITER");
    if (!v || !strcmp(v, "None")) s->limiter = LIM_NONE;
    else if (!strcmp(v, "van albada")) s->limiter = LIM_VAN_ALBADA;
    else if (!strcmp(v, "van leer")) s->limiter = LIM_VAN_LEER;
    else if (!strcmp(v, "min mod")) s->limiter = LIM_MIN_MOD;
    else return fail("Invalid value for key \"FLUX_LIMITER\" in configuration.");

    /* Config::getTimeIntegration (src/config.cpp:250-276) */
    const char* tik = cfg_get(c, "TIME_INTEGRATION") ? "TIME_INTEGRATION" : "TIME_INTEGRATION_TYPE";
    v = cfg_get(c, tik);
    char ti[64] = "0";
    if (v) {
        int w = 0;
        for (const char* p = v; *p && w < 63; p++)
            if (!isspace((unsigned char)*p)) ti[w++] = (char)tolower((unsigned char)*p);
        ti[w] = 0;
    }
    if (!strcmp(ti, "0") || !strcmp(ti, "explicit_rk4") || !strcmp(ti, "rk4") || !strcmp(ti, "runge_kutta_4")) {
        s->nstages = 4;
        s->coeffs[0] = 1.0 / 4.0; s->coeffs[1] = 5.0 / 14.0; s->coeffs[2] = 14.0 / 25.0; s->coeffs[3] = 1.0;
    } else if (!strcmp(ti, "1") || !strcmp(ti, "explicit_rk3") || !strcmp(ti, "rk3") || !strcmp(ti, "runge_kutta_3")) {
        s->nstages = 3;
        s->coeffs[0] = 8.0 / 17.0; s->coeffs[1] = 17.0 / 20.0; s->coeffs[2] = 1.0;
    } else {
        return fail("Only the explicit Runge-Kutta integrators are in the oracle's scope");
    }

    v = cfg_get(c, "TIME_STEP_METHOD");
    if (!v) return fail("Not found value for key \"TIME_STEP_METHOD\" in configuration.");
    if (!strcmp(v, "local")) s->dt_method = DT_LOCAL;
    else if (!strcmp(v, "global")) s->dt_method = DT_GLOBAL;
    else if (!strcmp(v, "fixed")) s->dt_method = DT_FIXED;
    else return fail("Invalid value for key \"TIME_STEP_METHOD\" in configuration.");
    /* Config::getCFL (include/config.hpp:124-133) */
    if (cfg_get(c, "CFL")) { if (cfg_float(c, "CFL", &s->cfl)) return 1; }
    else if (cfg_get(c, "CFL_START")) { if (cfg_float(c, "CFL_START", &s->cfl)) return 1; }
    else if (cfg_get(c, "CFL_MAX")) { if (cfg_float(c, "CFL_MAX", &s->cfl)) return 1; }
    else if (cfg_float(c, "CFL", &s->cfl)) return 1;
    if (s->dt_method == DT_FIXED && cfg_float(c, "FIXED_TIME_STEP", &s->fixed_dt)) return 1;

    if (cfg_bool(c, "VISCOSITY_ACTIVE", 0, &s->viscous)) return 1;
    v = cfg_get(c, "FLUID_MODEL");
    if (v && (!strcmp(v, "real") || !strcmp(v, "Real") || !strcmp(v, "REAL"))) {
        s->real = 1; /* the table is loaded by oracle_create, next to the ini */
        int stop = 0, regen = 0;
        if (cfg_bool(c, "STOP_ON_TABLE_OUT_OF_BOUNDS", 0, &stop)) return 1;
        if (stop) return fail("STOP_ON_TABLE_OUT_OF_BOUNDS is outside the oracle's scope");
        if (cfg_bool(c, "FLUID_TABLE_FORCE_REGENERATE", 0, &regen)) return 1;
        if (regen) return fail("Table regeneration is outside the oracle's scope");
    } else if (v && strcmp(v, "None") && strcmp(v, "Ideal") && strcmp(v, "ideal") && strcmp(v, "IDEAL")) {
        return fail("Invalid value for key \"FLUID_MODEL\" in configuration.");
    } else {
        if (cfg_float(c, "FLUID_GAMMA", &s->gamma)) return 1;
        if (cfg_float(c, "FLUID_R_CONSTANT", &s->rgas)) return 1;
        s->cp = (s->gamma * s->rgas) / (s->gamma - 1);
    }
    if (s->viscous && read_transport(s)) return 1;
    if (read_turbulence(s)) return 1;

    if (cfg_bool(c, "SIMULATION_IS_STEADY", 1, &s->steady)) return 1;
    if (cfg_int_def(c, "RESIDUALS_DROP_CONVERGENCE", 16, &s->drop)) return 1;
    if (cfg_float(c, "INIT_PRESSURE", &s->init_p)) return 1;
    if (cfg_float_def(c, "OUTLET_PRESSURE_RAMP_ITERATIONS", 0.0, &s->ramp_iters)) return 1;
    v = cfg_get(c, "INLET_REFERENCE_FRAME");
    if (!v || !strcmp(v, "Cartesian") || !strcmp(v, "cartesian") || !strcmp(v, "CARTESIAN") || !strcmp(v, "None")) s->inlet_cyl = 0;
    else if (!strcmp(v, "Cylindrical") || !strcmp(v, "cylindrical") || !strcmp(v, "CYLINDRICAL")) s->inlet_cyl = 1;
    else return fail("Invalid value for key \"INLET_REFERENCE_FRAME\" in configuration.");

    /* BFM (src/config.cpp:166-190, include/config.hpp) */
    if (cfg_bool(c, "BFM_ACTIVE", 0, &s->bfm_active)) return 1;
    if (cfg_bool(c, "BLOCKAGE_ACTIVE", 0, &s->blockage_active)) return 1;
    v = cfg_get(c, "BFM_MODEL");
    if (!v || !strcmp(v, "None")) s->bfm_model = BFM_NONE;
    else if (!strcmp(v, "Hall")) s->bfm_model = BFM_HALL;
    else if (!strcmp(v, "Hall-Thollet")) s->bfm_model = BFM_THOLLET;
    else if (!strcmp(v, "Lift-Drag")) s->bfm_model = BFM_LIFT_DRAG;
    else if (!strcmp(v, "Blockage")) s->bfm_model = BFM_BLOCKAGE;
    else if (!strcmp(v, "Chima")) s->bfm_model = BFM_CHIMA;
    else if (!strcmp(v, "Correlations")) s->bfm_model = BFM_CORRELATIONS;
    else return fail("BFM_MODEL '%s' is outside the oracle's scope", v);
    if (cfg_bool(c, "STALLED_BFM_ACTIVE", 0, &s->stalled)) return 1;
    if (cfg_bool(c, "PERTURBATION_BODY_FORCE", 0, &s->perturb)) return 1;
    if (cfg_float_def(c, "ROTATIONAL_SPEED_SCALING_FACTOR", 1.0, &s->speed_scale)) return 1;
    if (cfg_bool(c, "ACCELERATION_ACTIVE", 0, &s->accel)) return 1;
    if (s->accel) {
        if (s->dt_method != DT_FIXED) return fail("Rotational speed scaling factor is only active for fixed time step method");
        if (cfg_float(c, "ACCELERATION_INITIAL_TIME", &s->acc_t0) || cfg_float(c, "ACCELERATION_FINAL_TIME", &s->acc_t1) ||
            cfg_float(c, "ROTATIONAL_SPEED_SCALING_FACTOR_INITIAL", &s->acc_s0) ||
            cfg_float(c, "ROTATIONAL_SPEED_SCALING_FACTOR_FINAL", &s->acc_s1))
            return 1;
    }
    if (s->perturb) {
        char items[8][128];
        if (cfg_list(c, "PERTURBATION_CENTER", items, 8) < 3) return fail("PERTURBATION_CENTER needs 3 values");
        for (int q = 0; q < 3; q++) parse_double(items[q], &s->pert_center[q]);
        if (cfg_float(c, "PERTURBATION_RADIAL_EXTENSION", &s->pert_radius) ||
            cfg_float(c, "PERTURBATION_SCALING_FACTOR", &s->pert_scale) ||
            cfg_float(c, "PERTURBATION_TIME_START", &s->pert_t0) ||
            cfg_float(c, "PERTURBATION_TIME_DURATION", &s->pert_dur))
            return 1;
    }
    if (s->bfm_model == BFM_THOLLET) {
        if (cfg_float(c, "HALL_THOLLET_COEFFICIENT_KN", &s->kn) || cfg_float(c, "HALL_THOLLET_COEFFICIENT_KF", &s->kf) ||
            cfg_float(c, "HALL_THOLLET_COEFFICIENT_KD", &s->kd))
            return 1;
        v = cfg_get(c, "HALL_THOLLET_OFF_DESIGN_ACTIVE");
        if (!v) return fail("Not found value for key \"HALL_THOLLET_OFF_DESIGN_ACTIVE\" in configuration.");
        if (!strcmp(v, "true") || !strcmp(v, "yes") || !strcmp(v, "1")) s->offdesign = 1;
        else if (!strcmp(v, "false") || !strcmp(v, "no") || !strcmp(v, "0")) s->offdesign = 0;
        else return fail("Invalid value for key \"HALL_THOLLET_OFF_DESIGN_ACTIVE\" in configuration.");
        s->has_nu = cfg_get(c, "FLUID_KINEMATIC_VISCOSITY") != NULL;
        if (!s->has_nu) return fail("Hall-Thollet without FLUID_KINEMATIC_VISCOSITY is outside the oracle's scope");
        if (cfg_float(c, "FLUID_KINEMATIC_VISCOSITY", &s->nu)) return 1;
    }
    if (s->bfm_model == BFM_CORRELATIONS && cfg_float(c, "KN_CORRELATION_BFM_COEFFICIENT", &s->kn)) return 1;
    if (s->bfm_model == BFM_LIFT_DRAG || s->bfm_model == BFM_CHIMA || s->bfm_model == BFM_CORRELATIONS) {
        int le, te;
        double d;
        if (cfg_float(c, "LEADING_EDGE_INDEX", &d)) return 1;
        le = (int)d;
        if (cfg_float(c, "TRAILING_EDGE_INDEX", &d)) return 1;
        te = (int)d;
        s->le_idx = le; s->te_idx = te;
    }
    int turbo_out = 0;
    if (cfg_bool(c, "TURBO_OUTPUT", 0, &turbo_out)) return 1;
    if (cfg_bool(c, "ENABLE_GREITZER_MODELING", 0, &s->greitzer)) return 1;
    if (s->greitzer && s->dt_method != DT_FIXED) return fail("Greitzer modeling is only compatible with fixed time step method");
    if (s->greitzer) {
        if (cfg_get(c, "GREITZER_PLENUM_VOLUME")) { if (cfg_float(c, "GREITZER_PLENUM_VOLUME", &s->plenum_volume)) return 1; }
        else if (cfg_float(c, "GREITZER_PENUM_VOLUME", &s->plenum_volume)) return 1;
        if (cfg_float_def(c, "GREITZER_AMBIENT_PRESSURE", 101325.0, &s->ambient_p)) return 1;
    }
    s->need_turbo = turbo_out || s->greitzer;
    return 0;
}

/* Solver::updateTurboPerformance's inlet-orientation default
 * (src/solver.cpp:1654-1680). */
static void resolve_turbo_dir(oracle_solver* s) {
    const char* v = cfg_get(&s->cfg, "TURBO_DIRECTION");
    const char* d = v ? v : "i";
    if (!v) {
        for (int m = 0; m < s->npatches; m++)
            if (s->patches[m].type == BC_INLET || s->patches[m].type == BC_INLET_SUPERSONIC) {
                if (s->patches[m].orientation == BI_JSTART) { d = "j"; break; }
                if (s->patches[m].orientation == BI_JEND) { d = "-j"; break; }
            }
    }
    if (!strcmp(d, "-i")) s->turbo_dir = 1;
    else if (!strcmp(d, "j") || !strcmp(d, "+j")) s->turbo_dir = 2;
    else if (!strcmp(d, "-j")) s->turbo_dir = 3;
    else s->turbo_dir = 0;
}

/* ------------------------------------------------------------------ restart */
/* Solver::initializeSolutionFromRestart (src/solver.cpp:890-966) with
 * readRestartFile (:1155-1295), standardRestart (:968-1000),
 * axisymmetricRestart (:1002-1035) and nearestNeighborRestart (:1037-1153).
 * The nearest node is found by exhaustive search, the first of equal
 * distances in file order; the reference's k-d tree may pick another of
 * several exactly equidistant nodes, so the oracle meets the reference on
 * inputs without such ties (tie resolution is pinned by the golden fixtures
 * made with the reference build). */
typedef struct {
    long ni, nj, nk;
    vec3* xyz;
    double *rho, *vx, *vy, *vz, *T;
} restart_data;

static void restart_free(restart_data* r) {
    free(r->xyz); free(r->rho); free(r->vx); free(r->vy); free(r->vz); free(r->T);
    memset(r, 0, sizeof *r);
}

static char* trim_ws(char* t) {
    while (*t == ' ' || *t == '\t' || *t == '\r' || *t == '\n') t++;
    size_t n = strlen(t);
    while (n && (t[n - 1] == ' ' || t[n - 1] == '\t' || t[n - 1] == '\r' || t[n - 1] == '\n')) t[--n] = 0;
    return t;
}

/* FluidIdeal::computePressure_rho_T (src/fluid_ideal.cpp:66-68),
 * FluidReal::computePressure_rho_T (src/fluid_real.cpp:262-277) */
static double f_pressure_rho_T(const oracle_solver* s, double rho, double T) {
    if (s->real) {
        const table2d* tT = &s->lut->T;
        double eLo = tT->ymin, eHi = tT->ymax;
        for (int it = 0; it < 25; ++it) {
            double eMid = 0.5 * (eLo + eHi);
            if (table_interp(tT, rho, eMid) < T) eLo = eMid; else eHi = eMid;
        }
        return table_interp(&s->lut->p, rho, 0.5 * (eLo + eHi));
    }
    return rho * s->rgas * T;
}

static int restart_read(const oracle_solver* s, const char* path, restart_data* r) {
    memset(r, 0, sizeof *r);
    FILE* f = fopen(path, "r");
    if (!f) return fail("Failed to open restart file: %s", path);
    char* line = NULL;
    size_t cap = 0;
    long* dims[3] = {&r->ni, &r->nj, &r->nk};
    for (int d = 0; d < 3; d++) {
        char* eq;
        if (getline(&line, &cap, f) < 0 || !(eq = strchr(line, '='))) {
            free(line); fclose(f);
            return fail("Restart file %s lacks its NI/NJ/NK lines", path);
        }
        *dims[d] = strtol(eq + 1, NULL, 10);
    }
    if (getline(&line, &cap, f) < 0) { free(line); fclose(f); return fail("Restart file %s lacks its header", path); }
    long ix = -1, iy = -1, iz = -1, need[5] = {-1, -1, -1, -1, -1};
    const char* names[5] = {"Density", "Velocity X", "Velocity Y", "Velocity Z", "Total Energy"};
    {
        long c = 0;
        char* save = NULL;
        for (char* tok = strtok_r(line, ",", &save); tok; tok = strtok_r(NULL, ",", &save), c++) {
            char* t = trim_ws(tok);
            if (!strcmp(t, "x") || (!strcmp(t, "X") && ix < 0)) ix = c;
            if (!strcmp(t, "y") || (!strcmp(t, "Y") && iy < 0)) iy = c;
            if (!strcmp(t, "z") || (!strcmp(t, "Z") && iz < 0)) iz = c;
            for (int v = 0; v < 5; v++) if (!strcmp(t, names[v])) need[v] = c;
        }
    }
    for (int v = 0; v < 5; v++)
        if (need[v] < 0) { free(line); fclose(f); return fail("Restart file %s has no \"%s\" column", path, names[v]); }
    long n = r->ni * r->nj * r->nk;
    r->xyz = (vec3*)calloc(n > 0 ? n : 1, sizeof(vec3));
    double** arr[5] = {&r->rho, &r->vx, &r->vy, &r->vz, &r->T};
    for (int v = 0; v < 5; v++) *arr[v] = (double*)calloc(n > 0 ? n : 1, sizeof(double));
    long row = 0, i = 0, j = 0, k = 0;
    double vals[256];
    while (getline(&line, &cap, f) >= 0) {
        if (!*trim_ws(line)) continue;
        if (row >= n) { free(line); fclose(f); return fail("Restart file %s has more rows than NI*NJ*NK", path); }
        long nv = 0;
        char* save = NULL;
        for (char* tok = strtok_r(line, ",", &save); tok && nv < 256; tok = strtok_r(NULL, ",", &save)) {
            double v = strtod(tok, NULL);
            if (isnan(v) || isinf(v)) {
                free(line); fclose(f);
                return fail("Corrupted restart file '%s': NaN or Inf encountered at row index (%ld,%ld,%ld).", path, i, j, k);
            }
            vals[nv++] = v;
        }
        for (int v = 0; v < 5; v++) if (need[v] >= nv) { free(line); fclose(f); return fail("short restart row"); }
        if (ix >= 0 && iy >= 0 && iz >= 0 && ix < nv && iy < nv && iz < nv) r->xyz[row] = v3(vals[ix], vals[iy], vals[iz]);
        double rho = vals[need[0]];
        vec3 u = v3(vals[need[1]], vals[need[2]], vals[need[3]]);
        r->rho[row] = rho; r->vx[row] = u.x; r->vy[row] = u.y; r->vz[row] = u.z;
        r->T[row] = f_temperature_rho_u_et(s, rho, u, vals[need[4]]);
        row++;
        if (++k == r->nk) { k = 0; if (++j == r->nj) { j = 0; ++i; } }
    }
    free(line);
    fclose(f);
    if (row != n) return fail("Restart file %s has %ld rows, NI*NJ*NK = %ld", path, row, n);
    return 0;
}

static vec3 rotate_x(vec3 v, double th) { /* rotateVectorAlongXAxis (src/math_utils.cpp:109-115) */
    return v3(v.x, v.y * cos(th) - v.z * sin(th), v.y * sin(th) + v.z * cos(th));
}

static void restart_node(oracle_solver* s, long q, double rho, vec3 v, double T) {
    s->U[0][q] = rho;
    s->U[1][q] = rho * v.x;
    s->U[2][q] = rho * v.y;
    s->U[3][q] = rho * v.z;
    double p = f_pressure_rho_T(s, rho, T);
    double e = f_static_energy_p_rho(s, p, rho);
    double et = e + 0.5 * (v.x * v.x + v.y * v.y + v.z * v.z);
    s->U[4][q] = rho * et;
}

static int restart_solution(oracle_solver* s, const char* base) {
    const char* file = cfg_get(&s->cfg, "RESTART_SOLUTION_FILEPATH");
    if (!file) return fail("Not found value for key \"RESTART_SOLUTION_FILEPATH\" in configuration.");
    char path[4096];
    dir_join(path, sizeof path, base, file);
    restart_data r;
    if (restart_read(s, path, &r)) { restart_free(&r); return 1; }
    const char* type = cfg_get(&s->cfg, "RESTART_TYPE");
    if (!type) type = "None";
    int nearest = !strcmp(type, "nearest_neighbor") || !strcmp(type, "nearest_neighbor_axisymmetric");
    if (!nearest && (r.ni != s->ni || r.nj != s->nj || r.nk != s->nk)) {
        if (r.ni == s->ni && r.nj == s->nj && !strcmp(type, "axisymmetric")) {
            for (long i = 0; i < s->ni; i++)
                for (long j = 0; j < s->nj; j++)
                    for (long k = 0; k < s->nk; k++) {
                        vec3 a = s->vert[idx3(s, i, j, 0)], b = s->vert[idx3(s, i, j, k)];
                        double rot = atan2_0_2pi(b.z, b.y) - atan2_0_2pi(a.z, a.y);
                        long src = (i * r.nj + j) * r.nk;
                        vec3 vel = rotate_x(v3(r.vx[src], r.vy[src], r.vz[src]), rot);
                        restart_node(s, idx3(s, i, j, k), r.rho[src], vel, r.T[src]);
                    }
            restart_free(&r);
            return 0;
        }
        if (!strcmp(type, "standard")) {
            fail("Restart file dimensions (%ld,%ld,%ld) do not match solver dimensions (%ld,%ld,%ld) and "
                 "RESTART_TYPE=standard was requested.", r.ni, r.nj, r.nk, s->ni, s->nj, s->nk);
            restart_free(&r);
            return 1;
        }
        nearest = 1;
    }
    if (!nearest) {
        for (long q = 0; q < s->n; q++) restart_node(s, q, r.rho[q], v3(r.vx[q], r.vy[q], r.vz[q]), r.T[q]);
        restart_free(&r);
        return 0;
    }
    long n = r.ni * r.nj * r.nk;
    if (n == 0) { restart_free(&r); return fail("Cannot perform nearest-neighbor restart: restart data is empty."); }
    int axi = !strcmp(type, "axisymmetric") || !strcmp(type, "nearest_neighbor_axisymmetric") ||
              s->topology == TOPO_AXI || (r.nk == 1 && s->nk > 1 && s->periodic);
    for (long q = 0; q < s->n; q++) {
        vec3 p = s->vert[q];
        double x0 = p.x, x1 = axi ? sqrt(p.y * p.y + p.z * p.z) : p.y, x2 = p.z;
        long best = 0;
        double bd = DBL_MAX;
        for (long m = 0; m < n; m++) {
            vec3 c = r.xyz[m];
            double c1 = axi ? sqrt(c.y * c.y + c.z * c.z) : c.y;
            double d0 = x0 - c.x, d1 = x1 - c1, d2 = 0.0;
            double dd = 0.0;
            dd += d0 * d0;
            dd += d1 * d1;
            if (!axi) { d2 = x2 - c.z; dd += d2 * d2; }
            if (dd < bd) { bd = dd; best = m; }
        }
        vec3 vel = v3(r.vx[best], r.vy[best], r.vz[best]);
        if (axi) {
            vec3 c = r.xyz[best];
            vel = rotate_x(vel, atan2_0_2pi(p.z, p.y) - atan2_0_2pi(c.z, c.y));
        }
        restart_node(s, q, r.rho[best], vel, r.T[best]);
    }
    restart_free(&r);
    return 0;
}

/* FluidIdeal::computeInitFields (src/fluid_ideal.cpp:155-170) and
 * Solver::initializeSolutionFromScratch (src/solver.cpp:777-836). */
static int init_solution(oracle_solver* s, const char* base) {
    double M, T, p;
    if (cfg_float(&s->cfg, "INIT_MACH_NUMBER", &M) || cfg_float(&s->cfg, "INIT_TEMPERATURE", &T) ||
        cfg_float(&s->cfg, "INIT_PRESSURE", &p))
        return 1;
    int restart = 0;
    if (cfg_bool(&s->cfg, "RESTART_SOLUTION", 0, &restart)) return 1;
    if (restart) return restart_solution(s, base); /* Solver::initializeSolutionArrays (src/solver.cpp:783-789) */
    const char* raw = cfg_get(&s->cfg, "INIT_DIRECTION");
    int adaptive = 0;
    vec3 d0 = v3(0, 0, 0);
    if (raw && !strcmp(raw, "adaptive")) adaptive = 1;
    else {
        char items[8][128];
        int n = cfg_list(&s->cfg, "INIT_DIRECTION", items, 8);
        if (n != 3) return fail("INIT_DIRECTION must have 3 components or be 'adaptive'");
        parse_double(items[0], &d0.x); parse_double(items[1], &d0.y); parse_double(items[2], &d0.z);
        if (d0.x == 0.0 && d0.y == 0.0 && d0.z == 0.0) adaptive = 1;
    }
    for (long i = 0; i < s->ni; i++)
        for (long j = 0; j < s->nj; j++)
            for (long k = 0; k < s->nk; k++) {
                vec3 dir = d0;
                if (adaptive) { /* Mesh::computeAdaptiveFlowDirection (src/mesh.cpp:637-661) */
                    long ia = (i < s->ni - 1) ? i : s->ni - 2;
                    dir = vnormalized(vsub(s->vert[idx3(s, ia + 1, j, k)], s->vert[idx3(s, ia, j, k)]));
                }
                if (s->real) { /* FluidReal::computeInitFields (src/fluid_real.cpp:346-362) */
                    const lut* L = s->lut;
                    double rho = table_interp(&L->rho_pt, p, T);
                    double e = table_interp(&L->e_pt, p, T);
                    double a = table_interp(&L->a, rho, e);
                    double dm = vmag(dir);
                    vec3 dn = (dm > 1e-12) ? vdiv(dir, dm) : v3(1.0, 0.0, 0.0);
                    vec3 u = vmul(vmul(dn, a), M);
                    double et = e + 0.5 * vdot(u, u);
                    long q = idx3(s, i, j, k);
                    s->U[0][q] = rho;
                    s->U[1][q] = rho * u.x;
                    s->U[2][q] = rho * u.y;
                    s->U[3][q] = rho * u.z;
                    s->U[4][q] = rho * et;
                    continue;
                }
                double a = sqrt(s->gamma * s->rgas * T);
                vec3 u = vmul(vmul(vdiv(dir, vmag(dir)), a), M);
                double rho = p / (s->rgas * T);
                double e = f_static_energy_p_rho(s, p, rho);
                double um = vmag(u);
                double et = e + 0.5 * (um * um);
                long q = idx3(s, i, j, k);
                s->U[0][q] = rho;
                s->U[1][q] = rho * u.x;
                s->U[2][q] = rho * u.y;
                s->U[3][q] = rho * u.z;
                s->U[4][q] = rho * et;
            }
    return 0;
}

int oracle_create(const char* ini_path, oracle_solver** out) {
    *out = NULL;
    oracle_solver* s = (oracle_solver*)calloc(1, sizeof(oracle_solver));
    char base[4096], path[4096];
    snprintf(base, sizeof base, "%s", ini_path);
    char* slash = strrchr(base, '/');
    if (slash) *slash = 0; else snprintf(base, sizeof base, ".");
    if (cfg_load(&s->cfg, ini_path) || read_settings(s)) { oracle_destroy(s); return 1; }
    const char* grid = cfg_get(&s->cfg, "GRID_FILE");
    if (!grid) { fail("Not found value for key \"GRID_FILE\" in configuration."); oracle_destroy(s); return 1; }
    if (s->real) { /* Config::getFluidTableFile (src/config.cpp:492-497), relative to the ini */
        char tname[1024];
        const char* tf = cfg_get(&s->cfg, "FLUID_TABLE_FILE");
        const char* fname = cfg_get(&s->cfg, "FLUID_NAME");
        if (!fname) fname = cfg_get(&s->cfg, "FLUID");
        if (tf) snprintf(tname, sizeof tname, "%s", tf);
        else snprintf(tname, sizeof tname, "fluid_table_%s.lut", fname ? fname : "CO2");
        char tpath[4096];
        dir_join(tpath, sizeof tpath, base, tname);
        s->lut = (lut*)calloc(1, sizeof(lut));
        if (lut_load(s->lut, tpath)) { oracle_destroy(s); return 1; }
        s->gamma = s->lut->gnom;
        s->rgas = s->lut->R;
        s->cp = (s->gamma * s->rgas) / (s->gamma - 1);
    }
    dir_join(path, sizeof path, base, grid);
    if (read_grid(s, path)) { oracle_destroy(s); return 1; }
    if (s->ni < 3 || (s->topology != TOPO_1D && s->nj < 3) || (s->topology == TOPO_3D && s->nk < 3)) {
        fail("the grid needs at least 3 nodes along every swept direction");
        oracle_destroy(s);
        return 1;
    }
    if ((s->topology == TOPO_3D) != (s->nk > 1)) {
        fail("TOPOLOGY does not match the grid's NK");
        oracle_destroy(s);
        return 1;
    }
    long nd = (s->ni + 1) * (s->nj + 1) * (s->nk + 1);
    s->dual = (vec3*)calloc(nd, sizeof(vec3));
    long nI = (s->ni + 1) * s->nj * s->nk, nJ = s->ni * (s->nj + 1) * s->nk, nK = s->ni * s->nj * (s->nk + 1);
    s->sI = (vec3*)calloc(nI, sizeof(vec3)); s->cI = (vec3*)calloc(nI, sizeof(vec3));
    s->sJ = (vec3*)calloc(nJ, sizeof(vec3)); s->cJ = (vec3*)calloc(nJ, sizeof(vec3));
    s->sK = (vec3*)calloc(nK, sizeof(vec3)); s->cK = (vec3*)calloc(nK, sizeof(vec3));
    s->vol = (double*)calloc(s->n, sizeof(double));
    if (s->topology == TOPO_3D) build_dual_3d(s);
    else build_dual_2d(s);
    build_interfaces(s);
    build_volumes(s);
    if (s->bfm_active) {
        if (!s->field[F_BLOCKAGE]) { fail("blockage not found in the grid file"); oracle_destroy(s); return 1; }
        build_blockage_gradient(s);
        const int need[] = {F_NAX, F_NRAD, F_NTAN, F_RPM, F_BLADE_PRESENT, F_NBLADES};
        for (unsigned q = 0; q < sizeof need / sizeof need[0]; q++)
            if (!s->field[need[q]]) { fail("%s not found in the grid file", FIELD_NAMES[need[q]]); oracle_destroy(s); return 1; }
        if (s->bfm_model == BFM_CORRELATIONS) {
            const int needc[] = {F_STWL, F_METAL, F_CAMBER_CURV};
            for (unsigned q = 0; q < 3; q++)
                if (!s->field[needc[q]]) { fail("%s not found in the grid file", FIELD_NAMES[needc[q]]); oracle_destroy(s); return 1; }
        }
        if (s->bfm_model == BFM_CHIMA) {
            const int needc[] = {F_STWL, F_DANGMOM, F_DENTROPY};
            for (unsigned q = 0; q < 3; q++)
                if (!s->field[needc[q]]) { fail("%s not found in the grid file", FIELD_NAMES[needc[q]]); oracle_destroy(s); return 1; }
        }
    }
    if (s->bfm_model == BFM_CHIMA) { /* SourceBFMChima::SourceBFMChima (src/source_bfm_chima.cpp:3-13) */
        const char* cf = cfg_get(&s->cfg, "CHIMA_SCALING_FUNCTIONS_FILEPATH");
        if (!cf) { fail("Not found value for key \"CHIMA_SCALING_FUNCTIONS_FILEPATH\" in configuration."); oracle_destroy(s); return 1; }
        dir_join(path, sizeof path, base, cf);
        if (read_chima_table(s, path)) { oracle_destroy(s); return 1; }
        s->need_turbo = 1; /* src/solver.cpp:1319-1321 */
    }
    const char* bcf = cfg_get(&s->cfg, "BOUNDARY_CONDITIONS_FILEPATH");
    if (!bcf) { fail("Not found value for key \"BOUNDARY_CONDITIONS_FILEPATH\" in configuration."); oracle_destroy(s); return 1; }
    dir_join(path, sizeof path, base, bcf);
    if (read_boundaries(s, path) || build_boundary_structures(s)) { oracle_destroy(s); return 1; }
    resolve_turbo_dir(s);
    if (s->viscous && build_wall_mask(s)) { oracle_destroy(s); return 1; }
    if (setup_sa(s)) { oracle_destroy(s); return 1; }
    for (int m = 0; m < s->npatches; m++) {
        if (s->patches[m].type == BC_THROTTLE) { s->need_turbo = 1; s->throttle_kt = s->patches[m].values[0]; }
        if (s->patches[m].type == BC_MASS_FLOW) s->need_turbo = 1; /* src/solver.cpp:1311-1316 */
        if (s->patches[m].type == BC_INLET_SUPERSONIC && s->patches[m].nvalues < 5)
            { fail("inlet_supersonic needs pressure, temperature and 3 velocity components"); oracle_destroy(s); return 1; }
        if (s->patches[m].type == BC_FARFIELD && s->patches[m].nvalues < 6)
            { fail("farfield needs Mach number, pressure, temperature and a 3-component direction"); oracle_destroy(s); return 1; }
    }
    /* Config::getMassFlowRelaxation / getMassFlowMaxPressureChange (include/config.hpp:291-293) */
    s->mf_relax = 0.05;
    s->mf_max_change = 0.02;
    if (cfg_get(&s->cfg, "MASS_FLOW_RELAXATION") && cfg_float(&s->cfg, "MASS_FLOW_RELAXATION", &s->mf_relax))
        { oracle_destroy(s); return 1; }
    if (cfg_get(&s->cfg, "MASS_FLOW_MAX_PRESSURE_CHANGE") &&
        cfg_float(&s->cfg, "MASS_FLOW_MAX_PRESSURE_CHANGE", &s->mf_max_change))
        { oracle_destroy(s); return 1; }
    if (s->greitzer && s->throttle_kt == 0.0) {
        int found = 0;
        for (int m = 0; m < s->npatches; m++) if (s->patches[m].type == BC_THROTTLE) found = 1;
        if (!found) { fail("Greitzer modeling enabled but no throttle boundary condition found!"); oracle_destroy(s); return 1; }
    }
    for (int c = 0; c < 5; c++) {
        s->U[c] = (double*)calloc(s->n, sizeof(double));
        s->Utmp[c] = (double*)calloc(s->n, sizeof(double));
        s->R[c] = (double*)calloc(s->n, sizeof(double));
    }
    s->dt = (double*)calloc(s->n, sizeof(double));
    if (init_solution(s, base)) { oracle_destroy(s); return 1; }
    /* Greitzer initial state (src/solver.cpp:752-765) */
    if (s->greitzer) {
        update_mass_flows(s, s->U);
        update_turbo(s, s->U);
        sv5 W = prim_of(state_at(s, s->U, s->ni - 1, 0, 0));
        double ph = pressure_prim(s, W);
        double Th = f_temperature_rho_u_et(s, W.v[0], vel_of(W), W.v[4]);
        s->gz_p = ph; s->gz_min = s->turbo[0]; s->gz_mout = s->turbo[0]; s->gz_T = Th; s->gz_t = 0.0;
    }
    /* initial radial profiles (src/solver.cpp:818-834) */
    for (int m = 0; m < s->nprofiles; m++) {
        radial_profile* rp = &s->profiles[m];
        const patch* p = &s->patches[rp->patch];
        if (p->type == BC_MASS_FLOW && p->nvalues >= 2 && p->values[1] > 0.0) {
            for (int q = 0; q < rp->n; q++) rp->pressure[q] = p->values[1];
            continue;
        }
        long i = p->i_min > 0 ? p->i_min - 1 : 0;
        int kk = 0;
        for (long j = p->j_min; j < p->j_max && kk < rp->n; j++) {
            sv5 W = prim_of(state_at(s, s->U, i, j, 0));
            rp->pressure[kk++] = pressure_prim(s, W);
        }
    }
    *out = s;
    return 0;
}

void oracle_destroy(oracle_solver* s) {
    if (!s) return;
    cfg_free(&s->cfg);
    lut_free(s->lut);
    free(s->vert); free(s->dual);
    free(s->sI); free(s->sJ); free(s->sK); free(s->cI); free(s->cJ); free(s->cK);
    free(s->vol); free(s->gradb);
    free(s->chima_mf); free(s->chima_turn); free(s->chima_loss);
    for (int f = 0; f < F_COUNT; f++) free(s->field[f]);
    free(s->patches); free(s->mapI); free(s->mapJ); free(s->mapK);
    for (int m = 0; m < s->nprofiles; m++) { free(s->profiles[m].pressure); free(s->profiles[m].radius); }
    free(s->profiles);
    for (int c = 0; c < 5; c++) { free(s->U[c]); free(s->Utmp[c]); free(s->R[c]); }
    free(s->dt);
    free(s->wall);
    for (int v = 0; v < 4; v++) { free(s->grad[v]); free(s->gfield[v]); }
    free(s->nuhat); free(s->nul); free(s->wdist); free(s->sa_res); free(s->sa_diag); free(s->sa_dstar);
    free(s->sa_dnu); free(s->nuhat_grad); free(s->sa_vel);
    free(s->hist);
    free(s);
}

void oracle_shape(const oracle_solver* s, long long out[3]) {
    out[0] = s->ni; out[1] = s->nj; out[2] = s->nk;
}

#define HIST_W 16 /* 5 lognorm + 6 massflow + 4 turbo + 1 hub */

static void hist_push(oracle_solver* s, const double lr[5]) {
    if (s->nhist == s->hist_cap) {
        s->hist_cap = s->hist_cap ? 2 * s->hist_cap : 1024;
        s->hist = (double*)realloc(s->hist, sizeof(double) * HIST_W * s->hist_cap);
    }
    double* h = s->hist + HIST_W * s->nhist;
    for (int v = 0; v < 5; v++) h[v] = lr[v];
    for (int b = 0; b < 6; b++) h[5 + b] = s->massflow[b];
    for (int b = 0; b < 4; b++) h[11 + b] = s->need_turbo ? s->turbo[b] : 0.0;
    h[15] = s->hub_p;
    s->nhist++;
}

/* The explicit branch of Solver::solve (src/solver.cpp:1296-1398). The
 * state's first preprocessSolution(.., false) is a no-op for inviscid runs. */
int oracle_run(oracle_solver* s, long n_iter, long* n_done, int* converged) {
    *n_done = 0;
    *converged = 0;
    s->nhist = 0;
    no_slip_momentum(s, s->U);
    for (int c = 0; c < 5; c++) memcpy(s->Utmp[c], s->U[c], sizeof(double) * s->n);
    for (long it = s->iter + 1; it <= s->iter + n_iter; it++) {
        update_mass_flows(s, s->Utmp);
        if (s->need_turbo) update_turbo(s, s->Utmp);
        compute_timestep(s, s->Utmp);
        if (s->nprofiles || s->greitzer) update_radial_profiles(s, s->Utmp);
        no_slip_momentum(s, s->Utmp);
        if (s->sa) {  /* Solver::solve: computeSolutionGradient, updateTurbulenceSolution */
            solution_gradient(s, s->Utmp);
            if (sa_solve(s, s->Utmp)) { *n_done = it - s->iter; s->iter = it; return 2; }
        }
        for (int st = 0; st < s->nstages; st++) {
            solution_gradient(s, s->Utmp);
            compute_residuals(s, s->Utmp, it);
            update_solution(s, s->coeffs[st]);
            periodic_solution(s);
        }
        for (int c = 0; c < 5; c++) memcpy(s->U[c], s->Utmp[c], sizeof(double) * s->n);
        double m = s->dt[0];
        for (long q = 1; q < s->n; q++) if (s->dt[q] < m) m = s->dt[q];
        s->t += m;
        double lr[5];
        if (log_residual_norm(s, lr)) { *n_done = it - s->iter; s->iter = it; return 2; }
        if (!s->has_init_log) {
            for (int v = 0; v < 5; v++) s->init_log[v] = lr[v];
            s->has_init_log = 1;
        } else if (it <= 5) {
            for (int v = 0; v < 5; v++) s->init_log[v] = dmax(s->init_log[v], lr[v]);
        }
        hist_push(s, lr);
        *n_done = it - s->iter;
        if (check_convergence(s, lr)) { *converged = 1; break; }
    }
    s->iter += *n_done;
    return 0;
}

int oracle_residual(oracle_solver* s, double* dt, double* r0, double* r1, double* r2, double* r3,
                    double* r4) {
    no_slip_momentum(s, s->U);
    for (int c = 0; c < 5; c++) memcpy(s->Utmp[c], s->U[c], sizeof(double) * s->n);
    update_mass_flows(s, s->Utmp);
    if (s->need_turbo) update_turbo(s, s->Utmp);
    compute_timestep(s, s->Utmp);
    if (s->nprofiles || s->greitzer) update_radial_profiles(s, s->Utmp);
    no_slip_momentum(s, s->Utmp);
    solution_gradient(s, s->Utmp);
    compute_residuals(s, s->Utmp, s->iter + 1);
    memcpy(dt, s->dt, sizeof(double) * s->n);
    double* outs[5] = {r0, r1, r2, r3, r4};
    for (int c = 0; c < 5; c++) memcpy(outs[c], s->R[c], sizeof(double) * s->n);
    return 0;
}

/* The Spalart-Allmaras working variable nu hat per node (0 when the model is
 * off); returns whether the model is on. */
int oracle_get_nuhat(const oracle_solver* s, double* out) {
    for (long q = 0; q < s->n; q++) out[q] = s->sa ? s->nuhat[q] : 0.0;
    return s->sa;
}

void oracle_get_state(const oracle_solver* s, double* rho, double* rhou, double* rhov, double* rhow,
                      double* rhoe) {
    double* outs[5] = {rho, rhou, rhov, rhow, rhoe};
    for (int c = 0; c < 5; c++) memcpy(outs[c], s->U[c], sizeof(double) * s->n);
}

void oracle_set_state(oracle_solver* s, const double* rho, const double* rhou, const double* rhov,
                      const double* rhow, const double* rhoe) {
    const double* ins[5] = {rho, rhou, rhov, rhow, rhoe};
    for (int c = 0; c < 5; c++) memcpy(s->U[c], ins[c], sizeof(double) * s->n);
}

long oracle_history(const oracle_solver* s, double* lognorm, double* massflow, double* turbo,
                    double* hub) {
    for (long q = 0; q < s->nhist; q++) {
        const double* h = s->hist + HIST_W * q;
        if (lognorm) for (int v = 0; v < 5; v++) lognorm[5 * q + v] = h[v];
        if (massflow) for (int b = 0; b < 6; b++) massflow[6 * q + b] = h[5 + b];
        if (turbo) for (int b = 0; b < 4; b++) turbo[4 * q + b] = h[11 + b];
        if (hub) hub[q] = h[15];
    }
    return s->nhist;
}

double oracle_time(const oracle_solver* s) { return s->t; }
