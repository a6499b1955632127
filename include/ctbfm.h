/* ctbfm.h — C ABI of the B200-native CTurboBFM explicit residual-and-update loop.
 *
 * The reference (Propulsion-Power-TU-Delft/CTurboBFM) has no FFI; its
 * extension points are C++ classes driven per face / per node through virtual
 * calls. This header is the drop-in boundary that replaces them with batched
 * device execution. Each entry point names the reference interface it stands
 * for:
 *
 *   ctbfm_create_from_ini   Config(input.ini) + Mesh(config) + Solver(config, mesh)
 *                           (src/turbobfm.cpp:15-27, src/config.cpp:8-13,
 *                            src/mesh.cpp:11-40, src/solver.cpp:18-31)
 *   ctbfm_create            Solver(Config&, Mesh&) (include/solver.hpp:49-53) with
 *                           the settings, grid and patches given in memory
 *   ctbfm_solve             Solver::solve() explicit branch (src/solver.cpp:1296-1424)
 *   ctbfm_step              n iterations of that loop (src/solver.cpp:1337-1398),
 *                           never past N_ITERATIONS
 *   ctbfm_compute_residual  Solver::computeTimestepArray + Solver::computeResiduals
 *                           (src/solver.cpp:1531-1630, 1783-1833) on the current state
 *   ctbfm_get_state /
 *   ctbfm_set_state         Solver::_conservativeSolution (FlowSolution,
 *                           include/types.hpp:763-1018), reference layout
 *                           (i*NJ + j)*NK + k, five arrays of doubles
 *   ctbfm_get_lognorm       Solver::computeLogResidualNorm (src/solver.cpp:1488-1508)
 *   ctbfm_get_turbo         Solver::updateMassFlows / updateTurboPerformance
 *                           (src/solver.cpp:1633-1781)
 *   ctbfm_write_solution    Output::writeSolution (src/output.cpp:384-447): the
 *                           volume CSV that RESTART_SOLUTION reads back
 *                           (Solver::initializeSolutionFromRestart,
 *                           src/solver.cpp:890-1295, done at create time)
 *   ctbfm_last_error        the std::runtime_error text the reference would throw
 *
 * Conventions
 *   - every function returns 0 on success and a non-zero CTBFM_E* code on
 *     error; no C++ exception crosses this boundary; ctbfm_last_error() gives
 *     the message of the calling thread's last error;
 *   - the library owns all device memory; the caller owns host buffers;
 *   - divergence (NaN/Inf residual norm, the reference's "Solver diverged")
 *     is reported as CTBFM_E_DIVERGED, never as a device fault;
 *   - a handle is bound to one CUDA stream and is not thread safe; separate
 *     handles may be driven from separate host threads.
 */
#ifndef CTBFM_H
#define CTBFM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ctbfm_solver ctbfm_solver;

enum {
    CTBFM_OK = 0,
    CTBFM_E_CONFIG = 1,      /* invalid or unsupported input.ini / grid / boundary file */
    CTBFM_E_CUDA = 2,        /* CUDA runtime error (allocation, launch) */
    CTBFM_E_DIVERGED = 3,    /* NaN or Inf in a residual norm */
    CTBFM_E_ARGUMENT = 4,    /* bad argument (null pointer, wrong size) */
    CTBFM_E_UNSUPPORTED = 5  /* feature outside this library's scope */
};

enum {
    CTBFM_STATUS_RUNNING = 0,
    CTBFM_STATUS_CONVERGED = 1,
    CTBFM_STATUS_DIVERGED = 2,
    CTBFM_STATUS_DEVICE_ERROR = 3  /* stopped by a device error: a grid barrier wait of the
                                      persistent kernel ran out (reported as CTBFM_E_CUDA) */
};

typedef struct {
    int64_t ni, nj, nk;       /* nodes (= control volumes) per direction */
    int32_t topology;         /* 0 = 2D, 1 = 3D, 2 = axisymmetric */
    int32_t n_stages;         /* Runge-Kutta stages per iteration (4 or 3) */
    int64_t iteration;        /* iterations performed so far */
    int64_t max_iterations;   /* N_ITERATIONS */
    int32_t status;           /* CTBFM_STATUS_* */
    int32_t precision;        /* GPU_PRECISION: 0 = fp64, 1 = fp32_kahan */
    double time;              /* physical time sum of min(dt) */
    int64_t device_bytes;     /* device memory the solver holds */
    int32_t face_tile[3];     /* faces per block chosen by the autotuner per direction (I, J, K) */
    int32_t fused_stage;      /* 1: each Runge-Kutta stage runs as the fused kernel k_stage;
                                 0: as the split kernels k_prim, k_faces, k_nodes */
    int32_t persistent_stage; /* 1: whole iterations run in the persistent kernel k_run (one
                                 cooperative launch per 32 iterations, phases separated by a
                                 grid barrier) */
    double tuned_stage_ms[3]; /* the autotuner's time of one stage: split, fused, persistent
                                 (0: not timed) */
} ctbfm_info;

/* Builds a solver from an input.ini in the reference's format (the grid CSV and
 * boundaries.csv it names resolve relative to the ini's directory) and uploads
 * everything to the current CUDA device. */
int ctbfm_create_from_ini(const char* ini_path, ctbfm_solver** out);

/* One boundary patch: a row of the reference's boundaries.csv
 * (PATCH_NAME, I_MIN, I_MAX, J_MIN, J_MAX, K_MIN, K_MAX). Its type and values
 * come from the setting of the same name, as in input.ini
 * ("inlet" = "inlet, 101325, 288.15, 1, 0, 0"). */
typedef struct {
    const char* name;
    int64_t i_min, i_max, j_min, j_max, k_min, k_max;
} ctbfm_patch;

/* A case held in memory: what input.ini, the grid CSV and boundaries.csv carry
 * (the reference's Config, Mesh and boundary table, include/solver.hpp:49-53).
 * Node (i, j, k) of every grid array is element (i*nj + j)*nk + k, the grid
 * CSV's row order. ctbfm_create copies everything; the caller's arrays and
 * strings may be released when it returns. */
typedef struct {
    int64_t ni, nj, nk;               /* nodes per direction (nk = 1 in 2-D) */
    const double* x;                  /* ni*nj*nk node coordinates */
    const double* y;
    const double* z;
    int32_t n_fields;                 /* further grid columns: blockage, normalAxial, ... */
    const char* const* field_names;   /* n_fields column names, as in the grid CSV header */
    const double* const* fields;      /* n_fields arrays of ni*nj*nk values */
    int32_t n_patches;
    const ctbfm_patch* patches;
    int32_t n_settings;               /* input.ini settings as strings: keys[q] = values[q] */
    const char* const* keys;
    const char* const* values;
    const char* directory;            /* where the files that settings still name resolve
                                         (FLUID_TABLE_FILE, CHIMA_SCALING_FUNCTIONS_FILEPATH,
                                         RESTART_SOLUTION_FILEPATH); NULL = the current directory.
                                         GRID_FILE and BOUNDARY_CONDITIONS_FILEPATH are not read. */
} ctbfm_case_desc;

/* Builds a solver from a case held in memory (the same checks, results and
 * errors as ctbfm_create_from_ini on the same values) and uploads everything to
 * the current CUDA device. Returns CTBFM_E_ARGUMENT for a malformed
 * description (null arrays, negative counts) and CTBFM_E_CONFIG for settings
 * the ini path would reject. Replaces Solver(Config&, Mesh&)
 * (include/solver.hpp:49-53) with the Config and Mesh built in memory. */
int ctbfm_create(const ctbfm_case_desc* desc, ctbfm_solver** out);

/* Releases device memory, graphs and streams owned by the solver. */
void ctbfm_destroy(ctbfm_solver* s);

/* Binds the solver to a caller-owned CUDA stream (a cudaStream_t passed as
 * void*); NULL restores the solver's own stream. */
int ctbfm_set_stream(ctbfm_solver* s, void* cuda_stream);

int ctbfm_get_info(const ctbfm_solver* s, ctbfm_info* out);

/* Runs up to n_iter iterations (fewer if the convergence test fires, the
 * solution diverges or N_ITERATIONS is reached). *n_done receives the
 * iterations performed. Returns
 * CTBFM_E_DIVERGED when a residual norm is NaN/Inf. Synchronises the stream. */
int ctbfm_step(ctbfm_solver* s, int64_t n_iter, int64_t* n_done);

/* Enqueues exactly n_iter iterations on the solver's stream without any host
 * synchronisation (kernels of iterations after convergence or divergence
 * return immediately). For timing and CUDA-graph capture. */
int ctbfm_enqueue(ctbfm_solver* s, int64_t n_iter);

/* Runs the autotuner now unless it has run (otherwise it runs at the first
 * enqueue of at least 64 iterations): face tiles per direction, and with
 * GPU_STAGE_FUSION = auto which of the split, fused and persistent stage
 * kernels is fastest (the persistent kernel only where it is eligible: no
 * real-gas table, viscosity or turbulence model, and in a batch one convection
 * scheme for all members), timed on forced first-stage
 * evaluations that leave the state unchanged. Synchronises the stream. No
 * counterpart in the reference. */
int ctbfm_autotune(ctbfm_solver* s);

/* Runs the whole loop to N_ITERATIONS or convergence, like Solver::solve(). */
int ctbfm_solve(ctbfm_solver* s, int64_t* n_done);

/* One time-step + residual evaluation of the current state with the next
 * iteration's number, without advancing anything but the boundary-profile
 * and plenum state the reference also advances there. Outputs are NI*NJ*NK
 * doubles each (dt) and 5 arrays (residual, reference layout). */
int ctbfm_compute_residual(ctbfm_solver* s, double* dt, double* r_rho, double* r_rhou,
                           double* r_rhov, double* r_rhow, double* r_rhoe);

/* Same outputs as ctbfm_compute_residual, for callers that cannot call
 * cudaMalloc when they need a residual: processes whose device memory is
 * owned by another allocator (a framework's caching allocator, or a pool
 * reserved at start-up) and control loops that must not block in the
 * driver's allocator mid-step. It allocates no device memory: the per-face
 * flux contributions go to a static __device__ array of 16 MiB, 5 words per
 * face summed over the swept directions, i.e. at most 419430 faces in fp64
 * and 838860 in fp32_kahan (larger cases return CTBFM_E_CONFIG with the
 * sizes in the message). Every GPU on which a solver is created holds that
 * array until exit: solver creation looks up its device address
 * (cudaGetSymbolAddress), which also makes the driver back it under lazy
 * module loading, so this call never reserves memory. All calls on a device
 * share the array, so calls that overlap on the GPU race. The call runs on
 * the device the solver was created on and restores the caller's current
 * device. No counterpart in the reference. */
int ctbfm_compute_residual_noalloc(ctbfm_solver* s, double* dt, double* r_rho, double* r_rhou,
                                   double* r_rhov, double* r_rhow, double* r_rhoe);

/* Conservative state U^n (host buffers of NI*NJ*NK doubles each). */
int ctbfm_get_state(ctbfm_solver* s, double* rho, double* rhou, double* rhov, double* rhow,
                    double* rhoe);
int ctbfm_set_state(ctbfm_solver* s, const double* rho, const double* rhou, const double* rhov,
                    const double* rhow, const double* rhoe);

/* Writes the current state as a volume CSV in the reference's format
 * (NI/NJ/NK lines, "x,y,z,<fields sorted by name>", 16 significant digits;
 * OUTPUT_FIELDS_TYPE primary or secondary, the default). The file is a valid
 * restart file (RESTART_SOLUTION = yes, RESTART_SOLUTION_FILEPATH, RESTART_TYPE
 * standard / axisymmetric / nearest_neighbor / nearest_neighbor_axisymmetric).
 * CTBFM_E_CONFIG for OUTPUT_FIELDS_TYPE = turbo_bfm on a body-force case. */
int ctbfm_write_solution(ctbfm_solver* s, const char* path);

/* log10 residual norms of the last iteration (5 doubles). */
int ctbfm_get_lognorm(ctbfm_solver* s, double out[5]);

/* Per-iteration history of the last ctbfm_step / ctbfm_solve call:
 * log10 residual norms (5 per iteration), boundary mass flows (6: I start,
 * I end, J start, J end, K start, K end), turbo performance (4: mass flow,
 * PRtt, TRtt, eta_tt) and hub static pressure (1). Returns the number of rows
 * written in *n_rows; pass NULL arrays to query the count. */
int ctbfm_get_history(ctbfm_solver* s, int64_t max_rows, double* lognorm, double* massflow,
                      double* turbo, double* hub, int64_t* n_rows);

/* Physical time after each iteration of the same history (Solver::_time,
 * src/solver.cpp:1389-1390; the time column of turbo.csv). */
int ctbfm_get_history_time(ctbfm_solver* s, int64_t max_rows, double* time, int64_t* n_rows);

/* Mass flows (6) and turbo performance (4) of the current state, computed on
 * the device in FP64. */
int ctbfm_get_turbo(ctbfm_solver* s, double massflow[6], double turbo[4]);

/* Kernel kinds timed by ctbfm_profile_kernels, in output order. */
enum {
    CTBFM_K_BOUNDARY_INTEGRALS = 0, /* k_bint */
    CTBFM_K_TIME_STEP = 1,          /* k_dt */
    CTBFM_K_PRE_STAGE = 2,          /* k_pre */
    CTBFM_K_FACES_I = 3,            /* k_faces<I> */
    CTBFM_K_FACES_J = 4,            /* k_faces<J> */
    CTBFM_K_FACES_K = 5,            /* k_faces<K> (3-D) */
    CTBFM_K_NODES = 6,              /* k_nodes */
    CTBFM_K_PERIODIC = 7,           /* k_periodic (periodic cases) */
    CTBFM_K_FINALIZE = 8,           /* k_finalize */
    CTBFM_K_PRIMITIVES = 9,         /* k_prim */
    CTBFM_K_STAGE = 10,             /* k_stage, the fused stage kernel (GPU_STAGE_FUSION = fused) */
    CTBFM_K_COUNT = 11
};

/* Measurement hook (no counterpart in the reference): launches each kernel
 * kind of one iteration `reps` times on the solver's stream, bracketed by
 * CUDA events, and writes the average duration in milliseconds per launch to
 * out_ms[CTBFM_K_COUNT] (0 for kinds this case does not launch). The state,
 * time step and control block are restored afterwards. */
int ctbfm_profile_kernels(ctbfm_solver* s, int reps, double* out_ms);

/* ------------------------------------------------------------------------
 * Batches of operating points. No counterpart in the reference, which runs
 * one turbobfm process per operating point (python/Run_All_Cases.py:18-98).
 * A batch advances its solvers together: each kernel family is one launch
 * over a packed tile index of all members' nodes, faces and planes, so many
 * small grids share the GPU. Every member computes exactly what it computes
 * alone (per-member reductions in a fixed order).
 * ------------------------------------------------------------------------ */
typedef struct ctbfm_batch ctbfm_batch;

/* Groups n solvers of the same GPU_PRECISION (Runge-Kutta stage counts may
 * differ). The solvers stay owned by the caller, must outlive the batch and
 * must not be stepped on their own while it exists; their state, turbo and
 * history queries remain valid between batch steps. Duplicates, NULLs and
 * mixed precisions are CTBFM_E_ARGUMENT. */
int ctbfm_batch_create(ctbfm_solver* const* solvers, int32_t n, ctbfm_batch** out);
void ctbfm_batch_destroy(ctbfm_batch* b);
int ctbfm_batch_set_stream(ctbfm_batch* b, void* cuda_stream);

/* Enqueues n_iter iterations of every member that is still running (members
 * that converge or diverge stop on the device at that iteration). */
int ctbfm_batch_enqueue(ctbfm_batch* b, int64_t n_iter);

/* ctbfm_autotune for the batch's group. */
int ctbfm_batch_autotune(ctbfm_batch* b);

/* The batch's stage kernels: *mode = 0 the split kernels, 1 the fused stage
 * kernel k_stage (for the members that can run it), 2 the persistent kernel
 * k_run; and the autotuner's time of one stage of the whole batch in each
 * (split, fused, persistent; 0 when not timed). No counterpart in the
 * reference. */
int ctbfm_batch_stage_kernels(ctbfm_batch* b, int32_t* mode, double stage_ms[3]);

/* enqueue + synchronise. *n_done (nullable) receives the most iterations any
 * member advanced. A diverged member is reported through
 * ctbfm_batch_status, not as an error of the call. */
int ctbfm_batch_step(ctbfm_batch* b, int64_t n_iter, int64_t* n_done);

/* Per member (arrays of n, each nullable): CTBFM_STATUS_*, iterations done,
 * the last log10 residual norms (5 per member), and the convergence progress
 * best_drop = the largest min-over-variables drop of the log norm below its
 * initial maximum reached so far (orders of magnitude). */
int ctbfm_batch_status(ctbfm_batch* b, int32_t* status, int64_t* iterations, double* lognorm,
                       double* best_drop);

/* Continues a fp32_kahan solver in FP64 (state U - Uc, iteration count,
 * time, convergence reference, plenum and profile state carried over); a
 * no-op for FP64 solvers. A batch holding the solver must be destroyed
 * first. No counterpart in the reference (FP64 only). */
int ctbfm_promote_fp64(ctbfm_solver* s);

/* ------------------------------------------------------------------------
 * Serving: continuous batching of operating-point solves. No counterpart in
 * the reference (one process per operating point, run to the end). Requests
 * are prepared on host worker threads, admitted in arrival order while slots
 * and device memory allow, advance together with every other admitted solve
 * (one batch per GPU_PRECISION, each on its own stream), and retire as soon
 * as they converge, diverge or reach N_ITERATIONS. Each solve's state, BFM
 * fields and plenum state stay on the device from admission to retirement.
 * ------------------------------------------------------------------------ */
typedef struct ctbfm_server ctbfm_server;

typedef struct {
    int64_t id;
    int32_t status;      /* CTBFM_STATUS_*, -1 when the request failed before running */
    int32_t precision;   /* precision the solve finished in (0 fp64, 1 fp32_kahan) */
    int64_t iterations;
    double t_submit;     /* seconds since the server was created */
    double t_admit;
    double t_done;
    double massflow[6];  /* as ctbfm_get_turbo */
    double turbo[4];
    int32_t error;       /* CTBFM_OK or the request's error code */
    char message[240];   /* error message, truncated */
} ctbfm_result;

/* device_budget_bytes: device memory the admitted solves may hold (0: 90 % of
 * what is free at each admission); max_active: admitted solves at most;
 * max_active_nodes: grid nodes the admitted solves may hold together (0: no
 * limit; about the node count that fills the GPU keeps early arrivals from
 * sharing the device with every later one); chunk_iterations: iterations
 * per scheduling round; stall_window: a
 * fp32_kahan solve whose convergence progress (best_drop of
 * ctbfm_batch_status) has not grown by 0.05 for this many iterations
 * continues in FP64, and a fp32_kahan solve whose residual becomes NaN/Inf
 * is run again once, from its initial state, in FP64 (0: neither; a moved
 * solve's result reports precision 0); host_threads: request-preparation
 * workers. A result depends on its own request only, never on the rest of
 * the mix. */
int ctbfm_server_create(uint64_t device_budget_bytes, int32_t max_active, int64_t max_active_nodes,
                        int64_t chunk_iterations, int64_t stall_window, int32_t host_threads, ctbfm_server** out);
void ctbfm_server_destroy(ctbfm_server* s);

/* The precision pattern's other trigger: a fp32_kahan solve continues in FP64
 * once its best residual drop comes within `orders` of its
 * RESIDUALS_DROP_CONVERGENCE (best_drop >= drop - orders), at a scheduling
 * round; 0 (the default) turns it off. Set before the first submission. */
int ctbfm_server_set_promotion(ctbfm_server* s, double orders);

/* Where the pumping thread's time went since the server was created. */
typedef struct {
    int64_t rounds;      /* scheduling rounds that enqueued a chunk */
    int64_t rebuilds;    /* batch rebuilds (membership changes applied, a few rounds' worth at a time) */
    int64_t promotions;  /* fp32_kahan solves continued in FP64 */
    int64_t reruns;      /* diverged fp32_kahan solves run again in FP64 */
    double wait_s;       /* seconds waiting for the chunk in flight (the device busy) */
    double process_s;    /* seconds reporting and marking after a chunk */
    double rebuild_s;    /* seconds applying changes and rebuilding batches, of which */
    double promote_s;    /*   promoting solves to FP64 (and re-creating diverged ones), */
    double release_s;    /*   releasing finished solves, */
    double batch_s;      /*   releasing and building the two batches */
    double prepare_s;    /* seconds building the FP64 side of paused solves, while a chunk runs */
    double enqueue_s;    /* seconds enqueueing chunks (a new batch's autotuning included) */
    double admit_s;      /* seconds building admitted solves, while a chunk runs */
} ctbfm_server_stats;
int ctbfm_server_get_stats(ctbfm_server* s, ctbfm_server_stats* out);

/* Queues the operating point of an input.ini; thread safe. */
int ctbfm_server_submit(ctbfm_server* s, const char* ini_path, int64_t* request_id);

/* Queues the operating point of a case held in memory (copied before the call
 * returns; see ctbfm_create); thread safe. A malformed description returns
 * CTBFM_E_ARGUMENT here; invalid settings come back as the request's error. */
int ctbfm_server_submit_case(ctbfm_server* s, const ctbfm_case_desc* desc, int64_t* request_id);

/* One scheduling round on the calling thread (admit, advance every admitted
 * solve by chunk_iterations, retire, promote). n_active / n_waiting
 * (nullable) receive the counts after the round. */
int ctbfm_server_pump(ctbfm_server* s, int32_t* n_active, int32_t* n_waiting);

/* Moves up to max finished requests into out; *n_out receives how many. */
int ctbfm_server_results(ctbfm_server* s, ctbfm_result* out, int32_t max, int32_t* n_out);

/* Message of the calling thread's last error ("" if none). */
const char* ctbfm_last_error(void);

/* Library version string. */
const char* ctbfm_version(void);

#ifdef __cplusplus
}
#endif
#endif
