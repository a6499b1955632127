/* CPU oracle for the CTurboBFM explicit residual-and-update loop.
 *
 * TEST INFRASTRUCTURE ONLY. This is a plain-C restatement of the reference
 * solver's algorithm (Propulsion-Power-TU-Delft/CTurboBFM), used by the tests,
 * by __graft_entry__.smoke() and by bench.py's CPU-baseline leg as the checker.
 * The product library never links, loads or calls it.
 *
 * It reads the same three files as the reference (input.ini, the grid CSV and
 * boundaries.csv) and runs the same serial FP64 loop in the same operation
 * order, so that, compiled with -ffp-contract=off, it reproduces the
 * reference bit for bit (pinned in tests against oracle/_ref/ref_harness).
 */
#ifndef CTBFM_ORACLE_H
#define CTBFM_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct oracle_solver oracle_solver;

/* Builds Config + Mesh + Solver from an input.ini path (relative file names in
 * the ini resolve against the ini's directory). Returns 0 on success. */
int oracle_create(const char* ini_path, oracle_solver** out);
void oracle_destroy(oracle_solver* s);
const char* oracle_last_error(void);

/* Grid sizes. */
void oracle_shape(const oracle_solver* s, long long out[3]);

/* Runs up to n_iter pseudo-time iterations of the explicit Runge-Kutta loop
 * (Solver::solve, src/solver.cpp:1337-1398), stopping at convergence like the
 * reference. Returns 0, or 2 when the residual norm is NaN/Inf (the reference's
 * "Solver diverged" exception). *n_done receives the iterations performed,
 * *converged 1 if the convergence test fired. */
int oracle_run(oracle_solver* s, long n_iter, long* n_done, int* converged);

/* One residual evaluation of the initial state exactly as iteration 1 does it
 * (time step array + residual field). Does not advance the state. */
int oracle_residual(oracle_solver* s, double* dt, double* r0, double* r1, double* r2,
                    double* r3, double* r4);

/* Conservative state (reference layout, (i*nj + j)*nk + k). */
/* Spalart-Allmaras working variable per node (zeros without the model);
 * returns 1 when the model is on. */
int oracle_get_nuhat(const oracle_solver* s, double* out);
void oracle_get_state(const oracle_solver* s, double* rho, double* rhou, double* rhov,
                      double* rhow, double* rhoe);
void oracle_set_state(oracle_solver* s, const double* rho, const double* rhou,
                      const double* rhov, const double* rhow, const double* rhoe);

/* Per-iteration history of the last oracle_run call: log10 residual norms
 * (5 per iteration), boundary mass flows (6), turbo performance (mass flow,
 * PRtt, TRtt, eta; 4) and hub static pressure (1). Returns the count. */
long oracle_history(const oracle_solver* s, double* lognorm, double* massflow,
                    double* turbo, double* hub);

double oracle_time(const oracle_solver* s);

#ifdef __cplusplus
}
#endif
#endif
