// extern "C" boundary (include/ctbfm.h). Every entry point catches all C++
// exceptions and turns them into a status code plus a per-thread message, the
// way the reference's main turns exceptions into exit code 1
// (src/turbobfm.cpp:31-36).
#include "../../include/ctbfm.h"

#include <cuda_runtime.h>

#include <cmath>
#include <memory>
#include <string>

#include "host/config.hpp"
#include "host/mesh.hpp"
#include "host/solver.hpp"

struct ctbfm_solver {
    std::unique_ptr<ctbfm::Config> config;
    std::unique_ptr<ctbfm::Mesh> mesh;
    std::unique_ptr<ctbfm::Solver> solver;
};

namespace {

thread_local std::string g_error;

int setError(int code, const std::string& msg) {
    g_error = msg;
    return code;
}

template <typename F>
int guarded(F&& f) {
    try {
        g_error.clear();
        return f();
    } catch (const ctbfm::ConfigError& e) {
        return setError(CTBFM_E_CONFIG, e.what());
    } catch (const ctbfm::CudaError& e) {
        return setError(CTBFM_E_CUDA, e.what());
    } catch (const std::exception& e) {
        return setError(CTBFM_E_CONFIG, e.what());
    } catch (...) {
        return setError(CTBFM_E_CONFIG, "unknown error");
    }
}

int statusCode(ctbfm_solver* s) {
    const ctbfm::Control c = s->solver->control();
    if (c.status == 2) {
        int var = 0;
        for (int v = 0; v < 5; v++)
            if (std::isnan(c.lognorm[v]) || std::isinf(c.lognorm[v])) {
                var = v;
                break;
            }
        return setError(CTBFM_E_DIVERGED,
                        "Solver diverged: NaN or Inf detected in residual variable " + std::to_string(var));
    }
    return CTBFM_OK;
}

}  // namespace

extern "C" {

const char* ctbfm_last_error(void) { return g_error.c_str(); }

const char* ctbfm_version(void) { return "ctbfm-b200 0.1 (sm_100a, FP64 explicit loop)"; }

int ctbfm_create_from_ini(const char* ini_path, ctbfm_solver** out) {
    if (!ini_path || !out) return setError(CTBFM_E_ARGUMENT, "null argument");
    *out = nullptr;
    return guarded([&] {
        auto s = std::make_unique<ctbfm_solver>();
        s->config = std::make_unique<ctbfm::Config>(ini_path);
        s->mesh = std::make_unique<ctbfm::Mesh>(*s->config);
        s->solver = std::make_unique<ctbfm::Solver>(*s->config, *s->mesh);
        *out = s.release();
        return CTBFM_OK;
    });
}

void ctbfm_destroy(ctbfm_solver* s) {
    if (!s) return;
    try {
        delete s;
    } catch (...) {
    }
}

int ctbfm_set_stream(ctbfm_solver* s, void* stream) {
    if (!s) return setError(CTBFM_E_ARGUMENT, "null solver");
    return guarded([&] {
        s->solver->setStream(static_cast<cudaStream_t>(stream));
        return CTBFM_OK;
    });
}

int ctbfm_get_info(const ctbfm_solver* s, ctbfm_info* out) {
    if (!s || !out) return setError(CTBFM_E_ARGUMENT, "null argument");
    return guarded([&] {
        const ctbfm::Control c = s->solver->control();
        out->ni = s->solver->ni();
        out->nj = s->solver->nj();
        out->nk = s->solver->nk();
        out->topology = s->solver->topology();
        out->n_stages = s->solver->stages();
        out->iteration = c.it;
        out->max_iterations = s->solver->maxIterations();
        out->status = c.status;
        out->precision = s->solver->precision();
        out->time = c.t;
        return CTBFM_OK;
    });
}

int ctbfm_step(ctbfm_solver* s, int64_t n_iter, int64_t* n_done) {
    if (!s || n_iter < 0) return setError(CTBFM_E_ARGUMENT, "bad argument");
    return guarded([&] {
        const long long d = s->solver->step(n_iter);
        if (n_done) *n_done = d;
        return statusCode(s);
    });
}

int ctbfm_enqueue(ctbfm_solver* s, int64_t n_iter) {
    if (!s || n_iter < 0) return setError(CTBFM_E_ARGUMENT, "bad argument");
    return guarded([&] {
        s->solver->enqueue(n_iter);
        return CTBFM_OK;
    });
}

int ctbfm_solve(ctbfm_solver* s, int64_t* n_done) {
    if (!s) return setError(CTBFM_E_ARGUMENT, "null solver");
    return guarded([&] {
        const long long d = s->solver->solve();
        if (n_done) *n_done = d;
        return statusCode(s);
    });
}

int ctbfm_compute_residual(ctbfm_solver* s, double* dt, double* r0, double* r1, double* r2, double* r3, double* r4) {
    if (!s || !dt || !r0 || !r1 || !r2 || !r3 || !r4) return setError(CTBFM_E_ARGUMENT, "null argument");
    return guarded([&] {
        double* const r[5] = {r0, r1, r2, r3, r4};
        s->solver->computeResidual(dt, r);
        return CTBFM_OK;
    });
}

// See include/ctbfm.h: residual evaluation that allocates no device memory.
int ctbfm_compute_residual_noalloc(ctbfm_solver* s, double* dt, double* r0, double* r1, double* r2, double* r3,
                                   double* r4) {
    if (!s || !dt || !r0 || !r1 || !r2 || !r3 || !r4) return setError(CTBFM_E_ARGUMENT, "null argument");
    return guarded([&] {
        double* const r[5] = {r0, r1, r2, r3, r4};
        s->solver->computeResidualNoAlloc(dt, r);
        return CTBFM_OK;
    });
}

int ctbfm_get_state(ctbfm_solver* s, double* rho, double* rhou, double* rhov, double* rhow, double* rhoe) {
    if (!s || !rho || !rhou || !rhov || !rhow || !rhoe) return setError(CTBFM_E_ARGUMENT, "null argument");
    return guarded([&] {
        double* const out[5] = {rho, rhou, rhov, rhow, rhoe};
        s->solver->getState(out);
        return CTBFM_OK;
    });
}

int ctbfm_set_state(ctbfm_solver* s, const double* rho, const double* rhou, const double* rhov, const double* rhow,
                    const double* rhoe) {
    if (!s || !rho || !rhou || !rhov || !rhow || !rhoe) return setError(CTBFM_E_ARGUMENT, "null argument");
    return guarded([&] {
        const double* const in[5] = {rho, rhou, rhov, rhow, rhoe};
        s->solver->setState(in);
        return CTBFM_OK;
    });
}

int ctbfm_get_lognorm(ctbfm_solver* s, double out[5]) {
    if (!s || !out) return setError(CTBFM_E_ARGUMENT, "null argument");
    return guarded([&] {
        const ctbfm::Control c = s->solver->control();
        for (int v = 0; v < 5; v++) out[v] = c.lognorm[v];
        return CTBFM_OK;
    });
}

int ctbfm_get_history(ctbfm_solver* s, int64_t max_rows, double* lognorm, double* massflow, double* turbo,
                      double* hub, int64_t* n_rows) {
    if (!s) return setError(CTBFM_E_ARGUMENT, "null solver");
    return guarded([&] {
        const long long r = s->solver->history(max_rows, lognorm, massflow, turbo, hub);
        if (n_rows) *n_rows = r;
        return CTBFM_OK;
    });
}

int ctbfm_get_turbo(ctbfm_solver* s, double massflow[6], double turbo[4]) {
    if (!s || !massflow || !turbo) return setError(CTBFM_E_ARGUMENT, "null argument");
    return guarded([&] {
        s->solver->getTurbo(massflow, turbo);
        return CTBFM_OK;
    });
}

int ctbfm_profile_kernels(ctbfm_solver* s, int reps, double* out_ms) {
    if (!s || !out_ms || reps < 0) return setError(CTBFM_E_ARGUMENT, "bad argument");
    return guarded([&] {
        s->solver->profileKernels(reps, out_ms);
        return CTBFM_OK;
    });
}

}  // extern "C"
