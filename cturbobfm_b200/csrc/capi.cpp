// extern "C" boundary (include/ctbfm.h). Every entry point catches all C++
// exceptions and turns them into a status code plus a per-thread message, the
// way the reference's main turns exceptions into exit code 1
// (src/turbobfm.cpp:31-36).
#include "../../include/ctbfm.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "host/batch.hpp"
#include "host/config.hpp"
#include "host/mesh.hpp"
#include "host/server.hpp"
#include "host/solver.hpp"

struct ctbfm_solver {
    std::unique_ptr<ctbfm::Config> config;
    std::unique_ptr<ctbfm::Mesh> mesh;
    std::unique_ptr<ctbfm::Solver> solver;
};

struct ctbfm_batch {
    std::unique_ptr<ctbfm::Batch> batch;
};

struct ctbfm_server {
    std::unique_ptr<ctbfm::Server> server;
    std::vector<ctbfm::ServerResult> pending;  // taken from the server, not yet returned
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
    } catch (const std::invalid_argument& e) {
        return setError(CTBFM_E_ARGUMENT, e.what());
    } catch (const std::exception& e) {
        return setError(CTBFM_E_CONFIG, e.what());
    } catch (...) {
        return setError(CTBFM_E_CONFIG, "unknown error");
    }
}

int statusCode(ctbfm_solver* s) {
    const ctbfm::Control c = s->solver->control();
    if (c.status == 3)
        return setError(CTBFM_E_CUDA, "device error: a grid barrier wait of the persistent kernel ran out");
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

// A checked, owned copy of a case description; std::invalid_argument
// (CTBFM_E_ARGUMENT) for a malformed one.
std::unique_ptr<ctbfm::CaseData> caseData(const ctbfm_case_desc* d) {
    if (d->ni < 1 || d->nj < 1 || d->nk < 1) throw std::invalid_argument("ni, nj and nk must be at least 1");
    if (d->nj > (int64_t(1) << 40) / d->ni || d->nk > (int64_t(1) << 40) / (d->ni * d->nj))
        throw std::invalid_argument("the grid is too large");
    if (!d->x || !d->y || !d->z) throw std::invalid_argument("null grid coordinates");
    if (d->n_fields < 0 || d->n_patches < 0 || d->n_settings < 0)
        throw std::invalid_argument("negative count in the case description");
    if (d->n_fields > 0 && (!d->field_names || !d->fields)) throw std::invalid_argument("null grid field arrays");
    if (d->n_patches > 0 && !d->patches) throw std::invalid_argument("null patch array");
    if (d->n_settings > 0 && (!d->keys || !d->values)) throw std::invalid_argument("null settings arrays");
    auto c = std::make_unique<ctbfm::CaseData>();
    c->ni = static_cast<long>(d->ni);
    c->nj = static_cast<long>(d->nj);
    c->nk = static_cast<long>(d->nk);
    const size_t n = static_cast<size_t>(d->ni * d->nj * d->nk);
    c->x.assign(d->x, d->x + n);
    c->y.assign(d->y, d->y + n);
    c->z.assign(d->z, d->z + n);
    for (int32_t q = 0; q < d->n_fields; q++) {
        if (!d->field_names[q] || !d->fields[q]) throw std::invalid_argument("null grid field name or values");
        c->fields.emplace_back(d->field_names[q], std::vector<double>(d->fields[q], d->fields[q] + n));
    }
    for (int32_t q = 0; q < d->n_patches; q++) {
        const ctbfm_patch& p = d->patches[q];
        if (!p.name) throw std::invalid_argument("null patch name");
        ctbfm::PatchRow row;
        row.name = p.name;
        const int64_t r[6] = {p.i_min, p.i_max, p.j_min, p.j_max, p.k_min, p.k_max};
        for (int a = 0; a < 6; a++) row.range[a] = static_cast<long>(r[a]);
        c->patches.push_back(std::move(row));
    }
    for (int32_t q = 0; q < d->n_settings; q++) {
        if (!d->keys[q] || !d->values[q]) throw std::invalid_argument("null setting key or value");
        c->settings.emplace_back(d->keys[q], d->values[q]);
    }
    c->directory = d->directory ? d->directory : "";
    return c;
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

int ctbfm_create(const ctbfm_case_desc* d, ctbfm_solver** out) {
    if (!d || !out) return setError(CTBFM_E_ARGUMENT, "null argument");
    *out = nullptr;
    return guarded([&] {
        const std::unique_ptr<ctbfm::CaseData> data = caseData(d);
        auto s = std::make_unique<ctbfm_solver>();
        s->config = std::make_unique<ctbfm::Config>(data->settings, data->directory);
        s->mesh = data->mesh(*s->config);
        s->solver = std::make_unique<ctbfm::Solver>(*s->config, *s->mesh, &data->patches);
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
        out->device_bytes = static_cast<int64_t>(s->solver->deviceBytes());
        for (int d = 0; d < 3; d++) out->face_tile[d] = s->solver->faceTile(d);
        out->fused_stage = s->solver->fusedStage() ? 1 : 0;
        out->persistent_stage = s->solver->persistentStage() ? 1 : 0;
        for (int m = 0; m < 3; m++) out->tuned_stage_ms[m] = s->solver->tunedStageMs(m);
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

int ctbfm_autotune(ctbfm_solver* s) {
    if (!s) return setError(CTBFM_E_ARGUMENT, "null solver");
    return guarded([&] {
        s->solver->autotune();
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

int ctbfm_write_solution(ctbfm_solver* s, const char* path) {
    if (!s || !path) return setError(CTBFM_E_ARGUMENT, "null argument");
    return guarded([&] {
        s->solver->writeSolution(path);
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

int ctbfm_get_history_time(ctbfm_solver* s, int64_t max_rows, double* time, int64_t* n_rows) {
    if (!s) return setError(CTBFM_E_ARGUMENT, "null solver");
    return guarded([&] {
        const long long r = s->solver->history(max_rows, nullptr, nullptr, nullptr, nullptr, time);
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

int ctbfm_batch_create(ctbfm_solver* const* solvers, int32_t n, ctbfm_batch** out) {
    if (!solvers || !out || n <= 0) return setError(CTBFM_E_ARGUMENT, "bad argument");
    *out = nullptr;
    return guarded([&] {
        std::vector<ctbfm::Solver*> members;
        for (int32_t i = 0; i < n; i++) {
            if (!solvers[i]) throw std::invalid_argument("null solver in batch");
            members.push_back(solvers[i]->solver.get());
        }
        auto b = std::make_unique<ctbfm_batch>();
        b->batch = std::make_unique<ctbfm::Batch>(members);
        *out = b.release();
        return CTBFM_OK;
    });
}

void ctbfm_batch_destroy(ctbfm_batch* b) {
    if (!b) return;
    try {
        delete b;
    } catch (...) {
    }
}

int ctbfm_batch_set_stream(ctbfm_batch* b, void* stream) {
    if (!b) return setError(CTBFM_E_ARGUMENT, "null batch");
    return guarded([&] {
        b->batch->setStream(static_cast<cudaStream_t>(stream));
        return CTBFM_OK;
    });
}

int ctbfm_batch_enqueue(ctbfm_batch* b, int64_t n_iter) {
    if (!b || n_iter < 0) return setError(CTBFM_E_ARGUMENT, "bad argument");
    return guarded([&] {
        b->batch->enqueue(n_iter);
        return CTBFM_OK;
    });
}

int ctbfm_batch_autotune(ctbfm_batch* b) {
    if (!b) return setError(CTBFM_E_ARGUMENT, "null batch");
    return guarded([&] {
        b->batch->autotune();
        return CTBFM_OK;
    });
}

int ctbfm_batch_stage_kernels(ctbfm_batch* b, int32_t* mode, double stage_ms[3]) {
    if (!b || !mode || !stage_ms) return setError(CTBFM_E_ARGUMENT, "bad argument");
    return guarded([&] {
        *mode = b->batch->persistent() ? 2 : b->batch->fusedMode();
        for (int m = 0; m < 3; m++) stage_ms[m] = b->batch->stageMs(m);
        return CTBFM_OK;
    });
}

int ctbfm_batch_step(ctbfm_batch* b, int64_t n_iter, int64_t* n_done) {
    if (!b || n_iter < 0) return setError(CTBFM_E_ARGUMENT, "bad argument");
    return guarded([&] {
        const long long d = b->batch->step(n_iter);
        if (n_done) *n_done = d;
        return CTBFM_OK;
    });
}

int ctbfm_batch_status(ctbfm_batch* b, int32_t* status, int64_t* iterations, double* lognorm, double* best_drop) {
    if (!b) return setError(CTBFM_E_ARGUMENT, "null batch");
    return guarded([&] {
        std::vector<ctbfm::Control> c(static_cast<size_t>(b->batch->size()));
        b->batch->controls(c.data());
        for (size_t i = 0; i < c.size(); i++) {
            if (status) status[i] = c[i].status;
            if (iterations) iterations[i] = c[i].it;
            if (lognorm)
                for (int v = 0; v < 5; v++) lognorm[5 * i + v] = c[i].lognorm[v];
            if (best_drop) best_drop[i] = c[i].best_drop;
        }
        return CTBFM_OK;
    });
}

int ctbfm_promote_fp64(ctbfm_solver* s) {
    if (!s) return setError(CTBFM_E_ARGUMENT, "null solver");
    return guarded([&] {
        s->solver->promoteToFP64();
        return CTBFM_OK;
    });
}

int ctbfm_server_create(uint64_t device_budget_bytes, int32_t max_active, int64_t max_active_nodes,
                        int64_t chunk_iterations, int64_t stall_window, int32_t host_threads, ctbfm_server** out) {
    if (!out) return setError(CTBFM_E_ARGUMENT, "null argument");
    *out = nullptr;
    return guarded([&] {
        ctbfm::ServerOptions o;
        o.budget_bytes = static_cast<size_t>(device_budget_bytes);
        o.max_active = max_active;
        o.max_active_nodes = max_active_nodes;
        o.chunk = chunk_iterations;
        o.stall_window = stall_window;
        o.host_threads = host_threads;
        auto s = std::make_unique<ctbfm_server>();
        s->server = std::make_unique<ctbfm::Server>(o);
        *out = s.release();
        return CTBFM_OK;
    });
}

int ctbfm_server_set_promotion(ctbfm_server* s, double orders) {
    if (!s || !(orders >= 0.0)) return setError(CTBFM_E_ARGUMENT, "bad argument");
    return guarded([&] {
        s->server->setPromoteOrders(orders);
        return CTBFM_OK;
    });
}

int ctbfm_server_get_stats(ctbfm_server* s, ctbfm_server_stats* out) {
    if (!s || !out) return setError(CTBFM_E_ARGUMENT, "null argument");
    return guarded([&] {
        const ctbfm::ServerStats& st = s->server->stats();
        out->rounds = st.rounds;
        out->rebuilds = st.rebuilds;
        out->promotions = st.promotions;
        out->reruns = st.reruns;
        out->wait_s = st.wait_s;
        out->process_s = st.process_s;
        out->rebuild_s = st.rebuild_s;
        out->promote_s = st.promote_s;
        out->release_s = st.release_s;
        out->batch_s = st.batch_s;
        out->prepare_s = st.prepare_s;
        out->enqueue_s = st.enqueue_s;
        out->admit_s = st.admit_s;
        return CTBFM_OK;
    });
}

void ctbfm_server_destroy(ctbfm_server* s) {
    if (!s) return;
    try {
        delete s;
    } catch (...) {
    }
}

int ctbfm_server_submit(ctbfm_server* s, const char* ini_path, int64_t* request_id) {
    if (!s || !ini_path) return setError(CTBFM_E_ARGUMENT, "null argument");
    return guarded([&] {
        const long long id = s->server->submit(ini_path);
        if (request_id) *request_id = id;
        return CTBFM_OK;
    });
}

int ctbfm_server_submit_case(ctbfm_server* s, const ctbfm_case_desc* desc, int64_t* request_id) {
    if (!s || !desc) return setError(CTBFM_E_ARGUMENT, "null argument");
    return guarded([&] {
        const long long id = s->server->submit(caseData(desc));
        if (request_id) *request_id = id;
        return CTBFM_OK;
    });
}

int ctbfm_server_pump(ctbfm_server* s, int32_t* n_active, int32_t* n_waiting) {
    if (!s) return setError(CTBFM_E_ARGUMENT, "null server");
    return guarded([&] {
        int a = 0, w = 0;
        s->server->pump(&a, &w);
        if (n_active) *n_active = a;
        if (n_waiting) *n_waiting = w;
        return CTBFM_OK;
    });
}

int ctbfm_server_results(ctbfm_server* s, ctbfm_result* out, int32_t max, int32_t* n_out) {
    if (!s || (!out && max > 0) || max < 0) return setError(CTBFM_E_ARGUMENT, "bad argument");
    return guarded([&] {
        for (auto& r : s->server->take()) s->pending.push_back(std::move(r));
        const int32_t n = std::min<int32_t>(max, static_cast<int32_t>(s->pending.size()));
        for (int32_t i = 0; i < n; i++) {
            const ctbfm::ServerResult& r = s->pending[i];
            ctbfm_result& o = out[i];
            o.id = r.id;
            o.status = r.status;
            o.precision = r.precision;
            o.iterations = r.iterations;
            o.t_submit = r.t_submit;
            o.t_admit = r.t_admit;
            o.t_done = r.t_done;
            for (int b = 0; b < 6; b++) o.massflow[b] = r.massflow[b];
            for (int b = 0; b < 4; b++) o.turbo[b] = r.turbo[b];
            o.error = r.error;
            const size_t len = std::min(r.message.size(), sizeof(o.message) - 1);
            std::memcpy(o.message, r.message.data(), len);
            o.message[len] = 0;
        }
        s->pending.erase(s->pending.begin(), s->pending.begin() + n);
        if (n_out) *n_out = n;
        return CTBFM_OK;
    });
}

}  // extern "C"
