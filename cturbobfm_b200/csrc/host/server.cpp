// Server: see server.hpp.
#include "server.hpp"

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>

namespace ctbfm {

namespace {
double steadySeconds() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}
}  // namespace

Server::Server(const ServerOptions& o) : opt_(o), t0_(steadySeconds()) {
    if (opt_.chunk <= 0) throw std::invalid_argument("chunk must be positive");
    if (opt_.max_active <= 0) throw std::invalid_argument("max_active must be positive");
    if (opt_.max_active_nodes < 0) throw std::invalid_argument("max_active_nodes must be >= 0");
    if (opt_.stall_window < 0) throw std::invalid_argument("stall_window must be >= 0");
    const int nt = std::max(1, opt_.host_threads);
    for (int t = 0; t < nt; t++) workers_.emplace_back([this] { worker(); });
}

Server::~Server() {
    {
        std::lock_guard<std::mutex> l(mu_);
        stop_ = true;
    }
    cv_.notify_all();
    for (auto& w : workers_) w.join();
    b32_.reset();
    b64_.reset();
    active_.clear();
    pending_.clear();
}

double Server::now() const { return steadySeconds() - t0_; }

long long Server::submit(const std::string& iniPath) {
    auto j = std::make_unique<Job>();
    j->ini = iniPath;
    j->t_submit = now();
    return enqueue(std::move(j));
}

long long Server::submit(std::unique_ptr<CaseData> data) {
    auto j = std::make_unique<Job>();
    j->data = std::move(data);
    j->t_submit = now();
    return enqueue(std::move(j));
}

long long Server::enqueue(std::unique_ptr<Job> j) {
    std::lock_guard<std::mutex> l(mu_);
    j->id = nextId_++;
    prep_.push_back(j.get());
    const long long id = j->id;
    queue_.push_back(std::move(j));
    cv_.notify_one();
    return id;
}

// Host preparation: the Config and Mesh constructors (input file, grid, dual
// grid, metrics, blockage gradient). No CUDA call happens here.
void Server::worker() {
    while (true) {
        Job* j = nullptr;
        {
            std::unique_lock<std::mutex> l(mu_);
            cv_.wait(l, [this] { return stop_ || !prep_.empty(); });
            if (stop_) return;
            j = prep_.front();
            prep_.pop_front();
        }
        std::unique_ptr<Config> cfg;
        std::unique_ptr<Mesh> mesh;
        int err = 0;
        std::string msg;
        try {
            if (j->data) {
                cfg = std::make_unique<Config>(j->data->settings, j->data->directory);
                mesh = j->data->mesh(*cfg);
            } else {
                cfg = std::make_unique<Config>(j->ini);
                mesh = std::make_unique<Mesh>(*cfg);
            }
        } catch (const std::exception& e) {
            err = 1;  // CTBFM_E_CONFIG
            msg = e.what();
        }
        std::lock_guard<std::mutex> l(mu_);
        j->config = std::move(cfg);
        j->mesh = std::move(mesh);
        if (j->data) {
            j->patches = std::move(j->data->patches);
            j->data.reset();
        }
        j->error = err;
        j->message = msg;
        j->nodes = j->mesh ? static_cast<long long>(j->mesh->nodes()) : 0;
        j->prepared = true;
    }
}

size_t Server::estimate(const Job& j) const {
    const bool f32 = j.config && j.config->has("GPU_PRECISION") && j.config->get("GPU_PRECISION") == "fp32_kahan";
    const double per = bytesPerNode_[f32 ? 1 : 0] > 0 ? bytesPerNode_[f32 ? 1 : 0] : (f32 ? 700.0 : 1200.0);
    return static_cast<size_t>(per * static_cast<double>(j.nodes) * 1.05) + (size_t(1) << 20);
}

// The result of a request, reported now; the job itself stays as it is.
void Server::report(Job& job, const Control* ctl, int error, const std::string& msg) {
    ServerResult r;
    r.id = job.id;
    r.t_submit = job.t_submit;
    r.t_admit = job.t_admit;
    r.error = error;
    r.message = msg;
    if (job.solver && ctl) {
        r.status = ctl->status;
        if (ctl->status == 3 && !r.error) {
            r.error = 2;  // CTBFM_E_CUDA
            r.message = "device error: a grid barrier wait of the persistent kernel ran out";
        }
        r.iterations = ctl->it;
        r.precision = job.solver->precision();
        try {
            job.solver->getTurbo(r.massflow, r.turbo);
        } catch (const std::exception& e) {
            r.error = 2;  // CTBFM_E_CUDA
            r.message = e.what();
        }
    }
    r.t_done = now();
    done_.push_back(std::move(r));
}

// Reports and releases a job that no batch refers to.
void Server::retire(std::unique_ptr<Job> job, const Control* ctl, int error, const std::string& msg) {
    report(*job, ctl, error, msg);
    job.reset();  // releases the solve's device memory
}

void Server::rebuild() {
    b32_.reset();
    b64_.reset();
    idx32_.clear();
    idx64_.clear();
    std::vector<Solver*> m32, m64;
    for (size_t i = 0; i < active_.size(); i++) {
        Solver* s = active_[i]->solver.get();
        if (s->precision() == kFP32Kahan) {
            m32.push_back(s);
            idx32_.push_back(static_cast<int>(i));
        } else {
            m64.push_back(s);
            idx64_.push_back(static_cast<int>(i));
        }
    }
    // a batch of about the size an earlier batch was tuned on takes that
    // tuning; otherwise it times its own at its first chunk
    auto build = [this](std::vector<Solver*>& m, int p) {
        auto b = std::make_unique<Batch>(m);
        const GroupTuning& t = tuned_[p];
        const long long n = b->nodes();
        if (t.valid && n * 4 >= t.nodes && n <= 4 * t.nodes) b->adopt(t);
        return b;
    };
    if (!m32.empty()) b32_ = build(m32, 1);
    if (!m64.empty()) b64_ = build(m64, 0);
}

// Admission in arrival order while slots, device memory and the node limit
// allow (the solves built but not yet running count too); a request whose
// preparation failed retires at once.
void Server::admit() {
    while (true) {
        std::unique_ptr<Job> j;
        {
            std::lock_guard<std::mutex> l(mu_);
            if (queue_.empty() || !queue_.front()->prepared) break;
            if (queue_.front()->error == 0) {
                const bool idle = active_.empty() && pending_.empty();
                if (static_cast<int>(active_.size() + pending_.size()) >= opt_.max_active) break;
                const size_t need = estimate(*queue_.front());
                size_t budget = opt_.budget_bytes;
                if (budget == 0) {
                    size_t freeB = 0, totalB = 0;
                    cudaCheck(cudaMemGetInfo(&freeB, &totalB), "cudaMemGetInfo");
                    freeB += devicePoolIdle();  // released solves' blocks, kept for reuse
                    budget = used_ + freeB * 9 / 10;
                }
                if (used_ + need > budget && !idle) break;
                if (opt_.max_active_nodes > 0 && usedNodes_ + queue_.front()->nodes > opt_.max_active_nodes && !idle)
                    break;
            }
            j = std::move(queue_.front());
            queue_.pop_front();
        }
        if (j->error) {
            const int err = j->error;
            const std::string msg = j->message;
            retire(std::move(j), nullptr, err, msg);
            continue;
        }
        try {
            j->solver = std::make_unique<Solver>(*j->config, *j->mesh, j->ini.empty() ? &j->patches : nullptr);
        } catch (const ConfigError& e) {
            const std::string msg = e.what();
            retire(std::move(j), nullptr, 1, msg);
            continue;
        } catch (const CudaError& e) {
            const std::string msg = e.what();
            retire(std::move(j), nullptr, 2, msg);
            continue;
        }
        j->bytes = j->solver->deviceBytes();
        const int p = j->solver->precision() == kFP32Kahan ? 1 : 0;
        if (bytesPerNode_[p] == 0 && j->nodes > 0)
            bytesPerNode_[p] = static_cast<double>(j->bytes) / static_cast<double>(j->nodes);
        used_ += j->bytes;
        usedNodes_ += j->nodes;
        pending_.push_back(std::move(j));
    }
}

void Server::joinPending() {
    if (pending_.empty()) return;
    const double t = now();
    for (auto& j : pending_) {
        j->t_admit = t;
        active_.push_back(std::move(j));
    }
    pending_.clear();
}

std::vector<Control> Server::gather() {
    std::vector<Control> ctl(active_.size());
    std::vector<Control> tmp;
    if (b32_) {
        tmp.resize(idx32_.size());
        b32_->controls(tmp.data());
        for (size_t m = 0; m < idx32_.size(); m++) ctl[idx32_[m]] = tmp[m];
    }
    if (b64_) {
        tmp.resize(idx64_.size());
        b64_->controls(tmp.data());
        for (size_t m = 0; m < idx64_.size(); m++) ctl[idx64_[m]] = tmp[m];
    }
    return ctl;
}

// After a chunk, with both batches idle: marks the changes, which wait for
// the next rebuild. A finished solve is reported at once; a float solve that
// moves to FP64 is paused in its float batch (status 4, which the kernels
// skip) at exactly this iteration, so its result depends on its own request
// alone, however long the move waits.
void Server::process(const std::vector<Control>& ctl) {
    for (size_t i = 0; i < active_.size(); i++) {
        Job& j = *active_[i];
        if (j.action) continue;
        const Control& c = ctl[i];
        const bool f32 = j.solver->precision() == kFP32Kahan;
        if (opt_.stall_window > 0 && c.status == 2 && f32 && !j.rerun) {
            j.action = 3;
            continue;
        }
        if (c.status != 0 || c.it >= j.solver->maxIterations()) {
            report(j, &c, 0, "");
            j.action = 1;
            continue;
        }
        if (f32 && ((opt_.stall_window > 0 && c.it - c.it_best >= opt_.stall_window) ||
                    (opt_.promote_orders > 0 && c.best_drop >= j.solver->residualDrop() - opt_.promote_orders))) {
            j.solver->setStatus(4);
            j.action = 2;
        }
    }
}

void Server::applyChanges() {
    const double td = now();
    b32_.reset();
    b64_.reset();
    stats_.batch_s += now() - td;
    std::vector<std::unique_ptr<Job>> keep;
    for (auto& j : active_) {
        const double t0 = now();
        if (j->action == 1) {
            used_ -= std::min(used_, j->bytes);
            usedNodes_ -= std::min(usedNodes_, j->nodes);
            j.reset();
            stats_.release_s += now() - t0;
            continue;
        }
        if (j->action == 2) {
            used_ -= std::min(used_, j->bytes);
            j->solver->commitPromotion();  // prepared while a chunk ran, or now
            j->bytes = j->solver->deviceBytes();
            used_ += j->bytes;
            stats_.promotions++;
        } else if (j->action == 3) {
            // a float solve whose residual became NaN/Inf starts again from
            // its initial state in FP64; the outcome depends on the request alone
            used_ -= std::min(used_, j->bytes);
            j->solver.reset();
            j->rerun = true;
            j->config->set("GPU_PRECISION", "fp64");
            stats_.reruns++;
            try {
                j->solver = std::make_unique<Solver>(*j->config, *j->mesh, j->ini.empty() ? &j->patches : nullptr);
                j->bytes = j->solver->deviceBytes();
                used_ += j->bytes;
            } catch (const std::exception& e) {
                usedNodes_ -= std::min(usedNodes_, j->nodes);
                const std::string msg = e.what();
                retire(std::move(j), nullptr, 2, msg);
                continue;
            }
        }
        if (j->action) stats_.promote_s += now() - t0;
        j->action = 0;
        keep.push_back(std::move(j));
    }
    active_ = std::move(keep);
}

// Rounds that marked changes (finished, paused or diverged solves, solves
// built during a chunk) may wait before the batches are rebuilt for them,
// unless they make up a quarter of the membership or nothing is left running.
constexpr int kMaxWaitRounds = 2;

void Server::pump(int* nActive, int* nWaiting) {
    double t = now();
    // 1. the chunk in flight: wait for it, then mark what finished, diverged
    //    or moves to FP64, with the batches idle
    if (inflight_) {
        const std::vector<Control> ctl = gather();
        inflight_ = false;
        const double t1 = now();
        stats_.wait_s += t1 - t;
        process(ctl);
        t = now();
        stats_.process_s += t - t1;
    }
    // with nothing on the device, requests are admitted right away
    if (active_.empty() && pending_.empty()) {
        admit();
        const double t1 = now();
        stats_.admit_s += t1 - t;
        t = t1;
    }
    // 2. the batches are rebuilt for the marked changes and the solves built
    //    during the last chunk once they are worth it (a quarter of the
    //    membership, nothing left running, no batch yet, or waiting
    //    kMaxWaitRounds rounds); until then the batches run unchanged, their
    //    graphs and tuning reused
    auto count = [this](size_t& changed, size_t running[2]) {
        changed = pending_.size();
        running[0] = running[1] = 0;
        for (auto& j : active_) {
            if (j->action) changed++;
            else running[j->solver->precision() == kFP32Kahan ? 1 : 0]++;
        }
    };
    size_t changed = 0, running[2] = {0, 0};
    count(changed, running);
    if (changed) {
        waitRounds_++;
        const size_t members = active_.size() + pending_.size();
        if ((!b32_ && !b64_) || running[0] + running[1] == 0 || changed * 4 >= members ||
            waitRounds_ >= kMaxWaitRounds) {
            applyChanges();
            joinPending();
            const double tb = now();
            rebuild();
            stats_.batch_s += now() - tb;
            stats_.rebuilds++;
            waitRounds_ = 0;
            count(changed, running);
        }
        const double t1 = now();
        stats_.rebuild_s += t1 - t;
        t = t1;
    }
    // 3. the next chunk of every batch with a running member; the two
    //    precision groups run on their own streams and overlap on the device
    if (b32_ && running[1]) {
        b32_->enqueue(opt_.chunk);
        inflight_ = true;
    }
    if (b64_ && running[0]) {
        b64_->enqueue(opt_.chunk);
        inflight_ = true;
    }
    if (inflight_) {
        stats_.rounds++;
        // a batch that timed its own tuning hands it on to later batches
        if (b32_ && b32_->tuning().valid) tuned_[1] = b32_->tuning();
        if (b64_ && b64_->tuning().valid) tuned_[0] = b64_->tuning();
    }
    const double t2 = now();
    stats_.enqueue_s += t2 - t;
    // 4. while the chunk runs: the FP64 side of the paused solves (their
    //    float state does not change while they are paused), then the next
    //    requests that fit (device allocation and upload); both join at a
    //    later round
    for (auto& j : active_)
        if (j->action == 2 && !j->solver->promotionPrepared()) j->solver->preparePromotion();
    const double t3 = now();
    stats_.prepare_s += t3 - t2;
    admit();
    stats_.admit_s += now() - t3;
    if (nActive) *nActive = static_cast<int>(active_.size() + pending_.size());
    if (nWaiting) {
        std::lock_guard<std::mutex> l(mu_);
        *nWaiting = static_cast<int>(queue_.size());
    }
}

std::vector<ServerResult> Server::take() {
    std::vector<ServerResult> out;
    out.swap(done_);
    return out;
}

}  // namespace ctbfm
