// Server: continuous batching of operating-point solves. The reference runs
// one process per operating point to the end (python/Run_All_Cases.py:18-98);
// here requests arrive at any time, are prepared on host worker threads
// (input parsing, grid metrics), admitted in arrival order while device
// memory and slots allow, advance together with every other admitted solve
// (one Batch per working precision, each on its own stream, so FP32 and FP64
// work overlaps), and retire the moment they converge, diverge or reach
// N_ITERATIONS. A fp32_kahan solve whose convergence progress stalls for
// stall_window iterations, or that comes within promote_orders of its
// residual drop, continues in FP64 (the precision pattern: float for the
// bulk of the iterations, the convergence test and state in FP64).
#pragma once

#include <condition_variable>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "batch.hpp"
#include "config.hpp"
#include "mesh.hpp"
#include "solver.hpp"

namespace ctbfm {

struct ServerResult {
    long long id = 0;
    int status = -1;  // CTBFM_STATUS_*, -1 when the request failed before running
    int precision = 0;
    long long iterations = 0;
    double t_submit = 0, t_admit = 0, t_done = 0;  // seconds since the server started
    double massflow[6] = {0, 0, 0, 0, 0, 0};
    double turbo[4] = {0, 0, 0, 0};
    int error = 0;  // CTBFM_OK or the request's error code
    std::string message;
};

// Where a server's time went (seconds of wall time on the pumping thread).
struct ServerStats {
    long long rounds = 0;      // scheduling rounds that enqueued a chunk
    long long rebuilds = 0;    // batch rebuilds (membership changes applied)
    long long promotions = 0;  // fp32_kahan solves continued in FP64
    long long reruns = 0;      // diverged fp32_kahan solves run again in FP64
    double wait_s = 0;         // waiting for the chunk in flight (the device busy)
    double process_s = 0;      // retiring, pausing and reporting after a chunk
    double rebuild_s = 0;      // applying changes (promotions, releases) and rebuilding the batches
    double promote_s = 0;      //   of which promoting solves to FP64 (and re-creating diverged ones)
    double release_s = 0;      //   of which releasing finished solves
    double batch_s = 0;        //   of which releasing and building the two batches
    double prepare_s = 0;      // building the FP64 side of paused solves, while a chunk runs
    double enqueue_s = 0;      // enqueueing chunks (includes a new batch's autotuning)
    double admit_s = 0;        // building admitted solves (device allocation, upload) while a chunk runs
};

struct ServerOptions {
    size_t budget_bytes = 0;      // device memory the admitted solves may hold (0: 90 % of free)
    int max_active = 1024;        // admitted solves at most
    long long max_active_nodes = 0;  // grid nodes of the admitted solves together at most (0: no limit)
    long long chunk = 200;        // iterations between scheduling rounds
    long long stall_window = 0;   // fp32_kahan -> FP64 after this many iterations without progress, and
                                  // diverged fp32_kahan solves re-run in FP64 (0: neither)
    int host_threads = 4;         // workers preparing requests
    double promote_orders = 0.0;  // fp32_kahan -> FP64 once within this many orders of the residual drop
                                  // (best_drop >= RESIDUALS_DROP_CONVERGENCE - promote_orders; 0: off)
};

class Server {
public:
    explicit Server(const ServerOptions& o);
    ~Server();
    Server(const Server&) = delete;
    Server& operator=(const Server&) = delete;

    // Sets ServerOptions::promote_orders (before the first submission).
    void setPromoteOrders(double orders) { opt_.promote_orders = orders; }
    // Queues a request (thread safe); its host preparation starts at once.
    long long submit(const std::string& iniPath);
    // The same for a case held in memory (the server keeps the copy).
    long long submit(std::unique_ptr<CaseData> data);
    // One scheduling round: waits for the chunk the previous round enqueued
    // and retires, promotes and re-runs from its results; the solves built
    // during that chunk join the batches; the next chunk of `chunk`
    // iterations of every admitted solve is enqueued; and while it runs on
    // the device the next requests that fit are built (device memory and
    // upload), to join at the next round. Returns without waiting for the
    // chunk it enqueued.
    void pump(int* active, int* waiting);
    // Requests finished since the last call.
    std::vector<ServerResult> take();
    const ServerStats& stats() const { return stats_; }
    double now() const;

private:
    struct Job {
        long long id = 0;
        std::string ini;
        std::unique_ptr<CaseData> data;  // in-memory case, released once the mesh is built
        std::vector<PatchRow> patches;   // its boundary patches
        double t_submit = 0, t_admit = 0;
        bool prepared = false;
        int error = 0;
        std::string message;
        long long nodes = 0;
        std::unique_ptr<Config> config;
        std::unique_ptr<Mesh> mesh;
        std::unique_ptr<Solver> solver;  // declared last: released before the mesh and config it refers to
        size_t bytes = 0;
        bool rerun = false;  // a diverged float solve restarted in FP64
        // a change that waits for the next rebuild of the batches: 1 finished
        // (result reported; its device memory is held while a batch refers to
        // it), 2 continues in FP64 (paused in its float batch), 3 runs again
        // from its initial state in FP64 (diverged; the kernels skip it)
        int action = 0;
    };
    long long enqueue(std::unique_ptr<Job> j);
    void worker();
    void rebuild();
    // builds the Solvers of queued requests that fit the slots, memory and
    // node limits, in arrival order, into pending_
    void admit();
    // the pending solves join the active ones (next chunk)
    void joinPending();
    // every active solve's control block after the chunk in flight
    std::vector<Control> gather();
    // retire finished solves, re-run diverged float solves in FP64, promote
    // stalled float solves (batches idle)
    void process(const std::vector<Control>& ctl);
    void retire(std::unique_ptr<Job> job, const Control* ctl, int error, const std::string& msg);
    void report(Job& job, const Control* ctl, int error, const std::string& msg);
    // the marked changes, with both batches released: finished solves
    // released, paused ones promoted, diverged ones rebuilt in FP64
    void applyChanges();
    size_t estimate(const Job& j) const;

    ServerOptions opt_;
    double t0_ = 0;
    std::mutex mu_;
    std::condition_variable cv_;
    std::deque<Job*> prep_;                   // awaiting a worker
    std::deque<std::unique_ptr<Job>> queue_;  // submitted, in arrival order
    std::vector<std::thread> workers_;
    bool stop_ = false;
    long long nextId_ = 1;
    std::vector<std::unique_ptr<Job>> active_;
    std::vector<std::unique_ptr<Job>> pending_;  // built during the chunk in flight, join at the next round
    bool inflight_ = false;                      // a chunk of the current batches is enqueued
    // autotuner results per precision (0 fp64, 1 fp32_kahan), adopted by
    // later batches whose node count is within 4x of the tuned one
    GroupTuning tuned_[2];
    std::unique_ptr<Batch> b64_, b32_;
    std::vector<int> idx64_, idx32_;  // active_ index of each batch member
    size_t used_ = 0;
    long long usedNodes_ = 0;
    double bytesPerNode_[2] = {0, 0};  // measured per precision (0: not yet)
    std::vector<ServerResult> done_;
    ServerStats stats_;
    int waitRounds_ = 0;  // rounds in which marked changes waited for a rebuild
};

}  // namespace ctbfm
