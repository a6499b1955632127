// Batch: any number of solvers of one working precision advanced together,
// one launch per kernel family for all of them (GroupT over their
// instances). The reference runs one process per operating point
// (python/Run_All_Cases.py:18-98); here a whole compressor map shares each
// launch, so small grids no longer leave the GPU idle.
#pragma once

#include <cuda_runtime.h>

#include <memory>
#include <vector>

#include "engine.hpp"
#include "solver.hpp"

namespace ctbfm {

class Batch {
public:
    // All members need the same GPU_PRECISION; they must outlive the batch,
    // and must not be stepped on their own while the batch is in use.
    explicit Batch(const std::vector<Solver*>& members);
    ~Batch();
    Batch(const Batch&) = delete;
    Batch& operator=(const Batch&) = delete;

    void setStream(cudaStream_t s) { stream_ = s ? s : ownStream_; }
    cudaStream_t stream() const { return stream_; }
    int size() const { return static_cast<int>(members_.size()); }
    int precision() const { return prec_; }

    // n iterations of every member still running, no host synchronisation
    void enqueue(long long n);
    // runs the group's autotuner now (face tiles, stage fusion) unless it has run
    void autotune();
    int fusedMode() const { return g32_ ? g32_->fusedMode() : g64_->fusedMode(); }
    bool persistent() const { return g32_ ? g32_->persistent() : g64_->persistent(); }
    GroupTuning tuning() const { return g32_ ? g32_->tuning() : g64_->tuning(); }
    void adopt(const GroupTuning& t) {
        if (g32_) g32_->adopt(t);
        else g64_->adopt(t);
    }
    long long nodes() const { return g32_ ? g32_->nodes() : g64_->nodes(); }
    double stageMs(int mode) const { return g32_ ? g32_->stageMs(mode) : g64_->stageMs(mode); }
    // enqueue + synchronise; returns the most iterations any member advanced
    long long step(long long n);
    // every member's control block (synchronous), out[0..size())
    void controls(Control* out);

private:
    std::vector<Solver*> members_;
    int prec_ = kFP64;
    std::unique_ptr<GroupT<double>> g64_;
    std::unique_ptr<GroupT<float>> g32_;
    Control* dCtl_ = nullptr;  // gathered control blocks (device)
    Control* hCtl_ = nullptr;  // and their pinned host copy
    cudaStream_t ownStream_ = nullptr, stream_ = nullptr;
};

}  // namespace ctbfm
