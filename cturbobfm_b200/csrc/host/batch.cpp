// Batch: see batch.hpp.
#include "batch.hpp"

#include <algorithm>
#include <cstring>

namespace ctbfm {

Batch::Batch(const std::vector<Solver*>& members) : members_(members) {
    if (members_.empty()) throw std::invalid_argument("a batch needs at least one solver");
    prec_ = members_[0]->precision();
    for (Solver* m : members_) {
        if (!m) throw std::invalid_argument("null solver in batch");
        if (m->precision() != prec_) throw std::invalid_argument("all solvers of a batch need the same GPU_PRECISION");
    }
    for (size_t a = 0; a < members_.size(); a++)
        for (size_t b = a + 1; b < members_.size(); b++)
            if (members_[a] == members_[b]) throw std::invalid_argument("a solver appears twice in the batch");
    for (Solver* m : members_) cudaCheck(cudaStreamSynchronize(m->stream()), "cudaStreamSynchronize");
    if (prec_ == kFP32Kahan) {
        std::vector<InstanceT<float>*> v;
        for (Solver* m : members_) v.push_back(m->instance32());
        g32_ = std::make_unique<GroupT<float>>(v);
    } else {
        std::vector<InstanceT<double>*> v;
        for (Solver* m : members_) v.push_back(m->instance64());
        g64_ = std::make_unique<GroupT<double>>(v);
    }
    // the split stage if a member asks for it, else the fused stage if a
    // member asks for it, else the persistent kernel if a member asks for it
    // (split if the batch cannot run it), else autotuned
    static const int rank[4] = {0, 1, 3, 2};  // by GPU_STAGE_FUSION: split, fused, auto, persistent
    static const int byRank[4] = {0, 1, 3, 2};
    int r = 3;
    for (Solver* m : members_) r = std::min(r, rank[m->stageFusion()]);
    const int fusion = byRank[r];
    if (g32_) g32_->setFusedMode(fusion);
    else g64_->setFusedMode(fusion);
    cudaCheck(cudaStreamCreateWithFlags(&ownStream_, cudaStreamNonBlocking), "cudaStreamCreate");
    stream_ = ownStream_;
    dCtl_ = static_cast<Control*>(deviceAlloc(members_.size() * sizeof(Control)));
    hCtl_ = static_cast<Control*>(pinnedAlloc(members_.size() * sizeof(Control)));
}

Batch::~Batch() {
    if (ownStream_) cudaStreamSynchronize(ownStream_);
    if (stream_ && stream_ != ownStream_) cudaStreamSynchronize(stream_);
    g32_.reset();
    g64_.reset();
    deviceFree(dCtl_);
    pinnedFree(hCtl_, members_.size() * sizeof(Control));
    if (ownStream_) cudaStreamDestroy(ownStream_);
}

void Batch::enqueue(long long n) {
    if (g32_) g32_->enqueue(n, stream_);
    else g64_->enqueue(n, stream_);
}

void Batch::autotune() {
    if (g32_ && !g32_->tuned()) g32_->tune(stream_);
    if (g64_ && !g64_->tuned()) g64_->tune(stream_);
    cudaCheck(cudaStreamSynchronize(stream_), "cudaStreamSynchronize");
}

void Batch::controls(Control* out) {
    if (g32_) cudaCheck(Launcher<float>::gatherControl(g32_->view(), dCtl_, stream_), "launch k_gather_control");
    else cudaCheck(Launcher<double>::gatherControl(g64_->view(), dCtl_, stream_), "launch k_gather_control");
    cudaCheck(cudaMemcpyAsync(hCtl_, dCtl_, members_.size() * sizeof(Control), cudaMemcpyDeviceToHost, stream_),
              "cudaMemcpyAsync");
    cudaCheck(cudaStreamSynchronize(stream_), "cudaStreamSynchronize");
    std::memcpy(out, hCtl_, members_.size() * sizeof(Control));
}

long long Batch::step(long long n) {
    std::vector<Control> before(members_.size()), after(members_.size());
    controls(before.data());
    enqueue(n);
    controls(after.data());
    long long most = 0;
    for (size_t i = 0; i < members_.size(); i++) {
        if (after[i].status == 3) throw CudaError("device error: a grid barrier wait of the persistent kernel ran out");
        most = std::max(most, after[i].it - before[i].it);
    }
    return most;
}

}  // namespace ctbfm
