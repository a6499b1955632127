// Solver: the B200 counterpart of the reference's Solver(Config&, Mesh&) +
// solve() (include/solver.hpp:45-388) for the explicit Runge-Kutta path. It
// owns every device buffer of one operating point and runs the whole
// iteration (time step, boundary profiles, stages, norms, convergence) as a
// device-side sequence, captured in CUDA graphs, with no host round trip
// inside a chunk of iterations.
#pragma once

#include <cuda_runtime.h>

#include <array>
#include <memory>
#include <string>
#include <vector>

#include "../device/case.cuh"
#include "../device/kernels.hpp"
#include "config.hpp"
#include "mesh.hpp"
#include "models.hpp"

namespace ctbfm {

struct BoundaryPatch {
    std::string name;
    int type = kBcEmpty;
    std::vector<double> values;
    long i_min = 0, i_max = 0, j_min = 0, j_max = 0, k_min = 0, k_max = 0;
    int orientation = 0;  // 0 I start, 1 I end, 2 J start, 3 J end, 4 K start, 5 K end
    std::unique_ptr<BoundaryBase> flux;
};

class CudaError : public std::runtime_error {
public:
    using std::runtime_error::runtime_error;
};

class Solver {
public:
    Solver(Config& config, Mesh& mesh);
    ~Solver();
    Solver(const Solver&) = delete;
    Solver& operator=(const Solver&) = delete;

    void setStream(cudaStream_t s) { stream_ = s ? s : ownStream_; }
    cudaStream_t stream() const { return stream_; }

    // Enqueues n iterations (no host sync). Kernels of iterations after
    // convergence / divergence return immediately.
    void enqueue(long long n);
    // Runs up to n iterations; returns iterations done; syncs.
    long long step(long long n);
    long long solve();
    void computeResidual(double* dt, double* const r[5]);
    // Same outputs as computeResidual, with the face-flux scratch in the
    // library's static device array instead of the solver's face buffers.
    void computeResidualNoAlloc(double* dt, double* const r[5]);

    void getState(double* const out[5]);
    void setState(const double* const in[5]);
    void getTurbo(double massflow[6], double turbo[4]);
    Control control();  // synchronous copy of the control block
    void profileKernels(int reps, double* outMs);
    size_t deviceBytes() const { return deviceBytes_; }
    long long history(long long maxRows, double* lognorm, double* massflow, double* turbo, double* hub);

    long ni() const { return mesh_.ni(); }
    long nj() const { return mesh_.nj(); }
    long nk() const { return mesh_.nk(); }
    int topology() const { return static_cast<int>(topo_); }
    int stages() const { return static_cast<int>(coeffs_.size()); }
    long maxIterations() const { return maxIter_; }

private:
    void readBoundaries();
    void buildBoundaryStructures();
    void uploadBoundaryStructures();
    void validateSettings();
    void setupModels();
    void upload();
    void initializeSolution();
    void initializeProfilesAndPlenum();
    void enqueueIteration();
    void setLimits(long long itStop, long long histBase);
    void captureGraph();
    double* alloc(size_t count);
    const double* upload(const std::vector<double>& v);
    void check(cudaError_t e, const char* what);

    Config& config_;
    Mesh& mesh_;
    Topology topo_;
    std::vector<double> coeffs_;
    long maxIter_ = 0;
    std::unique_ptr<AdvectionBase> advection_;
    std::unique_ptr<SourceBFMBase> bfm_;
    std::vector<BoundaryPatch> boundaries_;
    bool needTurbo_ = false, profiles_ = false;
    double periodicAngleDeg_ = 0.0, periodicAngleRad_ = 0.0, periodicTransl_ = 0.0;

    DevCase c_{};
    std::vector<signed char> mapI_, mapJ_, mapK_;
    std::vector<double> profP_, profR_;
    std::vector<void*> allocations_;
    Control* hostCtl_ = nullptr;  // pinned
    cudaStream_t ownStream_ = nullptr, stream_ = nullptr;
    cudaGraphExec_t graph_ = nullptr;
    int graphIters_ = 0;
    long long itHost_ = 0;  // iteration counter as last seen by the host
    size_t deviceBytes_ = 0;
};

}  // namespace ctbfm
