// Solver: the B200 counterpart of the reference's Solver(Config&, Mesh&) +
// solve() (include/solver.hpp:45-388) for the explicit Runge-Kutta path. It
// validates the inputs exactly as the reference does, then owns the operating
// point's device data (InstanceT) in the working precision chosen by the
// GPU_PRECISION key (fp64, the default, or fp32_kahan), and runs whole
// iterations (time step, boundary profiles, stages, norms, convergence) as a
// device-side sequence captured in CUDA graphs, with no host round trip inside
// a chunk of iterations.
#pragma once

#include <cuda_runtime.h>

#include <array>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "../device/case.cuh"
#include "../device/kernels.hpp"
#include "config.hpp"
#include "engine.hpp"
#include "fluid_table.hpp"
#include "mesh.hpp"
#include "models.hpp"

namespace ctbfm {

class HostFluid;

struct BoundaryPatch {
    std::string name;
    int type = kBcEmpty;
    std::vector<double> values;
    long i_min = 0, i_max = 0, j_min = 0, j_max = 0, k_min = 0, k_max = 0;
    int orientation = 0;  // 0 I start, 1 I end, 2 J start, 3 J end, 4 K start, 5 K end
    std::unique_ptr<BoundaryBase> flux;
};

// One row of the boundary-conditions file (PATCH_NAME, I_MIN .. K_MAX).
struct PatchRow {
    std::string name;
    long range[6] = {0, 0, 0, 0, 0, 0};  // i_min, i_max, j_min, j_max, k_min, k_max
};

// A case held in memory, owned: what input.ini, the grid CSV and
// boundaries.csv carry.
struct CaseData {
    std::vector<std::pair<std::string, std::string>> settings;
    std::string directory;  // where files that settings name resolve ("" = current directory)
    long ni = 0, nj = 0, nk = 0;
    std::vector<double> x, y, z;  // node (i, j, k) at (i*nj + j)*nk + k
    std::vector<std::pair<std::string, std::vector<double>>> fields;
    std::vector<PatchRow> patches;

    std::unique_ptr<Mesh> mesh(const Config& config) const {
        std::vector<std::pair<std::string, const double*>> f;
        for (const auto& c : fields) f.emplace_back(c.first, c.second.data());
        return std::make_unique<Mesh>(config, ni, nj, nk, x.data(), y.data(), z.data(), f);
    }
};

enum Precision { kFP64 = 0, kFP32Kahan = 1 };

class Solver {
public:
    // The boundary patches come from the file BOUNDARY_CONDITIONS_FILEPATH
    // names, or from `patches` when it is given (an in-memory case).
    Solver(Config& config, Mesh& mesh, const std::vector<PatchRow>* patches = nullptr);
    ~Solver();
    Solver(const Solver&) = delete;
    Solver& operator=(const Solver&) = delete;

    void setStream(cudaStream_t s) { stream_ = s ? s : ownStream_; }
    cudaStream_t stream() const { return stream_; }
    int precision() const { return prec_; }
    int stageFusion() const { return fusion_; }
    bool realGas() const { return table_ != nullptr; }
    int faceTile(int d) const { return g64_ ? g64_->faceTile(d) : g32_->faceTile(d); }
    // the autotuner's time of one stage: 0 split, 1 fused, 2 persistent
    double tunedStageMs(int mode) const { return g64_ ? g64_->stageMs(mode) : g32_->stageMs(mode); }
    // iterations run in the persistent kernel k_run
    bool persistentStage() const { return g64_ ? g64_->persistent() : g32_->persistent(); }
    // the group runs the fused stage kernel and this instance can run it
    bool fusedStage() const {
        return g64_ ? (g64_->fusedMode() && i64_->c.fuse_ok) : (g32_->fusedMode() && i32_->c.fuse_ok);
    }

    // Enqueues n iterations (no host sync). Kernels of iterations after
    // convergence / divergence return immediately.
    void enqueue(long long n);
    // runs the group's autotuner now (face tiles, stage fusion) unless it has run
    void autotune();
    // Runs up to n iterations; returns iterations done; syncs.
    long long step(long long n);
    long long solve();
    void computeResidual(double* dt, double* const r[5]);
    // Same outputs as computeResidual, with the face-flux scratch in the
    // library's static device array instead of the solver's face buffers.
    void computeResidualNoAlloc(double* dt, double* const r[5]);

    void getState(double* const out[5]);
    void setState(const double* const in[5]);
    // The current state as a volume CSV in the reference's format
    // (Output::writeSolution, src/output.cpp:384-398), at `path`.
    void writeSolution(const std::string& path);
    void getTurbo(double massflow[6], double turbo[4]);
    // Writes the status word of the device control block (the server pauses
    // a member with a status the kernels skip, and releases it again).
    void setStatus(int status);
    Control control();  // synchronous copy of the control block
    void profileKernels(int reps, double* outMs);
    // Continues a fp32_kahan solve in FP64: the state U - Uc, the control
    // block (iteration, time, convergence reference, plenum), the radial
    // profiles and the history move to a new FP64 instance; the float
    // instance is released. No-op on an FP64 solver.
    void promoteToFP64();
    // promoteToFP64 in two steps: prepare builds the FP64 instance from the
    // current float state (device arrays, uploads, the state converted) and
    // may run while other groups' kernels run, as long as nothing advances
    // this solve (paused, or not in a running batch); commit swaps it in and
    // releases the float instance, with no batch referring to the solve. A
    // paused status (4) in the copied control block becomes running.
    void preparePromotion();
    void commitPromotion();
    bool promotionPrepared() const { return promo_ != nullptr; }
    long long history(long long maxRows, double* lognorm, double* massflow, double* turbo, double* hub,
                      double* time = nullptr);
    size_t deviceBytes() const;

    long ni() const { return mesh_.ni(); }
    long nj() const { return mesh_.nj(); }
    long nk() const { return mesh_.nk(); }
    int topology() const { return static_cast<int>(topo_); }
    int stages() const { return static_cast<int>(coeffs_.size()); }
    long maxIterations() const { return maxIter_; }
    // RESIDUALS_DROP_CONVERGENCE
    int residualDrop() const { return config_.getResidualsDropConvergence(); }

    // device data for batches (nullptr when the solver runs the other precision)
    InstanceT<double>* instance64() { return i64_.get(); }
    InstanceT<float>* instance32() { return i32_.get(); }

private:
    void readBoundaries(const std::vector<PatchRow>* patches);
    void addBoundary(const PatchRow& row);
    void buildBoundaryStructures();
    void setupScalars();
    void setupModels();
    void setupTransport();
    void buildWallMask();
    // TURBULENCE_ACTIVE / TURBULENCE_MODEL: the Spalart-Allmaras settings,
    // wall distance and boundary table (nothing without the model)
    void setupTurbulence();
    void viscousOutputFields(const double* const U[5], std::map<std::string, std::vector<double>>& out);
    // copies a state to the device as it is (setState adds the no-slip wall
    // preprocessing of viscous runs)
    void uploadState(const double* const in[5]);
    void validateSettings();
    template <typename R>
    void uploadArrays(InstanceT<R>& inst);
    template <typename R>
    void initializeState(InstanceT<R>& inst, GroupT<R>& grp);
    template <typename R>
    const DevLut* uploadLut(InstanceT<R>& inst);
    std::unique_ptr<HostFluid> hostFluid() const;
    template <typename F>
    auto visit(F&& f) {
        if (prec_ == kFP32Kahan) return f(*i32_, *g32_);
        return f(*i64_, *g64_);
    }

    Config& config_;
    Mesh& mesh_;
    Topology topo_;
    std::vector<double> coeffs_;
    long maxIter_ = 0;
    int prec_ = kFP64;
    int fusion_ = 2;  // GPU_STAGE_FUSION: 0 split stage kernels, 1 fused stage kernel, 2 autotuned
    std::unique_ptr<AdvectionBase> advection_;
    std::unique_ptr<SourceBFMBase> bfm_;
    std::unique_ptr<FluidTable> table_;  // FLUID_MODEL = real
    std::vector<BoundaryPatch> boundaries_;
    bool needTurbo_ = false;
    double periodicAngleDeg_ = 0.0, periodicAngleRad_ = 0.0, periodicTransl_ = 0.0;
    DevCaseT<double> proto_{};  // scalar settings shared by both precisions
    std::vector<signed char> mapI_, mapJ_, mapK_;
    std::vector<unsigned char> wall_;  // viscous runs: 1 on no-slip wall nodes
    // Spalart-Allmaras: wall distance per node, the boundary rows of DevCaseT
    // sa_bc and the initial nu hat
    std::vector<double> saWd_;
    std::vector<int> saBc_;
    double saInitNuHat_ = 0.0;
    std::vector<double> profP_, profR_;

    std::unique_ptr<InstanceT<double>> i64_;
    std::unique_ptr<GroupT<double>> g64_;
    std::unique_ptr<InstanceT<float>> i32_;
    std::unique_ptr<GroupT<float>> g32_;
    struct Promotion {
        std::unique_ptr<InstanceT<double>> inst;
        std::unique_ptr<GroupT<double>> grp;
        Control ctl;
    };
    std::unique_ptr<Promotion> promo_;  // a prepared promotion, not yet committed
    Control* hostCtl_ = nullptr;  // pinned
    cudaStream_t ownStream_ = nullptr, stream_ = nullptr;
    int device_ = 0;  // the CUDA device current when the solver was created
};

}  // namespace ctbfm
