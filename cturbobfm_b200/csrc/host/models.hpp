// Host-side model objects with the reference's class names. In the reference
// these classes are called per face / per node through virtual functions
// (include/advection_base.hpp:21-25, include/boundary_base.hpp:26-32,
// include/source_bfm_base.hpp:20-31). Here they are parameter carriers: each
// one validates its settings and writes the parameters the batched device
// kernels read; the arithmetic itself runs on the GPU. They fill the
// double-typed scalar description (DevCase) that the solver copies into the
// instance of either working precision.
#pragma once

#include <memory>
#include <string>
#include <vector>

#include "../device/case.cuh"
#include "config.hpp"

namespace ctbfm {

// AdvectionBase / AdvectionJst / AdvectionRoe (include/advection_*.hpp).
class AdvectionBase {
public:
    explicit AdvectionBase(const Config& config)
        : muscl_(config.getMUSCLreconstruction()), limiter_(config.getFluxLimiter()) {}
    virtual ~AdvectionBase() = default;
    virtual Scheme scheme() const = 0;
    void configure(DevCase& c) const {
        c.scheme = static_cast<int>(scheme());
        c.muscl = muscl_ ? 1 : 0;
        c.limiter = static_cast<int>(limiter_);
    }

protected:
    bool muscl_;
    Limiter limiter_;
};

class AdvectionJst : public AdvectionBase {
public:
    using AdvectionBase::AdvectionBase;
    Scheme scheme() const override { return Scheme::JST; }
    // include/advection_jst.hpp:23; the device kernel uses these constants.
    static constexpr double kappa2 = 0.5, kappa4 = 0.02, c4 = 2.0;
};

class AdvectionRoe : public AdvectionBase {
public:
    using AdvectionBase::AdvectionBase;
    Scheme scheme() const override { return Scheme::Roe; }
    static constexpr double entropyFixCoefficient = 0.01;  // include/advection_roe.hpp:63
};

// BoundaryBase family (include/boundary_*.hpp): one object per patch.
class BoundaryBase {
public:
    virtual ~BoundaryBase() = default;
    virtual DevPatch toDevice() const = 0;
};

class BoundaryInlet : public BoundaryBase {
public:
    explicit BoundaryInlet(const std::vector<double>& values) : values_(values) {
        if (values_.size() < 5) throw ConfigError("inlet needs total pressure, total temperature and a 3-component direction");
    }
    DevPatch toDevice() const override {
        DevPatch p{kBcInlet, -1, {}};
        for (int i = 0; i < 5; i++) p.v[i] = values_[i];
        return p;
    }

private:
    std::vector<double> values_;
};

class BoundaryOutlet : public BoundaryBase {
public:
    explicit BoundaryOutlet(double p) : p_(p) {}
    DevPatch toDevice() const override { return DevPatch{kBcOutlet, -1, {p_}}; }

private:
    double p_;
};

// BoundaryOutletThrottle / BoundaryOutletRadialEquilibrium read a per-j
// pressure profile updated every iteration (src/solver.cpp:2688-2787).
class BoundaryOutletProfile : public BoundaryBase {
public:
    BoundaryOutletProfile(int type, int profile) : type_(type), profile_(profile) {}
    DevPatch toDevice() const override { return DevPatch{type_, profile_, {}}; }

private:
    int type_, profile_;
};

// BoundaryInletSupersonic (fixed p, T, velocity) and BoundaryFarfield
// (Mach, p, T, direction): the patch values, at least `need` of them.
class BoundaryWithValues : public BoundaryBase {
public:
    BoundaryWithValues(int type, const std::vector<double>& values, size_t need, const char* what)
        : type_(type), values_(values) {
        if (values_.size() < need) throw ConfigError(what);
    }
    DevPatch toDevice() const override {
        DevPatch p{type_, -1, {}};
        for (size_t i = 0; i < values_.size() && i < 8; i++) p.v[i] = values_[i];
        return p;
    }

private:
    int type_;
    std::vector<double> values_;
};

class BoundaryInviscidWall : public BoundaryBase {
public:
    DevPatch toDevice() const override { return DevPatch{kBcInviscidWall, -1, {}}; }
};

// Periodic and wedge faces carry no flux (src/boundary_fake.cpp:4-13).
class BoundaryFake : public BoundaryBase {
public:
    explicit BoundaryFake(int type) : type_(type) {}
    DevPatch toDevice() const override { return DevPatch{type_, -1, {}}; }

private:
    int type_;
};

// SourceBFMBase family (include/source_bfm_*.hpp).
class SourceBFMBase {
public:
    explicit SourceBFMBase(const Config& config)
        : blockage_(config.isBlockageActive()),
          stalled_(config.isStalledBfmActive()),
          perturb_(config.isPerturbationBodyForceActive()) {}
    virtual ~SourceBFMBase() = default;
    virtual BfmModel model() const { return BfmModel::None; }
    virtual void configure(DevCase& c) const {
        c.bfm_model = static_cast<int>(model());
        c.blockage = blockage_ ? 1 : 0;
        c.stalled = stalled_ ? 1 : 0;
        c.perturb = perturb_ ? 1 : 0;
    }

protected:
    bool blockage_, stalled_, perturb_;
};

class SourceBFMHall : public SourceBFMBase {
public:
    using SourceBFMBase::SourceBFMBase;
    BfmModel model() const override { return BfmModel::Hall; }
};

class SourceBFMThollet : public SourceBFMBase {
public:
    explicit SourceBFMThollet(const Config& config)
        : SourceBFMBase(config),
          kn_(config.parseFloat("HALL_THOLLET_COEFFICIENT_KN")),
          kf_(config.parseFloat("HALL_THOLLET_COEFFICIENT_KF")),
          kd_(config.parseFloat("HALL_THOLLET_COEFFICIENT_KD")),
          offDesign_(config.getHallTholletOffDesignActive()) {
        if (!config.has("FLUID_KINEMATIC_VISCOSITY"))
            throw ConfigError("Hall-Thollet needs FLUID_KINEMATIC_VISCOSITY in this library");
        nu_ = config.parseFloat("FLUID_KINEMATIC_VISCOSITY");
    }
    BfmModel model() const override { return BfmModel::HallThollet; }
    void configure(DevCase& c) const override {
        SourceBFMBase::configure(c);
        c.kn = kn_;
        c.kf = kf_;
        c.kd = kd_;
        c.nu = nu_;
        c.offdesign = offDesign_ ? 1 : 0;
    }

private:
    double kn_, kf_, kd_, nu_ = 0;
    bool offDesign_;
};

class SourceBFMLiftDrag : public SourceBFMBase {
public:
    explicit SourceBFMLiftDrag(const Config& config)
        : SourceBFMBase(config),
          le_(static_cast<int>(config.parseFloat("LEADING_EDGE_INDEX"))),
          te_(static_cast<int>(config.parseFloat("TRAILING_EDGE_INDEX"))) {}
    BfmModel model() const override { return BfmModel::LiftDrag; }
    void configure(DevCase& c) const override {
        SourceBFMBase::configure(c);
        c.le_idx = le_;
        c.te_idx = te_;
    }

private:
    int le_, te_;
};

// SourceBFMChima (src/source_bfm_chima.cpp:3-13): leading / trailing edge
// indices and the scaling functions of turning and loss over the mass flow,
// read from CHIMA_SCALING_FUNCTIONS_FILEPATH (a CSV table with the columns
// MassFlow, PhiTurn, PhiLoss; InputTable, src/input_table.cpp:8-55).
class SourceBFMChima : public SourceBFMBase {
public:
    explicit SourceBFMChima(const Config& config);
    BfmModel model() const override { return BfmModel::Chima; }
    void configure(DevCase& c) const override {
        SourceBFMBase::configure(c);
        c.le_idx = le_;
        c.te_idx = te_;
    }
    const std::vector<double>& massFlow() const { return mf_; }
    const std::vector<double>& turning() const { return turn_; }
    const std::vector<double>& loss() const { return loss_; }

private:
    int le_, te_;
    std::vector<double> mf_, turn_, loss_;
};

// SourceBFMCorrelations (src/source_bfm_correlations.cpp:3-10,
// include/config.hpp:345): leading / trailing edge indices and KN.
class SourceBFMCorrelations : public SourceBFMBase {
public:
    explicit SourceBFMCorrelations(const Config& config)
        : SourceBFMBase(config),
          le_(static_cast<int>(config.parseFloat("LEADING_EDGE_INDEX"))),
          te_(static_cast<int>(config.parseFloat("TRAILING_EDGE_INDEX"))) {}
    BfmModel model() const override { return BfmModel::Correlations; }
    void configure(DevCase& c) const override {
        SourceBFMBase::configure(c);
        c.le_idx = le_;
        c.te_idx = te_;
    }

private:
    int le_, te_;
};

}  // namespace ctbfm
