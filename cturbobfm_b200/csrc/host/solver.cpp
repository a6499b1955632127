// Solver: see solver.hpp.
#include "solver.hpp"

#include "host_fluid.hpp"
#include "output.hpp"
#include "restart.hpp"

#include <algorithm>
#include <atomic>
#include <cctype>
#include <cmath>
#include <cstring>
#include <fstream>
#include <sstream>

namespace ctbfm {

namespace {


int boundaryTypeFromString(std::string s) {  // include/types.hpp:202-232, path subset
    std::transform(s.begin(), s.end(), s.begin(), [](unsigned char ch) { return std::tolower(ch); });
    if (s == "inlet") return kBcInlet;
    if (s == "outlet") return kBcOutlet;
    if (s == "radial_equilibrium") return kBcRadialEq;
    if (s == "inviscid_wall") return kBcInviscidWall;
    if (s == "wedge") return kBcWedge;
    if (s == "periodic") return kBcPeriodic;
    if (s == "throttle") return kBcThrottle;
    if (s == "empty") return kBcEmpty;
    if (s == "inlet_supersonic") return kBcInletSupersonic;
    if (s == "outlet_supersonic") return kBcOutletSupersonic;
    if (s == "mass_flow" || s == "outlet_mass_flow" || s == "massflow" || s == "mass_flow_rate") return kBcMassFlow;
    if (s == "transparent") return kBcTransparent;
    if (s == "farfield") return kBcFarfield;
    // the reference never assigns the 2-D inlet file's path (Solver::_inlet2DfilePath
    // stays empty, include/solver.hpp:345), so its inlet_2d cannot run
    if (s == "inlet_2d")
        throw ConfigError("BoundaryType inlet_2d: the reference reads its 2-D inlet file from an empty path; not supported");
    if (s == "no_slip_wall") return kBcNoSlipWall;
    throw ConfigError("Unknown BoundaryType: " + s);
}

// Host copies of the FluidIdeal functions used at set-up (src/fluid_ideal.cpp).
struct HostGas {
    double g, R;
    double staticEnergy(const Vec3& u, double et) const {
        const double m = u.magnitude();
        const double m2 = m * m;
        return et - 0.5 * m2;
    }
    double pressure(double rho, const Vec3& u, double et) const { return (g - 1) * rho * staticEnergy(u, et); }
    double temperature(double rho, const Vec3& u, double et) const { return pressure(rho, u, et) / (rho * R); }
};

}  // namespace

// The input-field names a CSV table may carry (FieldNameMapper,
// include/types.hpp:1083-1127); an unknown name is an error.
static bool knownFieldName(const std::string& n) {
    static const char* names[] = {
        "x", "y", "z", "rho", "rho_u", "rho_v", "rho_w", "rho_e", "blockage", "normalAxial", "normalRadial",
        "normalTangential", "rpm", "streamwiseLength", "bladePresent", "numberBlades", "spanwiseLength", "Dht_Dm",
        "Ds_Dm", "MassFlow", "PhiTurn", "PhiLoss", "PhiDev", "bladeMetalAngle", "bladeGasPathAngle", "bladeLeanAngle",
        "bladeCamberCurvature", "Pt", "Tt", "nx", "ny", "nz", "dbladeMetalAngle_dm", "deviationAnglePivot",
        "deltaAngularMomentum", "deltaEntropy", "deltaFlowAngle", "deviationAngleStall", "liftDragBeta0",
        "liftDragBetaEtamax", "liftDragKpEtamax"};
    for (const char* k : names)
        if (n == k) return true;
    return false;
}

SourceBFMChima::SourceBFMChima(const Config& config) : SourceBFMBase(config), le_(0), te_(0) {
    // InputTable::readCsvFile (src/input_table.cpp:14-55): a header line of
    // field names, then rows of values, column by column
    if (!config.has("CHIMA_SCALING_FUNCTIONS_FILEPATH"))
        throw ConfigError("Not found value for key \"CHIMA_SCALING_FUNCTIONS_FILEPATH\" in configuration.");
    std::string path = config.get("CHIMA_SCALING_FUNCTIONS_FILEPATH");
    if (!path.empty() && path[0] != '/' && !config.directory().empty()) path = config.directory() + "/" + path;
    std::ifstream f(path);
    if (!f) throw ConfigError("Error opening file: " + path);
    std::string line;
    std::vector<std::string> head;
    if (std::getline(f, line)) {
        std::stringstream hs(line);
        std::string col;
        while (std::getline(hs, col, ',')) {
            if (!knownFieldName(col)) throw ConfigError("Unknown field name: " + col);
            head.push_back(col);
        }
    }
    std::vector<std::vector<double>> cols(head.size());
    while (std::getline(f, line)) {
        std::stringstream ss(line);
        std::string tok;
        size_t idx = 0;
        while (std::getline(ss, tok, ',') && idx < head.size()) {
            try {
                cols[idx].push_back(std::stod(tok));
            } catch (const std::exception&) {
            }
            ++idx;
        }
    }
    auto column = [&](const char* name) -> const std::vector<double>& {
        for (size_t q = 0; q < head.size(); q++)
            if (head[q] == name) return cols[q];
        throw ConfigError(std::string("Chima scaling functions file ") + path + " has no " + name + " column");
    };
    mf_ = column("MassFlow");
    turn_ = column("PhiTurn");
    loss_ = column("PhiLoss");
    if (mf_.empty() || turn_.size() != mf_.size() || loss_.size() != mf_.size())
        throw ConfigError("Chima scaling functions file " + path + " needs equally long MassFlow, PhiTurn, PhiLoss columns");
    // the table member is initialised before the edge indices (include/source_bfm_chima.hpp:48-52)
    le_ = static_cast<int>(config.parseFloat("LEADING_EDGE_INDEX"));
    te_ = static_cast<int>(config.parseFloat("TRAILING_EDGE_INDEX"));
}

Solver::Solver(Config& config, Mesh& mesh, const std::vector<PatchRow>* patches)
    : config_(config), mesh_(mesh), topo_(config.getTopology()) {
    // Config::getFluidModel (src/config.cpp:468-481)
    const std::string fluid = config.has("FLUID_MODEL") ? config.get("FLUID_MODEL") : "None";
    if (fluid == "real" || fluid == "Real" || fluid == "REAL") {
        if (config.parseBool("STOP_ON_TABLE_OUT_OF_BOUNDS", false))
            throw ConfigError("STOP_ON_TABLE_OUT_OF_BOUNDS is outside this library's scope");
        if (config.parseBool("FLUID_TABLE_FORCE_REGENERATE", false))
            throw ConfigError("Regenerating the fluid table is outside this library's scope (pass a .lut file)");
        // Solver::buildFluidModel (src/solver.cpp:48-74) with an existing table
        table_ = std::make_unique<FluidTable>(fluidTablePath(config));
    } else if (fluid != "None" && fluid != "Ideal" && fluid != "ideal" && fluid != "IDEAL") {
        throw ConfigError("Invalid value for key \"FLUID_MODEL\" in configuration.");
    }
    if (config.isViscosityActive()) setupTransport();
    if (config.isAccelerationActive() && config.getTimeStepMethod() != TimeStepMethod::Fixed)
        throw ConfigError("Rotational speed scaling factor is only active for fixed time step method");
    // GPU_PRECISION (this library's key; the reference ignores unknown keys)
    const std::string prec = config.has("GPU_PRECISION") ? config.get("GPU_PRECISION") : "fp64";
    if (prec == "fp64") prec_ = kFP64;
    else if (prec == "fp32_kahan") prec_ = kFP32Kahan;
    else throw ConfigError("Invalid value for key \"GPU_PRECISION\" (fp64 or fp32_kahan)");
    // GPU_STAGE_FUSION (this library's key): the fused stage kernel
    // ("fused"), the split stage kernels ("split") or the faster of the two
    // as the autotuner measures them ("auto", the default); FP64 results are
    // the same either way
    // ("fused"), the split stage kernels ("split"), the persistent iteration
    // kernel ("persistent": one cooperative launch per 32 iterations, for
    // ideal-gas inviscid cases without the SA model) or the fastest of them
    // as the autotuner measures them ("auto")
    const std::string fusion = config.has("GPU_STAGE_FUSION") ? config.get("GPU_STAGE_FUSION") : "auto";
    if (fusion == "fused") fusion_ = 1;
    else if (fusion == "split") fusion_ = 0;
    else if (fusion == "auto") fusion_ = 2;
    else if (fusion == "persistent") fusion_ = 3;
    else throw ConfigError("Invalid value for key \"GPU_STAGE_FUSION\" (auto, fused, split or persistent)");
    if (fusion_ == 3 && (table_ || config.isViscosityActive() || config.parseBool("TURBULENCE_ACTIVE", false)))
        throw ConfigError("GPU_STAGE_FUSION = persistent runs ideal-gas inviscid cases without a turbulence model");
    coeffs_ = config.getTimeIntegrationCoeffs();
    maxIter_ = config.getMaxIterations();
    // every setting and input file is validated before the first CUDA call,
    // so that input errors are reported as such on any machine
    setupModels();
    readBoundaries(patches);
    buildBoundaryStructures();
    buildWallMask();
    validateSettings();
    setupScalars();
    setupTurbulence();  // after setupScalars: needs the gas constant
    cudaCheck(cudaGetDevice(&device_), "cudaGetDevice");
    cudaCheck(cudaStreamCreateWithFlags(&ownStream_, cudaStreamNonBlocking), "cudaStreamCreate");
    stream_ = ownStream_;
    // back the static scratch of computeResidualNoAlloc on this device now
    // (under lazy module loading the driver reserves it at the first address
    // look-up), so that the no-allocation entry point never reserves memory
    {
        double* scratch = nullptr;
        size_t bytes = 0;
        cudaCheck(noallocScratch(device_, &scratch, &bytes), "static scratch set-up (cudaGetSymbolAddress)");
    }
    hostCtl_ = static_cast<Control*>(pinnedAlloc(sizeof(Control)));
    std::memset(hostCtl_, 0, sizeof(Control));
    // the device arrays of a solve come from one slab when its size is
    // known: the bytes per node of the last solve of this precision, with
    // slack (a further slab when they do not fit)
    static std::atomic<double> perNode[2] = {{0.0}, {0.0}};
    const double nodesD = static_cast<double>(mesh_.nodes());
    auto reserveLike = [&](auto& inst, int p) {
        const double b = perNode[p].load();
        if (b > 0) inst.reserve(static_cast<size_t>(b * nodesD * 1.1) + (size_t(1) << 16));
    };
    auto learn = [&](const auto& inst, int p) { perNode[p].store(static_cast<double>(inst.usedBytes()) / nodesD); };
    if (prec_ == kFP32Kahan) {
        i32_ = std::make_unique<InstanceT<float>>();
        reserveLike(*i32_, 1);
        uploadArrays(*i32_);
        learn(*i32_, 1);
        g32_ = std::make_unique<GroupT<float>>(std::vector<InstanceT<float>*>{i32_.get()});
        g32_->setFusedMode(fusion_);
        initializeState(*i32_, *g32_);
    } else {
        i64_ = std::make_unique<InstanceT<double>>();
        reserveLike(*i64_, 0);
        uploadArrays(*i64_);
        learn(*i64_, 0);
        g64_ = std::make_unique<GroupT<double>>(std::vector<InstanceT<double>*>{i64_.get()});
        g64_->setFusedMode(fusion_);
        initializeState(*i64_, *g64_);
    }
    // host-to-device copies from pageable memory may still be in flight when
    // cudaMemcpy returns; the solver's kernels run on a non-blocking stream.
    // Only the legacy default stream (the copies) and the solver's own stream
    // are waited for, so a solver can be built while other solvers' batches
    // run on the device (continuous batching).
    cudaCheck(cudaStreamSynchronize(cudaStreamLegacy), "cudaStreamSynchronize");
    cudaCheck(cudaStreamSynchronize(stream_), "cudaStreamSynchronize");
}

// Solver::buildAdvectionModel / buildBfmInfo (src/solver.cpp:185-198, 701-749).
void Solver::setupModels() {
    if (config_.getAdvectionScheme() == Scheme::JST) advection_ = std::make_unique<AdvectionJst>(config_);
    else advection_ = std::make_unique<AdvectionRoe>(config_);
    switch (config_.getBFMModel()) {
        case BfmModel::Hall: bfm_ = std::make_unique<SourceBFMHall>(config_); break;
        case BfmModel::HallThollet: bfm_ = std::make_unique<SourceBFMThollet>(config_); break;
        case BfmModel::LiftDrag: bfm_ = std::make_unique<SourceBFMLiftDrag>(config_); break;
        case BfmModel::Chima: bfm_ = std::make_unique<SourceBFMChima>(config_); break;
        case BfmModel::Correlations: bfm_ = std::make_unique<SourceBFMCorrelations>(config_); break;
        default: bfm_ = std::make_unique<SourceBFMBase>(config_); break;
    }
}

// setTransportProperties of FluidIdeal (src/fluid_ideal.cpp:209-222) and
// FluidReal (src/fluid_real.cpp:378-385), called when the fluid is built
// (src/solver.cpp:72-74), with Config::getViscosityModel and getFluidMuConstant
// (src/config.cpp:575-598). FluidReal's viscosity stays at its 2.0e-5 default
// (include/fluid_real.hpp:168-171) unless the model is constant.
void Solver::setupTransport() {
    DevCaseT<double>& c = proto_;
    c.viscous = 1;
    const std::string raw = config_.has("FLUID_VISCOSITY_MODEL") ? config_.get("FLUID_VISCOSITY_MODEL") : "None";
    bool constant;
    if (raw == "None") {
        constant = config_.has("FLUID_MU_CONSTANT") || config_.has("FLUID_CONSTANT_MU");
    } else {
        std::string key = raw;
        std::transform(key.begin(), key.end(), key.begin(), [](unsigned char ch) { return std::tolower(ch); });
        if (key == "sutherland") constant = false;
        else if (key == "constant") constant = true;
        else throw ConfigError("Unknown ViscosityModel: " + raw + ". Supported options: Sutherland, Constant.");
    }
    auto muConstant = [&]() {
        if (config_.has("FLUID_MU_CONSTANT")) return config_.parseFloat("FLUID_MU_CONSTANT");
        if (config_.has("FLUID_CONSTANT_MU")) return config_.parseFloat("FLUID_CONSTANT_MU");
        if (config_.has("FLUID_SUTHERLAND_MU_REF")) return config_.parseFloat("FLUID_SUTHERLAND_MU_REF");
        throw ConfigError("Missing constant viscosity value: please specify \"FLUID_MU_CONSTANT\" in configuration.");
    };
    c.visc_const = 1;
    if (constant) {
        c.mu_const = muConstant();
    } else if (table_) {
        c.mu_const = 2.0e-5;
    } else {
        c.visc_const = 0;
        c.suth_mu = config_.parseFloat("FLUID_SUTHERLAND_MU_REF");
        c.suth_T = config_.parseFloat("FLUID_SUTHERLAND_T_REF");
        c.suth_S = config_.parseFloat("FLUID_SUTHERLAND_S");
    }
    c.vcp = config_.parseFloat("FLUID_CP");
    c.vpr = config_.parseFloat("FLUID_PRANDTL_NUMBER");
}

// reconstructNuTildeFromEddyViscosity (src/math_utils.cpp:641-675): nu hat
// whose fv1 nu hat rho is mu_t (Newton on chi^4 - y chi^3 - cv1^3 y).
static double nuTildeOfEddyViscosity(double mu_t, double mu_L, double rho, double cv1) {
    if (mu_t <= 0.0 || mu_L <= 0.0 || rho <= 0.0) return 0.0;
    const double nu = mu_L / rho;
    const double y = mu_t / mu_L;
    const double cv1_3 = cv1 * cv1 * cv1;
    const double cv1_3_y = cv1_3 * y;
    double chi = std::max(y, std::pow(cv1_3_y, 0.25));
    for (int iter = 0; iter < 12; ++iter) {
        const double chi2 = chi * chi;
        const double chi3 = chi2 * chi;
        const double chi4 = chi3 * chi;
        const double f = chi4 - y * chi3 - cv1_3_y;
        const double df = 4.0 * chi3 - 3.0 * y * chi2;
        if (std::abs(df) < 1e-14) break;
        const double delta = f / df;
        chi -= delta;
        if (std::abs(delta) < 1e-10 * (1.0 + chi)) break;
    }
    return std::max(0.0, chi * nu);
}

// Config::isTurbulenceActive / getTurbulenceModel (src/config.cpp:165-207);
// TurbulenceModelSA::setupInitialValues / initializeFromZero
// (src/turbulence_model_sa.cpp:32-71); Solver::computeWallDistance /
// computeMinimumDistanceToBoundary (src/solver.cpp:657-698): the least
// distance of each node to a node of a no-slip wall patch; the boundary rows
// of updateBoundaryValues (src/turbulence_model_sa.cpp:250-345) in the
// boundary file's order. The model runs with VISCOSITY_ACTIVE, the ideal gas
// and a start from the initial field (a restarted turbulence field is outside
// this library's scope).
void Solver::setupTurbulence() {
    DevCaseT<double>& c = proto_;
    c.sa = 0;
    if (!config_.parseBool("TURBULENCE_ACTIVE", false)) return;
    if (!config_.has("TURBULENCE_MODEL"))
        throw ConfigError("Not found value for key \"TURBULENCE_MODEL\" in configuration.");
    const std::string model = config_.get("TURBULENCE_MODEL");
    if (model == "None") return;
    if (model != "SA") throw ConfigError("Invalid value for key \"TURBULENCE_MODEL\" in configuration.");
    if (!c.viscous) throw ConfigError("TURBULENCE_MODEL = SA needs VISCOSITY_ACTIVE in this library");
    if (table_) throw ConfigError("the Spalart-Allmaras model with FLUID_MODEL = real is outside this library's scope");
    if (config_.parseBool("RESTART_SOLUTION", false))
        throw ConfigError("a restarted Spalart-Allmaras field is outside this library's scope");
    c.sa = 1;
    c.sa_prt = config_.has("TURBULENT_PRANDTL_NUMBER") ? config_.parseFloat("TURBULENT_PRANDTL_NUMBER") : 0.86;
    c.sa_relax = config_.has("IMPLICIT_UNDER_RELAXATION") ? config_.parseFloat("IMPLICIT_UNDER_RELAXATION") : 1.0;
    const double T = config_.getInitTemperature(), p = config_.getInitPressure();
    const double rho = p / (c.rgas * T);
    const double mu = c.visc_const ? c.mu_const
                                   : c.suth_mu * std::pow(T / c.suth_T, 1.5) * ((c.suth_T + c.suth_S) / (T + c.suth_S));
    c.sa_init_nu = mu / rho;
    if (config_.has("TURBULENCE_NU_TILDE_RATIO")) c.sa_ff = config_.parseFloat("TURBULENCE_NU_TILDE_RATIO");
    else if (config_.has("TURBULENCE_EDDY_VISCOSITY_RATIO"))
        c.sa_ff = nuTildeOfEddyViscosity(config_.parseFloat("TURBULENCE_EDDY_VISCOSITY_RATIO"), 1.0, 1.0, 7.1);
    else c.sa_ff = 3.0;
    const double initScale =
        config_.has("TURBULENCE_INIT_NU_TILDE_RATIO") ? config_.parseFloat("TURBULENCE_INIT_NU_TILDE_RATIO") : c.sa_ff;
    saInitNuHat_ = initScale * c.sa_init_nu;
    const long NI = mesh_.ni(), NJ = mesh_.nj(), NK = mesh_.nk(), N = mesh_.nodes();
    // node range and donor step of a patch (fetchBoundaryNodesIndexRange,
    // src/boundary_base.cpp:227-267; Boundary::computeOrientation,
    // include/boundary_base.hpp:109-119)
    auto range = [&](const auto& b, long r[6], int st[3]) {
        r[0] = b.i_min; r[1] = b.i_max; r[2] = b.j_min; r[3] = b.j_max; r[4] = b.k_min; r[5] = b.k_max;
        if (r[0] == r[1] && r[0] == 0) r[1] = 1;
        else if (r[0] == r[1] && r[0] == NI) { r[0] = NI - 1; r[1] = r[0] + 1; }
        else if (r[2] == r[3] && r[2] == 0) r[3] = 1;
        else if (r[2] == r[3] && r[2] == NJ) { r[2] = NJ - 1; r[3] = r[2] + 1; }
        else if (r[4] == r[5] && r[4] == 0) r[5] = 1;
        else if (r[4] == r[5] && r[4] == NK) { r[4] = NK - 1; r[5] = r[4] + 1; }
        else throw ConfigError("Invalid indexing on boundary condition specs for patch " + b.name);
        st[0] = st[1] = st[2] = 0;
        if (b.i_min == b.i_max) st[0] = b.i_min == 0 ? 1 : -1;
        else if (b.j_min == b.j_max) st[1] = b.j_min == 0 ? 1 : -1;
        else if (b.k_min == b.k_max) st[2] = b.k_min == 0 ? 1 : -1;
    };
    const auto& P = mesh_.vertices();
    saWd_.assign(static_cast<size_t>(N), 1.0E9);
    saBc_.clear();
    for (const auto& b : boundaries_) {
        long r[6];
        int st[3];
        int kind = -1;
        if (b.type == kBcNoSlipWall) kind = 0;
        else if (b.type == kBcInlet || b.type == kBcInletSupersonic || b.type == kBcFarfield) kind = 1;
        else if (b.type == kBcOutlet || b.type == kBcRadialEq || b.type == kBcThrottle || b.type == kBcMassFlow ||
                 b.type == kBcOutletSupersonic || b.type == kBcInviscidWall || b.type == kBcTransparent)
            kind = 2;
        if (kind < 0) continue;
        range(b, r, st);
        saBc_.insert(saBc_.end(), {kind, int(r[0]), int(r[1]), int(r[2]), int(r[3]), int(r[4]), int(r[5]), st[0],
                                   st[1], st[2]});
    }
    c.sa_npatch = static_cast<int>(saBc_.size() / 10);
    for (long q = 0; q < N; q++) {
        double mn = 1.0E9;
        for (const auto& b : boundaries_) {
            if (b.type != kBcNoSlipWall) continue;
            long r[6];
            int st[3];
            range(b, r, st);
            double pm = 1.0E9;
            for (long ib = r[0]; ib < r[1]; ib++)
                for (long jb = r[2]; jb < r[3]; jb++)
                    for (long kb = r[4]; kb < r[5]; kb++) {
                        const auto& a = P[q];
                        const auto& w = P[mesh_.idx(ib, jb, kb)];
                        const double dx = a.x - w.x, dy = a.y - w.y, dz = a.z - w.z;
                        const double dd = std::sqrt(dx * dx + dy * dy + dz * dz);
                        if (dd < pm) pm = dd;
                    }
            if (pm < mn) mn = pm;
        }
        saWd_[q] = mn;
    }
}

// The nodes of every no-slip wall patch (Solver::buildBoundaryFluxes,
// src/solver.cpp:369-388, with fetchBoundaryNodesIndexRange,
// src/boundary_base.cpp:227-267). With viscosity on, the reference reads the
// wall velocity from the patch's first three values at every iteration
// (src/solver.cpp:3189-3203), so they must be there; walls at rest only.
void Solver::buildWallMask() {
    const long NI = mesh_.ni(), NJ = mesh_.nj(), NK = mesh_.nk();
    wall_.clear();
    for (const auto& b : boundaries_) {
        if (b.type != kBcNoSlipWall) continue;
        long i0 = b.i_min, i1 = b.i_max, j0 = b.j_min, j1 = b.j_max, k0 = b.k_min, k1 = b.k_max;
        if (i0 == i1 && i0 == 0) i1 = 1;
        else if (i0 == i1 && i0 == NI) { i0 = NI - 1; i1 = i0 + 1; }
        else if (j0 == j1 && j0 == 0) j1 = 1;
        else if (j0 == j1 && j0 == NJ) { j0 = NJ - 1; j1 = j0 + 1; }
        else if (k0 == k1 && k0 == 0) k1 = 1;
        else if (k0 == k1 && k0 == NK) { k0 = NK - 1; k1 = k0 + 1; }
        else throw ConfigError("Invalid indexing on boundary condition specs for patch " + b.name);
        if (!proto_.viscous) continue;
        if (b.values.size() < 3)
            throw ConfigError("no_slip_wall patch " + b.name + " needs the wall velocity (3 values) when VISCOSITY_ACTIVE");
        if (b.values[0] != 0.0 || b.values[1] != 0.0 || b.values[2] != 0.0)
            throw ConfigError("no_slip_wall patch " + b.name + ": moving walls are outside this library's scope");
        if (wall_.empty()) wall_.assign(static_cast<size_t>(mesh_.nodes()), 0);
        for (long i = std::max(i0, 0L); i < std::min(i1, NI); i++)
            for (long j = std::max(j0, 0L); j < std::min(j1, NJ); j++)
                for (long k = std::max(k0, 0L); k < std::min(k1, NK); k++) wall_[static_cast<size_t>(mesh_.idx(i, j, k))] = 1;
    }
    if (proto_.viscous && wall_.empty()) wall_.assign(static_cast<size_t>(mesh_.nodes()), 0);
}

// Solver::readBoundaryFile (src/solver.cpp:232-294).
void Solver::readBoundaries(const std::vector<PatchRow>* patches) {
    if (patches) {
        for (const PatchRow& row : *patches) addBoundary(row);
    } else {
        std::string path = config_.boundaryConditionsFilePath();
        if (!path.empty() && path[0] != '/') path = config_.directory() + "/" + path;
        std::ifstream file(path);
        if (!file.is_open()) throw ConfigError("Cannot open file: " + path);
        std::string line;
        bool inData = false;
        while (std::getline(file, line)) {
            if (!line.empty() && line.back() == '\r') line.pop_back();
            if (line.empty()) continue;
            if (line.find('=') != std::string::npos) continue;
            if (line.find("PATCH_NAME") != std::string::npos) {
                inData = true;
                continue;
            }
            if (!inData) continue;
            std::stringstream ss(line);
            std::string tok;
            PatchRow row;
            std::getline(ss, tok, ',');
            tok.erase(std::remove(tok.begin(), tok.end(), ' '), tok.end());
            row.name = tok;
            for (int q = 0; q < 6; q++) {
                if (!std::getline(ss, tok, ',')) throw ConfigError("bad boundary row for " + row.name);
                tok.erase(std::remove(tok.begin(), tok.end(), ' '), tok.end());
                row.range[q] = std::stoi(tok);
            }
            addBoundary(row);
        }
    }
    if (boundaries_.size() > static_cast<size_t>(kMaxPatches))
        throw ConfigError("more than 16 boundary patches");
}

// One patch: its index range, and its type and values from the setting of
// the same name (src/solver.cpp:296-345 via Config::getBoundaryInfo).
void Solver::addBoundary(const PatchRow& row) {
    BoundaryPatch p;
    p.name = row.name;
    if (p.name.empty()) throw ConfigError("a boundary patch needs a name");
    const long* v = row.range;
    p.i_min = v[0]; p.i_max = v[1]; p.j_min = v[2]; p.j_max = v[3]; p.k_min = v[4]; p.k_max = v[5];
    const std::vector<std::string> info = config_.parseList(p.name);
    if (info.empty()) throw ConfigError("Boundary info for " + p.name + " is missing in configuration.");
    p.type = boundaryTypeFromString(info[0]);
    for (size_t q = 1; q < info.size(); q++) {
        try {
            p.values.push_back(std::stod(info[q]));
        } catch (const std::exception&) {
            throw ConfigError("Invalid float format for boundary value \"" + info[q] + "\" in configuration.");
        }
    }
    if (p.i_min == p.i_max) p.orientation = p.i_min == 0 ? 0 : 1;
    else if (p.j_min == p.j_max) p.orientation = p.j_min == 0 ? 2 : 3;
    else p.orientation = p.k_min == 0 ? 4 : 5;
    boundaries_.push_back(std::move(p));
}

// Solver::buildBoundaryDataStructures, buildBoundaryFluxes,
// buildBoundaryConditionsMap, checkBoundaryConditionsMap
// (src/solver.cpp:296-593).
void Solver::buildBoundaryStructures() {
    const long NI = mesh_.ni(), NJ = mesh_.nj(), NK = mesh_.nk();
    std::vector<double> profP, profR;
    int nprof = 0;
    proto_.periodic = 0;
    for (size_t m = 0; m < boundaries_.size(); m++) {
        BoundaryPatch& b = boundaries_[m];
        if (b.type == kBcRadialEq || b.type == kBcThrottle || b.type == kBcMassFlow) {
            // Solver::buildBoundaryDataStructures (src/solver.cpp:296-345): a
            // mass-flow outlet uses radial equilibrium when its 4th value says
            // so (or, without one, in axisymmetric or body-force cases) and the
            // patch is an i-end face; otherwise one pressure for the patch
            bool radial = true;
            if (b.type == kBcMassFlow) {
                const bool canDoRadial = b.i_min == b.i_max && b.i_min != 0 && b.j_max > b.j_min;
                if (b.values.size() >= 4) radial = b.values[3] > 0.5 && canDoRadial;
                else radial = canDoRadial && (topo_ == Topology::Axisymmetric || config_.isBFMActive());
                if (b.values.empty() || b.values[0] <= 0.0)
                    throw ConfigError("Target mass flow for boundary patch " + b.name + " must be specified and positive.");
                if (b.i_min != b.i_max || b.i_min == 0)
                    throw ConfigError("mass-flow outlets on other than the i-end face are outside this library's scope");
            }
            if (b.i_min != b.i_max) throw ConfigError("Radial equilibrium only supported on j-k patches");
            if (b.i_min == 0) throw ConfigError("Radial equilibrium only supported to the last i-position");
            if (b.j_max <= b.j_min) throw ConfigError("Invalid boundary indices for radial equilibrium patch: " + b.name);
            if (b.j_min != 0) throw ConfigError("radial profiles must start at j = 0 (the profile is indexed by the face's j)");
            if (nprof >= kMaxProfiles) throw ConfigError("too many radial profiles");
            const int n = static_cast<int>(b.j_max - b.j_min);
            proto_.prof_off[nprof] = static_cast<int>(profP.size());
            proto_.prof_n[nprof] = n;
            proto_.prof_type[nprof] = b.type;
            proto_.prof_i[nprof] = static_cast<int>(b.i_min > 0 ? b.i_min - 1 : 0);
            proto_.prof_j0[nprof] = static_cast<int>(b.j_min);
            proto_.prof_kt[nprof] = b.type == kBcThrottle ? (b.values.empty() ? 0.0 : b.values[0]) : 0.0;
            proto_.prof_fill[nprof] = radial ? 0 : 1;
            proto_.prof_mf[nprof] = b.type == kBcMassFlow ? b.values[0] : 0.0;
            proto_.prof_plane[nprof] = b.orientation;
            // Config::getMassFlowRelaxation (include/config.hpp:291) or the patch's 3rd value
            double relax = config_.parseFloat("MASS_FLOW_RELAXATION", 0.05);
            if (b.type == kBcMassFlow && b.values.size() >= 3 && b.values[2] > 0.0) relax = b.values[2];
            proto_.prof_relax[nprof] = relax;
            for (long j = b.j_min; j < b.j_max; j++) {
                profR.push_back(mesh_.radius(b.i_max - 1, j, 0));
                profP.push_back(0.0);
            }
            b.flux = std::make_unique<BoundaryOutletProfile>(b.type, nprof);
            nprof++;
        } else if (b.type == kBcPeriodic) {
            if (b.values.size() < 3) throw ConfigError("periodic patch needs id, translation and angle");
            const double id = b.values[0];
            if (id == 0) {
                periodicTransl_ = b.values[1];
                periodicAngleDeg_ = b.values[2];
                if (periodicAngleDeg_ == 360.0) periodicAngleDeg_ = 0.0;
                periodicAngleRad_ = periodicAngleDeg_ * M_PI / 180.0;
                mesh_.checkPeriodicity(periodicTransl_, periodicAngleRad_);
                proto_.periodic = 1;
            }
            if (b.k_min != b.k_max) throw ConfigError("Periodic boundary only supported on i-j patches");
            if (b.i_min != 0 || b.j_min != 0 || b.i_max != NI || b.j_max != NJ)
                throw ConfigError("Periodic boundary only supported on full i-j patches");
            if (b.k_min == 0 && id != 0) throw ConfigError("Periodic boundary with i_min=0 must have boundary id 0");
            b.flux = std::make_unique<BoundaryFake>(kBcPeriodic);
        } else if (b.type == kBcInlet) {
            b.flux = std::make_unique<BoundaryInlet>(b.values);
        } else if (b.type == kBcOutlet) {
            if (b.values.empty()) throw ConfigError("outlet needs a static pressure");
            b.flux = std::make_unique<BoundaryOutlet>(b.values[0]);
        } else if (b.type == kBcInviscidWall) {
            b.flux = std::make_unique<BoundaryInviscidWall>();
        } else if (b.type == kBcInletSupersonic) {
            b.flux = std::make_unique<BoundaryWithValues>(kBcInletSupersonic, b.values, 5,
                                                          "inlet_supersonic needs pressure, temperature and 3 velocity components");
        } else if (b.type == kBcFarfield) {
            b.flux = std::make_unique<BoundaryWithValues>(kBcFarfield, b.values, 6,
                                                          "farfield needs Mach number, pressure, temperature and a 3-component direction");
        } else {
            b.flux = std::make_unique<BoundaryFake>(b.type);
        }
        proto_.patch[m] = b.flux->toDevice();
    }
    proto_.npatches = static_cast<int>(boundaries_.size());
    proto_.nprofiles = nprof;

    std::vector<signed char> mapI(2 * NJ * NK, -1), mapJ(NI * 2 * NK, -1), mapK(NI * NJ * 2, -1);
    for (size_t m = 0; m < boundaries_.size(); m++) {
        const BoundaryPatch& b = boundaries_[m];
        if (b.i_min == b.i_max) {
            const long t = b.i_min == 0 ? 0 : 1;
            for (long j = b.j_min; j < b.j_max; j++)
                for (long k = b.k_min; k < b.k_max; k++) {
                    if (j < 0 || j >= NJ || k < 0 || k >= NK) throw ConfigError("patch " + b.name + " outside the grid");
                    mapI[(t * NJ + j) * NK + k] = static_cast<signed char>(m);
                }
        } else if (b.j_min == b.j_max) {
            const long t = b.j_min == 0 ? 0 : 1;
            for (long i = b.i_min; i < b.i_max; i++)
                for (long k = b.k_min; k < b.k_max; k++) {
                    if (i < 0 || i >= NI || k < 0 || k >= NK) throw ConfigError("patch " + b.name + " outside the grid");
                    mapJ[(i * 2 + t) * NK + k] = static_cast<signed char>(m);
                }
        } else if (b.k_min == b.k_max) {
            const long t = b.k_min == 0 ? 0 : 1;
            for (long i = b.i_min; i < b.i_max; i++)
                for (long j = b.j_min; j < b.j_max; j++) {
                    if (i < 0 || i >= NI || j < 0 || j >= NJ) throw ConfigError("patch " + b.name + " outside the grid");
                    mapK[(i * NJ + j) * 2 + t] = static_cast<signed char>(m);
                }
        } else {
            throw ConfigError("Invalid boundary definition: " + b.name);
        }
    }
    auto missing = [](const std::vector<signed char>& mp, const char* d) {
        for (signed char v : mp)
            if (v < 0) throw ConfigError(std::string("Missing boundary condition on a ") + d + " face");
    };
    missing(mapI, "I");
    missing(mapJ, "J");
    if (topo_ == Topology::ThreeD) missing(mapK, "K");
    // the K map is never read outside 3-D; keep it valid for the kernels
    for (auto& v : mapK)
        if (v < 0) v = 0;
    mapI_ = std::move(mapI);
    mapJ_ = std::move(mapJ);
    mapK_ = std::move(mapK);
    profP_ = std::move(profP);
    profR_ = std::move(profR);

    // turbo performance, throttle and plenum (src/solver.cpp:1309-1321, 735-748)
    needTurbo_ = config_.saveTurboOutput();
    proto_.inlet_pt = 0.0;
    for (const auto& b : boundaries_)
        if (b.type == kBcInlet) {
            proto_.inlet_pt = b.values[0];
            break;
        }
    proto_.throttle_kt = 0.0;
    bool hasThrottle = false;
    for (const auto& b : boundaries_)
        if (b.type == kBcThrottle) {
            hasThrottle = true;
            proto_.throttle_kt = b.values.empty() ? 0.0 : b.values[0];
        }
    proto_.greitzer = config_.enableGreitzerModeling() ? 1 : 0;
    if (proto_.greitzer && !hasThrottle) throw ConfigError("Greitzer modeling enabled but no throttle boundary condition found!");
    if (proto_.greitzer || hasThrottle) needTurbo_ = true;
    for (const auto& b : boundaries_)
        if (b.type == kBcMassFlow) needTurbo_ = true;  // src/solver.cpp:1311-1316
    // the Chima model scales its forces by the current mass flow (src/solver.cpp:1319-1321)
    if (config_.isBFMActive() && config_.getBFMModel() == BfmModel::Chima) needTurbo_ = true;
    // Config::getMassFlowMaxPressureChange (include/config.hpp:293)
    proto_.mf_max_change = config_.parseFloat("MASS_FLOW_MAX_PRESSURE_CHANGE", 0.02);
    if (proto_.greitzer) {
        proto_.plenum_volume = config_.getGreitzerPlenumVolume();
        proto_.ambient_p = config_.getGreitzerAmbientPressure();
    }
    proto_.need_turbo = needTurbo_ ? 1 : 0;
    // TURBO_DIRECTION or the inlet orientation (src/solver.cpp:1654-1680)
    std::string dir = config_.has("TURBO_DIRECTION") ? config_.get("TURBO_DIRECTION") : "i";
    if (!config_.has("TURBO_DIRECTION"))
        for (const auto& b : boundaries_)
            if (b.type == kBcInlet || b.type == kBcInletSupersonic) {
                if (b.orientation == 2) { dir = "j"; break; }
                if (b.orientation == 3) { dir = "-j"; break; }
            }
    proto_.turbo_dir = dir == "-i" ? 1 : ((dir == "j" || dir == "+j") ? 2 : (dir == "-j" ? 3 : 0));
}

// Parses every key the device set-up reads (the reference's getters throw on
// the same inputs).
void Solver::validateSettings() {
    const TimeStepMethod m = config_.getTimeStepMethod();
    config_.getCFL();
    if (m == TimeStepMethod::Fixed) config_.getFixedTimeStep();
    if (!table_) {
        config_.getFluidGamma();
        config_.getFluidGasConstant();
    }
    config_.getInitMachNumber();
    config_.getInitTemperature();
    config_.getInitPressure();
    const std::string raw = config_.has("INIT_DIRECTION") ? config_.get("INIT_DIRECTION") : "";
    if (raw != "adaptive") {
        const auto items = config_.parseList("INIT_DIRECTION");
        if (items.size() != 3) throw ConfigError("INIT_DIRECTION must have 3 components or be 'adaptive'");
        for (const auto& it : items) {
            try {
                (void)std::stod(it);
            } catch (const std::exception&) {
                throw ConfigError("Invalid vector element for key \"INIT_DIRECTION\": \"" + it + "\"");
            }
        }
    }
    config_.getResidualsDropConvergence();
    config_.isSimulationSteady();
    config_.isInletCylindrical();
    config_.getOutletPressureRampMaxIterations();
    config_.getRotationalSpeedScalingFactor();
    if (config_.isAccelerationActive()) {
        config_.parseFloat("ACCELERATION_INITIAL_TIME");
        config_.parseFloat("ACCELERATION_FINAL_TIME");
        config_.parseFloat("ROTATIONAL_SPEED_SCALING_FACTOR_INITIAL");
        config_.parseFloat("ROTATIONAL_SPEED_SCALING_FACTOR_FINAL");
    }
    if (config_.isPerturbationBodyForceActive()) {
        if (config_.parseList("PERTURBATION_CENTER").size() < 3) throw ConfigError("PERTURBATION_CENTER needs 3 values");
        config_.parseFloat("PERTURBATION_RADIAL_EXTENSION");
        config_.parseFloat("PERTURBATION_SCALING_FACTOR");
        config_.parseFloat("PERTURBATION_TIME_START");
        config_.parseFloat("PERTURBATION_TIME_DURATION");
    }
}


Solver::~Solver() {
    if (ownStream_) cudaStreamSynchronize(ownStream_);
    if (stream_ && stream_ != ownStream_) cudaStreamSynchronize(stream_);
    g32_.reset();
    g64_.reset();
    i32_.reset();
    i64_.reset();
    pinnedFree(hostCtl_, sizeof(Control));
    if (ownStream_) cudaStreamDestroy(ownStream_);
}

size_t Solver::deviceBytes() const { return i64_ ? i64_->deviceBytes() : i32_->deviceBytes(); }

// Scalar settings of the device description (both precisions).
void Solver::setupScalars() {
    DevCaseT<double>& c = proto_;
    const long NI = mesh_.ni(), NJ = mesh_.nj(), NK = mesh_.nk(), N = mesh_.nodes();
    c.ni = static_cast<int>(NI);
    c.nj = static_cast<int>(NJ);
    c.nk = static_cast<int>(NK);
    c.n = N;
    c.topo = static_cast<int>(topo_);
    advection_->configure(c);
    c.nstages = static_cast<int>(coeffs_.size());
    for (size_t s = 0; s < coeffs_.size(); s++) c.coeffs[s] = coeffs_[s];
    c.dt_method = static_cast<int>(config_.getTimeStepMethod());
    c.steady = config_.isSimulationSteady() ? 1 : 0;
    c.drop = config_.getResidualsDropConvergence();
    // FluidReal::getGamma / getRconstant (include/fluid_real.hpp:100-101): the
    // table's nominal values
    c.gamma = table_ ? table_->gammaNominal() : config_.getFluidGamma();
    c.rgas = table_ ? table_->gasConstant() : config_.getFluidGasConstant();
    c.cp = (c.gamma * c.rgas) / (c.gamma - 1);
    c.cfl = config_.getCFL();
    c.fixed_dt = c.dt_method == 2 ? config_.getFixedTimeStep() : 0.0;
    c.per_angle_deg = periodicAngleDeg_;
    c.per_cos_p = std::cos(periodicAngleRad_);
    c.per_sin_p = std::sin(periodicAngleRad_);
    c.per_cos_m = std::cos(-periodicAngleRad_);
    c.per_sin_m = std::sin(-periodicAngleRad_);
    c.wedge = mesh_.wedgeAngle();
    c.ramp_iters = config_.getOutletPressureRampMaxIterations();
    c.init_p = config_.getInitPressure();
    c.inlet_cyl = config_.isInletCylindrical() ? 1 : 0;
    c.bfm = config_.isBFMActive() ? 1 : 0;
    bfm_->configure(c);
    c.speed_scale = config_.getRotationalSpeedScalingFactor();
    c.accel = config_.isAccelerationActive() ? 1 : 0;
    if (c.accel) {
        c.acc_t0 = config_.parseFloat("ACCELERATION_INITIAL_TIME");
        c.acc_t1 = config_.parseFloat("ACCELERATION_FINAL_TIME");
        c.acc_s0 = config_.parseFloat("ROTATIONAL_SPEED_SCALING_FACTOR_INITIAL");
        c.acc_s1 = config_.parseFloat("ROTATIONAL_SPEED_SCALING_FACTOR_FINAL");
    }
    if (c.perturb) {
        const auto pc = config_.parseList("PERTURBATION_CENTER");
        if (pc.size() < 3) throw ConfigError("PERTURBATION_CENTER needs 3 values");
        for (int q = 0; q < 3; q++) c.pert_c[q] = std::stod(pc[q]);
        c.pert_r = config_.parseFloat("PERTURBATION_RADIAL_EXTENSION");
        c.pert_s = config_.parseFloat("PERTURBATION_SCALING_FACTOR");
        c.pert_t0 = config_.parseFloat("PERTURBATION_TIME_START");
        c.pert_dur = config_.parseFloat("PERTURBATION_TIME_DURATION");
    }
    if (c.bfm && c.bfm_model == 6)  // Config::getKnCorrelationBfmCoefficient (include/config.hpp:345)
        c.kn = config_.parseFloat("KN_CORRELATION_BFM_COEFFICIENT");
    if (c.bfm && (c.bfm_model == 3 || c.bfm_model == 5 || c.bfm_model == 6)) {
        if (c.le_idx < 0 || c.le_idx >= NI || c.te_idx < 0 || c.te_idx >= NI)
            throw ConfigError("LEADING_EDGE_INDEX / TRAILING_EDGE_INDEX outside the grid");
    }
    c.compensated = prec_ == kFP32Kahan ? 1 : 0;
    c.node_tiles = static_cast<int>((N + kTileSize - 1) / kTileSize);
    c.per_tiles = c.periodic ? static_cast<int>((NI * NJ + kPeriodicTile - 1) / kPeriodicTile) : 0;
    c.hist_cap = std::min<long long>(std::max<long long>(maxIter_, 1024), 1 << 20);
    c.max_it = maxIter_;
    // fused stage kernel: inviscid instances without the Chima / Correlations
    // forces. The box (at most kFusedBoxNodes nodes, one per thread) is
    // chosen to carry the most nodes per round of face evaluations (a block's
    // faces are a pool of 256 per round; the primitives and the node phase
    // weigh in less), counting the nodes the grid's ragged last boxes leave
    // out, with k (the contiguous index) 16 or 32 wide in 3-D, within
    // kFusedFaceCap faces and the shared memory of 3 (Roe) or 2 (JST) blocks
    // per SM in FP64
    c.fuse_ok = (!c.viscous && !bfmRareModel(c)) ? 1 : 0;
    {
        const bool three = c.topo == 1;
        const int fields = c.scheme == 0 ? 7 : 5;
        const size_t smemMax = size_t(c.scheme == 0 ? 104 : 70) << 10;
        double best = -1.0;
        int bb[3] = {1, 1, 1};
        std::vector<int> bks;
        if (three) {
            for (int w : {16, 32}) bks.push_back(std::min(c.nk, w));
        } else {
            bks.push_back(1);
        }
        // An instance whose best boxes would not give every SM a block runs
        // latency-bound when alone: then the boxes that finish one stage in
        // the fewest rounds of face evaluations (waves of 3 blocks per SM of
        // a 148-SM device) are taken, the larger of equals.
        constexpr double kSlots = 148.0 * 3.0;
        for (int pass = 0; pass < 2; pass++) {
            double bestTime = 1e30;
            for (int bk : bks)
                for (int bj = 1; bj <= std::min(c.nj, 64); bj++)
                    for (int bi = 1; bi <= std::min(c.ni, kFusedBoxNodes / (bj * bk)); bi++) {
                        const int nodes = bi * bj * bk;
                        const int faces = (bi + 1) * bj * bk + bi * (bj + 1) * bk + (three ? bi * bj * (bk + 1) : 0);
                        const int nW = nodes + 4 * bj * bk + 4 * bi * bk + (three ? 4 * bi * bj : 0);
                        if (nodes > kFusedBoxNodes || faces > kFusedFaceCap) continue;
                        if ((static_cast<size_t>(fields) * nW + 5 * static_cast<size_t>(faces)) * 8 > smemMax)
                            continue;
                        const double boxes = std::ceil(double(c.ni) / bi) * std::ceil(double(c.nj) / bj) *
                                             std::ceil(double(c.nk) / bk);
                        const double cost = std::ceil(faces / 256.0) + 0.15 * std::ceil(nW / 256.0) + 0.5;
                        const double score = double(c.n) / boxes / cost;
                        const double time = std::ceil(boxes / kSlots) * cost;
                        const bool better = pass == 0 ? score > best + 1e-9
                                                      : (time < bestTime - 1e-9 ||
                                                         (time < bestTime + 1e-9 && score > best + 1e-9));
                        if (better) {
                            best = score;
                            bestTime = time;
                            bb[0] = bi;
                            bb[1] = bj;
                            bb[2] = bk;
                        }
                    }
            const double boxes = std::ceil(double(c.ni) / bb[0]) * std::ceil(double(c.nj) / bb[1]) *
                                 std::ceil(double(c.nk) / bb[2]);
            if (pass == 0 && (best < 0 || boxes >= 148.0)) break;
            if (pass == 0) best = -1.0;
        }
        if (best < 0) c.fuse_ok = 0;
        for (int d = 0; d < 3; d++) c.fbox[d] = bb[d];
    }
    c.fnb[0] = (c.ni + c.fbox[0] - 1) / c.fbox[0];
    c.fnb[1] = (c.nj + c.fbox[1] - 1) / c.fbox[1];
    c.fnb[2] = (c.nk + c.fbox[2] - 1) / c.fbox[2];
    c.nboxes = c.fnb[0] * c.fnb[1] * c.fnb[2];
}

// Device arrays of the operating point in precision R.
template <typename R>
void Solver::uploadArrays(InstanceT<R>& inst) {
    DevCaseT<R>& c = inst.c;
    static_assert(sizeof(DevCaseT<R>) == sizeof(DevCaseT<double>), "same layout for both precisions");
    std::memcpy(static_cast<void*>(&c), &proto_, sizeof(c));  // scalars; every pointer is set below
    const long NI = mesh_.ni(), NJ = mesh_.nj(), NK = mesh_.nk(), N = mesh_.nodes();
    // boundary tables and radial profiles
    auto up8 = [&](const std::vector<signed char>& v) {
        void* d = inst.allocBytes(v.size());
        cudaCheck(cudaMemcpy(d, v.data(), v.size(), cudaMemcpyHostToDevice), "cudaMemcpy");
        return static_cast<const signed char*>(d);
    };
    c.mapI = up8(mapI_);
    c.mapJ = up8(mapJ_);
    c.mapK = up8(mapK_);
    c.prof_p = nullptr;
    c.prof_r = nullptr;
    if (c.nprofiles) {
        c.prof_p = inst.allocD(profP_.size());
        cudaCheck(cudaMemcpy(c.prof_p, profP_.data(), profP_.size() * sizeof(double), cudaMemcpyHostToDevice),
                  "cudaMemcpy");
        c.prof_r = inst.uploadD(profR_);
    }
    // face metrics: unit normal n = S/|S| and |S| (computeAdvectionFluxFromPrimitive)
    for (int d = 0; d < 3; d++) {
        const auto& S = mesh_.surfaces(d);
        std::vector<double> nx(S.size()), ny(S.size()), nz(S.size()), ar(S.size());
        for (size_t f = 0; f < S.size(); f++) {
            const double m = S[f].magnitude();
            nx[f] = S[f].x / m;
            ny[f] = S[f].y / m;
            nz[f] = S[f].z / m;
            ar[f] = m;
        }
        if (c.viscous) {  // raw S and the Green-Gauss weights of the face's left and right node
            std::vector<double> sx(S.size()), sy(S.size()), sz(S.size()), wl(S.size(), 0.0), wr(S.size(), 0.0);
            std::vector<double> dl(c.sa ? S.size() : 0, 0.0), dr(c.sa ? S.size() : 0, 0.0);
            const auto& C = mesh_.centers(d);
            const auto& P = mesh_.vertices();
            const long nfi = NI + (d == 0), nfj = NJ + (d == 1), nfk = NK + (d == 2);
            const long nlast = d == 0 ? NI : (d == 1 ? NJ : NK);
            const long st = d == 0 ? NJ * NK : (d == 1 ? NK : 1);
            for (long fi = 0; fi < nfi; fi++)
                for (long fj = 0; fj < nfj; fj++)
                    for (long fk = 0; fk < nfk; fk++) {
                        const long f = (fi * nfj + fj) * nfk + fk;
                        sx[f] = S[f].x;
                        sy[f] = S[f].y;
                        sz[f] = S[f].z;
                        const long df = d == 0 ? fi : (d == 1 ? fj : fk);
                        if (df == 0 || df == nlast) continue;
                        const long qr = mesh_.idx(fi, fj, fk), ql = qr - st;
                        // computeGradientsGreenGauss4 (src/math_utils.cpp:270-353): w = d0 / (d0 + d1)
                        // with d0 the face centre's distance to the node itself
                        {
                            const double d0 = (C[f] - P[qr]).magnitude(), d1 = (C[f] - P[ql]).magnitude();
                            wr[f] = d0 / (d0 + d1);
                        }
                        {
                            const double d0 = (C[f] - P[ql]).magnitude(), d1 = (C[f] - P[qr]).magnitude();
                            wl[f] = d0 / (d0 + d1);
                        }
                        // interpolateScalar of the SA gradient (src/math_utils.cpp:457-460): the
                        // face centre's distances to the left and the right node
                        if (c.sa) {
                            dl[f] = (C[f] - P[ql]).magnitude();
                            dr[f] = (C[f] - P[qr]).magnitude();
                        }
                    }
            c.sraw[d][0] = inst.uploadR(sx);
            c.sraw[d][1] = inst.uploadR(sy);
            c.sraw[d][2] = inst.uploadR(sz);
            c.gwL[d] = inst.uploadR(wl);
            c.gwR[d] = inst.uploadR(wr);
            if (c.sa) {
                c.sa_dL[d] = inst.uploadR(dl);
                c.sa_dR[d] = inst.uploadR(dr);
            }
            if (d < 2 || topo_ == Topology::ThreeD)
                for (int v = 0; v < 4; v++) c.V[d][v] = inst.allocR(S.size());
        }
        c.f[d].nx = inst.uploadR(nx);
        c.f[d].ny = inst.uploadR(ny);
        c.f[d].nz = inst.uploadR(nz);
        c.f[d].area = inst.uploadR(ar);
        c.f[d].n2x = c.f[d].n2y = nullptr;
        if (c.scheme == 1) {  // AdvectionRoe's normal triad (src/advection_roe.cpp:41-58), second vector
            std::vector<double> n2x(nx.size()), n2y(nx.size());
            for (size_t f = 0; f < nx.size(); f++) {
                double ax = -ny[f], ay = nx[f];
                if (nx[f] == 0.0 && ny[f] == 0.0) {
                    ax = 1.0;
                    ay = 0.0;
                }
                const double m = std::sqrt(ax * ax + ay * ay + 0.0 * 0.0);
                n2x[f] = m == 0.0 ? 0.0 : ax / m;
                n2y[f] = m == 0.0 ? 0.0 : ay / m;
            }
            c.f[d].n2x = inst.uploadR(n2x);
            c.f[d].n2y = inst.uploadR(n2y);
        }
        for (int v = 0; v < 5; v++) c.f[d].c[v] = inst.allocR(S.size());
    }
    // per node: volume, radius, theta rotation, edges of the dual cell
    std::vector<double> cst(N), snt(N), rad(N), aK(N, 0.0);
    std::array<std::vector<double>, 12> edge;
    for (auto& e : edge) e.resize(N);
    const auto& D = mesh_.dualNodes();
    for (long i = 0; i < NI; i++)
        for (long j = 0; j < NJ; j++)
            for (long k = 0; k < NK; k++) {
                const long q = mesh_.idx(i, j, k);
                const double th = mesh_.theta(i, j, k);
                cst[q] = std::cos(th);
                snt[q] = std::sin(th);
                rad[q] = mesh_.radius(i, j, k);
                aK[q] = mesh_.surfaces(2)[mesh_.faceIdx(2, i, j, 0)].magnitude();
                // Mesh::getElementEdges (src/mesh.cpp:559-568)
                const Vec3& p0 = D[mesh_.dualIdx(i, j, k)];
                const Vec3 e3[3] = {D[mesh_.dualIdx(i + 1, j, k)] - p0, D[mesh_.dualIdx(i, j + 1, k)] - p0,
                                    D[mesh_.dualIdx(i, j, k + 1)] - p0};
                for (int d = 0; d < 3; d++) {
                    const double ds = e3[d].magnitude();
                    const Vec3 dir = e3[d] / ds;
                    edge[4 * d + 0][q] = dir.x;
                    edge[4 * d + 1][q] = dir.y;
                    edge[4 * d + 2][q] = dir.z;
                    edge[4 * d + 3][q] = ds;
                }
            }
    c.vol = inst.uploadR(mesh_.volumes());
    c.cost = inst.uploadR(cst);
    c.sint = inst.uploadR(snt);
    c.radius = inst.uploadR(rad);
    c.areaK0 = inst.uploadR(aK);
    c.cost64 = inst.uploadD(cst);
    c.sint64 = inst.uploadD(snt);
    for (int e = 0; e < 12; e++) c.edge[e] = inst.uploadR(edge[e]);
    {
        std::vector<double> vx(N), vy(N), vz(N);
        for (long q = 0; q < N; q++) {
            vx[q] = mesh_.vertices()[q].x;
            vy[q] = mesh_.vertices()[q].y;
            vz[q] = mesh_.vertices()[q].z;
        }
        c.vx = inst.uploadD(vx);
        c.vy = inst.uploadD(vy);
        c.vz = inst.uploadD(vz);
    }
    if (c.viscous) {  // no-slip wall nodes and the node gradients
        void* d = inst.allocBytes(wall_.size());
        cudaCheck(cudaMemcpy(d, wall_.data(), wall_.size(), cudaMemcpyHostToDevice), "cudaMemcpy");
        c.wall = static_cast<const unsigned char*>(d);
        for (int g = 0; g < 12; g++) {
            c.G[g] = inst.allocR(N);
            cudaCheck(cudaMemset(c.G[g], 0, N * sizeof(R)), "cudaMemset");
        }
    }
    if (c.sa) {  // Spalart-Allmaras: nu hat, laminar viscosity (0 until the first solve), work arrays
        c.nuhat = const_cast<R*>(inst.uploadR(std::vector<double>(static_cast<size_t>(N), saInitNuHat_)));
        c.nul = inst.allocR(N);
        cudaCheck(cudaMemset(c.nul, 0, N * sizeof(R)), "cudaMemset");
        c.sa_wd = inst.uploadR(saWd_);
        c.sa_res = inst.allocR(N);
        c.sa_diag = inst.allocR(N);
        c.sa_dstar = inst.allocR(N);
        c.sa_dnu = inst.allocR(N);
        for (int x = 0; x < 3; x++) {
            c.sa_g[x] = inst.allocR(N);
            c.sa_vel[x] = inst.allocR(N);
        }
        void* d = inst.allocBytes(saBc_.size() * sizeof(int));
        cudaCheck(cudaMemcpy(d, saBc_.data(), saBc_.size() * sizeof(int), cudaMemcpyHostToDevice), "cudaMemcpy");
        c.sa_bc = static_cast<const int*>(d);
    }
    // boundary planes (raw surface vectors) for the surface integrals
    for (int b = 0; b < 6; b++) {
        std::vector<double> sx, sy, sz;
        const int dir = b / 2;
        const auto& S = mesh_.surfaces(dir);
        long na = dir == 0 ? NJ : NI, nb = dir == 2 ? NJ : NK;
        for (long a = 0; a < na; a++)
            for (long bb = 0; bb < nb; bb++) {
                long f;
                if (b == 0) f = mesh_.faceIdx(0, 0, a, bb);
                else if (b == 1) f = mesh_.faceIdx(0, NI, a, bb);
                else if (b == 2) f = mesh_.faceIdx(1, a, 0, bb);
                else if (b == 3) f = mesh_.faceIdx(1, a, NJ, bb);
                else if (b == 4) f = mesh_.faceIdx(2, a, bb, 0);
                else f = mesh_.faceIdx(2, a, bb, NK);
                sx.push_back(S[f].x);
                sy.push_back(S[f].y);
                sz.push_back(S[f].z);
            }
        c.bsx[b] = inst.uploadD(sx);
        c.bsy[b] = inst.uploadD(sy);
        c.bsz[b] = inst.uploadD(sz);
    }
    {  // chunks of the eight boundary integrals (k_bint / k_pre)
        auto points = [&](int plane) -> long {
            if (plane <= 1) return NJ * NK;
            if (plane <= 3) return NI * NK;
            return NI * NJ;
        };
        const int td = c.turbo_dir;
        const int turbo[2] = {td == 1 ? 1 : (td == 2 ? 2 : (td == 3 ? 3 : 0)),
                              td == 1 ? 0 : (td == 2 ? 3 : (td == 3 ? 2 : 1))};
        c.bint_off[0] = 0;
        for (int b = 0; b < 8; b++) {
            const long p = points(b < 6 ? b : turbo[b - 6]);
            c.bint_off[b + 1] = c.bint_off[b] + static_cast<int>((p + kBintChunk - 1) / kBintChunk);
        }
        c.bint_part = inst.allocD(static_cast<size_t>(c.bint_off[8]) * 4);
    }
    // BFM fields (include/types.hpp:1036-1078 names)
    c.blk = c.gbx = c.gby = c.gbz = c.nax = c.nrad = c.ntan = c.rpm = c.stwl = c.bpresent = c.nblades = nullptr;
    c.nhat[0] = c.nhat[1] = c.nhat[2] = c.pitch = c.omega0 = nullptr;
    c.cosmetal = c.devpivot = c.devstall = c.ldbeta0 = c.ldkp = c.dangmom = c.dentropy = nullptr;
    c.chima_mf = c.chima_turn = c.chima_loss = nullptr;
    c.metal = nullptr;
    c.chima_n = 0;
    if (c.bfm) {
        auto need = [&](const char* name) { return inst.uploadR(mesh_.field(name)); };
        auto opt = [&](const char* name) -> const R* {
            return mesh_.hasField(name) ? inst.uploadR(mesh_.field(name)) : nullptr;
        };
        c.blk = need("blockage");
        const auto& gb = mesh_.blockageGradient();
        std::vector<double> gx(N), gy(N), gz(N);
        for (long q = 0; q < N; q++) {
            gx[q] = gb[q].x;
            gy[q] = gb[q].y;
            gz[q] = gb[q].z;
        }
        c.gbx = inst.uploadR(gx);
        c.gby = inst.uploadR(gy);
        c.gbz = inst.uploadR(gz);
        c.bpresent = need("bladePresent");
        c.nblades = need("numberBlades");
        if (c.bfm_model != 0 && c.bfm_model != 4) {
            // SourceBFMBase::computeFlowState reads all of these (src/source_bfm_base.cpp:104-149)
            c.nax = need("normalAxial");
            c.nrad = need("normalRadial");
            c.ntan = need("normalTangential");
            c.rpm = need("rpm");
            {  // bfmFlowState's per-node constants, in the device's operation order
                const auto& nx = mesh_.field("normalAxial");
                const auto& ny = mesh_.field("normalRadial");
                const auto& nz = mesh_.field("normalTangential");
                const auto& nbl = mesh_.field("numberBlades");
                const auto& rpm = mesh_.field("rpm");
                std::vector<double> hx(N), hy(N), hz(N), pitch(N), om(N);
                for (long q = 0; q < N; q++) {
                    const double m = std::sqrt(nx[q] * nx[q] + ny[q] * ny[q] + nz[q] * nz[q]);
                    hx[q] = nx[q] / m;
                    hy[q] = ny[q] / m;
                    hz[q] = nz[q] / m;
                    pitch[q] = 2.0 * M_PI * rad[q] / nbl[q];
                    om[q] = rpm[q] * 2.0 * M_PI / 60.0;
                }
                c.nhat[0] = inst.uploadR(hx);
                c.nhat[1] = inst.uploadR(hy);
                c.nhat[2] = inst.uploadR(hz);
                c.pitch = inst.uploadR(pitch);
                c.omega0 = inst.uploadR(om);
            }
            mesh_.field("bladeLeanAngle");
            mesh_.field("bladeGasPathAngle");
            const auto& metal = mesh_.field("bladeMetalAngle");
            std::vector<double> cm(N);
            for (long q = 0; q < N; q++) cm[q] = std::cos(metal[q]);
            c.cosmetal = inst.uploadR(cm);
        } else {
            c.rpm = opt("rpm");
        }
        if (c.bfm_model == 2 || c.bfm_model == 3 || c.bfm_model == 5 || c.bfm_model == 6)
            c.stwl = need("streamwiseLength");
        if (c.bfm_model == 6) {  // SourceBFMCorrelations reads the metal angle and the camber curvature
            c.metal = need("bladeMetalAngle");
            mesh_.field("bladeCamberCurvature");
        }
        if (c.bfm_model == 5) {  // SourceBFMChima::computeInviscid/ViscousComponent
            c.dangmom = need("deltaAngularMomentum");
            c.dentropy = need("deltaEntropy");
            const auto* chima = static_cast<const SourceBFMChima*>(bfm_.get());
            c.chima_n = static_cast<int>(chima->massFlow().size());
            c.chima_mf = inst.uploadD(chima->massFlow());
            c.chima_turn = inst.uploadD(chima->turning());
            c.chima_loss = inst.uploadD(chima->loss());
        }
        if (c.bfm_model == 2 && c.offdesign) c.devpivot = need("deviationAnglePivot");
        if (c.stalled) c.devstall = need("deviationAngleStall");
        if (c.bfm_model == 3) {
            c.ldbeta0 = need("liftDragBeta0");
            c.ldkp = need("liftDragKpEtamax");
        }
        if (topo_ == Topology::ThreeD && !c.rpm) c.rpm = need("rpm");
    }
    // state, stage buffers, reductions, control block, history
    for (int v = 0; v < 5; v++) {
        c.U[v] = inst.allocR(N);
        c.Uc[v] = c.compensated ? inst.allocR(N) : nullptr;
        c.S1[v] = inst.allocR(N);
        c.S2[v] = inst.allocR(N);
        c.Rp[v] = inst.allocR(2 * NI * NJ);
        c.W[v] = inst.allocR(N);
    }
    c.Wp = c.scheme == 0 ? inst.allocR(N) : nullptr;
    c.Wr = c.scheme == 0 ? inst.allocR(N) : nullptr;
    c.dt = inst.allocR(N);
    c.partial = inst.allocD(static_cast<size_t>(c.node_tiles + c.per_tiles) * 5 + c.node_tiles +
                            static_cast<size_t>(c.nboxes) * 5);
    c.lut = table_ ? uploadLut(inst) : nullptr;
    c.ctl = static_cast<Control*>(inst.allocBytes(sizeof(Control)));
    c.hist = inst.allocD(static_cast<size_t>(c.hist_cap) * kHistWidth);
}

// FluidIdeal::computeInitFields (src/fluid_ideal.cpp:155-170),
// Solver::initializeSolutionFromScratch (src/solver.cpp:777-836), and the
// Greitzer initial state and initial radial profiles of
// Solver::initializeSolutionArrays (src/solver.cpp:750-776).
template <typename R>
void Solver::initializeState(InstanceT<R>& inst, GroupT<R>& grp) {
    const double M = config_.getInitMachNumber(), T = config_.getInitTemperature(), p = config_.getInitPressure();
    const double g = proto_.gamma, Rg = proto_.rgas;
    const std::string raw = config_.has("INIT_DIRECTION") ? config_.get("INIT_DIRECTION") : "";
    bool adaptive = raw == "adaptive";
    Vec3 d0;
    if (!adaptive) {
        const auto items = config_.parseList("INIT_DIRECTION");
        if (items.size() != 3) throw ConfigError("INIT_DIRECTION must have 3 components or be 'adaptive'");
        d0 = Vec3(std::stod(items[0]), std::stod(items[1]), std::stod(items[2]));
        if (d0.x == 0.0 && d0.y == 0.0 && d0.z == 0.0) adaptive = true;
    }
    const long NI = mesh_.ni(), NJ = mesh_.nj(), NK = mesh_.nk(), N = mesh_.nodes();
    std::array<std::vector<double>, 5> U;
    for (auto& a : U) a.resize(N);
    const auto& V = mesh_.vertices();
    // Solver::initializeSolutionArrays (src/solver.cpp:783-789)
    const bool restart = config_.parseBool("RESTART_SOLUTION", false);
    if (restart) restartState(config_, mesh_, topo_, proto_.periodic != 0, *hostFluid(), U);
    for (long i = 0; i < NI && !restart; i++)
        for (long j = 0; j < NJ; j++)
            for (long k = 0; k < NK; k++) {
                Vec3 dir = d0;
                if (adaptive) {  // Mesh::computeAdaptiveFlowDirection (src/mesh.cpp:637-661)
                    const long ia = i < NI - 1 ? i : NI - 2;
                    const Vec3 dv = V[mesh_.idx(ia + 1, j, k)] - V[mesh_.idx(ia, j, k)];
                    const double m = dv.magnitude();
                    dir = (m == 0) ? Vec3(0, 0, 0) : dv / m;
                }
                const long q = mesh_.idx(i, j, k);
                if (table_) {  // FluidReal::computeInitFields (src/fluid_real.cpp:346-362)
                    const double rho = table_->density_p_T(p, T);
                    const double e = table_->energy_p_T(p, T);
                    const double a = table_->soundSpeed_rho_e(rho, e);
                    const double dm = dir.magnitude();
                    const Vec3 dn = (dm > 1e-12) ? dir / dm : Vec3(1.0, 0.0, 0.0);
                    const Vec3 u = (dn * a) * M;
                    const double et = e + 0.5 * u.dot(u);
                    U[0][q] = rho;
                    U[1][q] = rho * u.x;
                    U[2][q] = rho * u.y;
                    U[3][q] = rho * u.z;
                    U[4][q] = rho * et;
                    continue;
                }
                const double a = std::sqrt(g * Rg * T);
                const Vec3 u = (dir / dir.magnitude()) * a * M;
                const double rho = p / (Rg * T);
                const double e = p / ((g - 1) * rho);
                const double um = u.magnitude();
                const double et = e + 0.5 * (um * um);
                U[0][q] = rho;
                U[1][q] = rho * u.x;
                U[2][q] = rho * u.y;
                U[3][q] = rho * u.z;
                U[4][q] = rho * et;
            }
    std::memset(hostCtl_, 0, sizeof(Control));
    cudaCheck(cudaMemcpy(inst.c.ctl, hostCtl_, sizeof(Control), cudaMemcpyHostToDevice), "cudaMemcpy");
    const double* in[5] = {U[0].data(), U[1].data(), U[2].data(), U[3].data(), U[4].data()};
    uploadState(in);  // the plenum and the profiles start from the state before the wall preprocessing
    const HostGas gas{g, Rg};
    auto prim = [&](long q, double& rho, Vec3& u, double& et) {
        rho = U[0][q];
        u = Vec3(U[1][q] / U[0][q], U[2][q] / U[0][q], U[3][q] / U[0][q]);
        et = U[4][q] / U[0][q];
    };
    if (proto_.greitzer) {
        double mf[6], tp[4];
        getTurbo(mf, tp);
        double rho, et;
        Vec3 u;
        prim(mesh_.idx(NI - 1, 0, 0), rho, u, et);
        Control ctl = control();
        if (table_) {  // FluidBase::computePressure_primitive / computeTemperature_rho_u_et
            const double e = FluidTable::staticEnergy_u_et(u, et);
            ctl.gz_p = table_->pressure_rho_e(rho, e);
            ctl.gz_T = table_->temperature_rho_e(rho, e);
        } else {
            ctl.gz_p = gas.pressure(rho, u, et);
            ctl.gz_T = gas.temperature(rho, u, et);
        }
        ctl.gz_min = tp[0];
        ctl.gz_mout = tp[0];
        ctl.gz_t = 0.0;
        ctl.has_turbo = 0;
        *hostCtl_ = ctl;
        cudaCheck(cudaMemcpy(inst.c.ctl, hostCtl_, sizeof(Control), cudaMemcpyHostToDevice), "cudaMemcpy");
    }
    if (proto_.nprofiles) {
        // Solver::initializeSolutionArrays (src/solver.cpp:819-834): a mass-flow
        // outlet with a positive 2nd value starts from it, every other profile
        // from the state's static pressure at i_max - 1
        std::vector<const BoundaryPatch*> profPatch;
        for (const auto& b : boundaries_)
            if (b.type == kBcRadialEq || b.type == kBcThrottle || b.type == kBcMassFlow) profPatch.push_back(&b);
        std::vector<double> profP(profP_.size());
        for (int m = 0; m < proto_.nprofiles; m++) {
            const BoundaryPatch& b = *profPatch[static_cast<size_t>(m)];
            if (b.type == kBcMassFlow && b.values.size() >= 2 && b.values[1] > 0.0) {
                for (int jj = 0; jj < proto_.prof_n[m]; jj++) profP[proto_.prof_off[m] + jj] = b.values[1];
                continue;
            }
            for (int jj = 0; jj < proto_.prof_n[m]; jj++) {
                double rho, et;
                Vec3 u;
                prim(mesh_.idx(proto_.prof_i[m], proto_.prof_j0[m] + jj, 0), rho, u, et);
                profP[proto_.prof_off[m] + jj] =
                    table_ ? table_->pressure_rho_e(rho, FluidTable::staticEnergy_u_et(u, et)) : gas.pressure(rho, u, et);
            }
        }
        cudaCheck(cudaMemcpy(inst.c.prof_p, profP.data(), profP.size() * sizeof(double), cudaMemcpyHostToDevice),
                  "cudaMemcpy");
    }
    if (proto_.viscous) setState(in);
    (void)grp;
}

// ------------------------------------------------------------------ running

void Solver::enqueue(long long n) {
    promo_.reset();  // a prepared promotion holds the state before these iterations
    visit([&](auto& inst, auto& grp) { grp.enqueue(n, stream_); (void)inst; });
}

void Solver::autotune() {
    visit([&](auto& inst, auto& grp) {
        (void)inst;
        if (!grp.tuned()) grp.tune(stream_);
    });
    cudaCheck(cudaStreamSynchronize(stream_), "cudaStreamSynchronize");
}

Control Solver::control() {
    visit([&](auto& inst, auto&) {
        cudaCheck(cudaMemcpyAsync(hostCtl_, inst.c.ctl, sizeof(Control), cudaMemcpyDeviceToHost, stream_),
                  "cudaMemcpyAsync");
    });
    cudaCheck(cudaStreamSynchronize(stream_), "cudaStreamSynchronize");
    return *hostCtl_;
}

long long Solver::step(long long n) {
    const Control before = control();
    if (before.status != 0) return 0;
    enqueue(n);
    const Control after = control();
    return after.it - before.it;
}

long long Solver::solve() {
    long long done = 0;
    const long long chunk = 256;
    while (true) {
        const Control c = control();
        if (c.status != 0 || c.it >= maxIter_) break;
        done += step(std::min<long long>(chunk, maxIter_ - c.it));
    }
    return done;
}

namespace {

// One time-step + residual evaluation of U^n with the next iteration's number
// (boundary integrals, time step, profiles, stage -1 into S2).
template <typename R>
void residualSequence(const BatchView<R>& v, cudaStream_t s) {
    cudaCheck(Launcher<R>::boundaryIntegrals(v, false, 1, s), "launch k_bint");
    cudaCheck(Launcher<R>::timeStep(v, 1, s), "launch k_dt");
    cudaCheck(Launcher<R>::pre(v, false, true, true, 1, s), "launch k_pre");
    cudaCheck(Launcher<R>::stage(v, -1, 1, s), "launch stage");
}

// Device array of R -> host doubles, without any allocation: a float array is
// copied into the first half of the output buffer and widened in place from
// the back (double q occupies bytes [8q, 8q+8), the floats still to be read
// lie below byte 4q).
template <typename R>
void copyOut(const R* d, double* h, size_t n, cudaStream_t s) {
    cudaCheck(cudaMemcpyAsync(h, d, n * sizeof(R), cudaMemcpyDeviceToHost, s), "cudaMemcpyAsync");
    cudaCheck(cudaStreamSynchronize(s), "cudaStreamSynchronize");
    if (sizeof(R) != sizeof(double)) {
        const R* f = reinterpret_cast<const R*>(h);
        for (size_t q = n; q-- > 0;) h[q] = static_cast<double>(f[q]);
    }
}

}  // namespace

void Solver::computeResidual(double* dt, double* const r[5]) {
    const long N = mesh_.nodes();
    visit([&](auto& inst, auto& grp) {
        residualSequence(grp.view(), stream_);
        const Control c1 = control();
        if (inst.c.dt_method == 0) copyOut(inst.c.dt, dt, N, stream_);
        else std::fill(dt, dt + N, inst.c.dt_method == 2 ? inst.c.fixed_dt : c1.dt_min);
        for (int v = 0; v < 5; v++) copyOut(inst.c.S2[v], r[v], N, stream_);
    });
}

// The residual evaluation of computeResidual with its per-face flux
// contributions kept in the static scratch array of noalloc.cu; nothing is
// allocated on the device (the caller cannot, or must not, call cudaMalloc).
// Runs on the solver's own device (restoring the caller's current device on
// return) and always points the solver back at its own face buffers, also
// when an error is thrown.
void Solver::computeResidualNoAlloc(double* dt, double* const r[5]) {
    int callerDevice = -1;
    cudaCheck(cudaGetDevice(&callerDevice), "cudaGetDevice");
    if (callerDevice != device_) cudaCheck(cudaSetDevice(device_), "cudaSetDevice");
    struct DeviceGuard {
        int dev, own;
        ~DeviceGuard() {
            if (dev != own) cudaSetDevice(dev);
        }
    } deviceGuard{callerDevice, device_};
    double* scratch = nullptr;
    size_t bytes = 0;
    cudaCheck(noallocScratch(device_, &scratch, &bytes), "static scratch set-up (cudaGetSymbolAddress)");
    const long N = mesh_.nodes();
    visit([&](auto& inst, auto& grp) {
        using R = std::remove_reference_t<decltype(*inst.c.U[0])>;
        const int dirs = inst.c.topo == 1 ? 3 : 2;
        size_t faces = 0;
        for (int d = 0; d < dirs; d++) faces += static_cast<size_t>(mesh_.faceCount(d));
        if (faces * 5 * sizeof(R) > bytes)
            throw ConfigError("ctbfm_compute_residual_noalloc: the case has " + std::to_string(faces) +
                              " faces and needs " + std::to_string(faces * 5 * sizeof(R)) +
                              " bytes of face scratch; the static array holds " + std::to_string(bytes) +
                              " bytes (at most " + std::to_string(bytes / (5 * sizeof(R))) + " faces in " +
                              (sizeof(R) == 8 ? "fp64" : "fp32_kahan") + ")");
        // restores the solver's own face buffers on every exit: a solver left
        // pointing at the shared array would race with other callers' noalloc
        // evaluations and could write past the array in its next step
        struct FaceGuard {
            decltype(inst)& in;
            decltype(grp)& g;
            cudaStream_t st;
            DevFacesT<R> saved[3];
            bool active = false;
            ~FaceGuard() {
                if (!active) return;
                for (int d = 0; d < 3; d++) in.c.f[d] = saved[d];
                try {
                    g.refresh(st);
                } catch (...) {
                }
            }
        } guard{inst, grp, stream_, {inst.c.f[0], inst.c.f[1], inst.c.f[2]}};
        R* base = reinterpret_cast<R*>(scratch);
        size_t off = 0;
        guard.active = true;
        for (int d = 0; d < dirs; d++) {
            const size_t nf = static_cast<size_t>(mesh_.faceCount(d));
            for (int v = 0; v < 5; v++) inst.c.f[d].c[v] = base + off + v * nf;
            off += 5 * nf;
        }
        grp.refresh(stream_);
        // the split stage, whose face kernels write the per-face flux
        // contributions the scratch holds (the fused stage kernel keeps them
        // in shared memory and would leave the scratch unused)
        BatchView<R> split = grp.view();
        split.fusedMode = 0;
        residualSequence(split, stream_);
        guard.active = false;
        for (int d = 0; d < 3; d++) inst.c.f[d] = guard.saved[d];
        grp.refresh(stream_);
        const Control c1 = control();
        if (inst.c.dt_method == 0) copyOut(inst.c.dt, dt, N, stream_);
        else std::fill(dt, dt + N, inst.c.dt_method == 2 ? inst.c.fixed_dt : c1.dt_min);
        for (int v = 0; v < 5; v++) copyOut(inst.c.S2[v], r[v], N, stream_);
    });
}

// The state as double (float path: U - Uc); copies run on the solver's stream
// (asynchronous when the host buffers are pinned) and complete on return.
void Solver::getState(double* const out[5]) {
    const long N = mesh_.nodes();
    visit([&](auto& inst, auto&) {
        using R = std::remove_reference_t<decltype(*inst.c.U[0])>;
        if (sizeof(R) == sizeof(double)) {
            for (int v = 0; v < 5; v++)
                cudaCheck(cudaMemcpyAsync(out[v], inst.c.U[v], N * sizeof(double), cudaMemcpyDeviceToHost, stream_),
                          "cudaMemcpyAsync");
            cudaCheck(cudaStreamSynchronize(stream_), "cudaStreamSynchronize");
        } else {
            std::vector<R> u(N), cc(N);
            for (int v = 0; v < 5; v++) {
                cudaCheck(cudaMemcpyAsync(u.data(), inst.c.U[v], N * sizeof(R), cudaMemcpyDeviceToHost, stream_),
                          "cudaMemcpyAsync");
                cudaCheck(cudaMemcpyAsync(cc.data(), inst.c.Uc[v], N * sizeof(R), cudaMemcpyDeviceToHost, stream_),
                          "cudaMemcpyAsync");
                cudaCheck(cudaStreamSynchronize(stream_), "cudaStreamSynchronize");
                for (long q = 0; q < N; q++) out[v][q] = static_cast<double>(u[q]) - static_cast<double>(cc[q]);
            }
        }
    });
}

std::unique_ptr<HostFluid> Solver::hostFluid() const {
    if (table_) return std::make_unique<RealFluid>(*table_);
    return std::make_unique<IdealFluid>(proto_.gamma, proto_.rgas);
}

void Solver::writeSolution(const std::string& path) {
    const long N = mesh_.nodes();
    std::array<std::vector<double>, 5> U;
    double* out[5];
    for (int v = 0; v < 5; v++) {
        U[v].resize(N);
        out[v] = U[v].data();
    }
    getState(out);
    const double* in[5] = {out[0], out[1], out[2], out[3], out[4]};
    if (!proto_.viscous) {
        writeSolutionCsv(path, config_, mesh_, *hostFluid(), in);
        return;
    }
    std::map<std::string, std::vector<double>> extra;
    viscousOutputFields(in, extra);
    writeSolutionCsv(path, config_, mesh_, *hostFluid(), in, &extra);
}

// Output::updateViscousFields (src/output.cpp:240-306) with
// computeWallShearStress (:308-367): molecular viscosity of every node's
// temperature, the eddy viscosity of the model (0 without one; with SA
// getEddyViscosity of the state's density and the model's last laminar
// viscosity) and its working variable ("Nu Tilde"), and on the nodes of
// each no-slip wall (patch order; a later patch overwrites a shared node)
// the wall shear stress from the latest stage's velocity gradients and
// y+ = sqrt(|tau_w| rho) d / mu, d the wall-distance step to the next node
// off the wall (Solver::computeWallDistance, src/solver.cpp:657-700: the
// smallest node-to-node distance to any no-slip wall). Before the first
// iteration the gradients are zero (the reference has its start-up
// gradients there).
void Solver::viscousOutputFields(const double* const U[5], std::map<std::string, std::vector<double>>& out) {
    const long N = mesh_.nodes(), NI = mesh_.ni(), NJ = mesh_.nj(), NK = mesh_.nk();
    const auto fluid = hostFluid();
    const DevCaseT<double>& c = proto_;
    auto mu = [&](double T) {  // FluidIdeal / FluidReal::computeMolecularDynamicViscosity
        if (c.visc_const) return c.mu_const;
        return c.suth_mu * std::pow(T / c.suth_T, 1.5) * ((c.suth_T + c.suth_S) / (T + c.suth_S));
    };
    auto& muL = out["Molecular Viscosity"];
    out["Eddy Viscosity"].assign(static_cast<size_t>(N), 0.0);
    auto& wx = out["Wall Shear Stress X"];
    auto& wy = out["Wall Shear Stress Y"];
    auto& wz = out["Wall Shear Stress Z"];
    auto& yp = out["Y Plus"];
    muL.resize(static_cast<size_t>(N));
    for (auto* a : {&wx, &wy, &wz, &yp}) a->assign(static_cast<size_t>(N), 0.0);
    for (long q = 0; q < N; q++) {
        const Vec3 u(U[1][q] / U[0][q], U[2][q] / U[0][q], U[3][q] / U[0][q]);
        muL[q] = mu(fluid->temperature_rho_u_et(U[0][q], u, U[4][q] / U[0][q]));
    }
    if (c.sa) {  // TurbulenceModelSA::getEddyViscosity / getWorkingVariable
        std::vector<double> nuHat(static_cast<size_t>(N)), nuL(static_cast<size_t>(N));
        visit([&](auto& inst, auto&) {
            using R = std::remove_reference_t<decltype(*inst.c.U[0])>;
            std::vector<R> tmp(static_cast<size_t>(N));
            cudaCheck(cudaMemcpy(tmp.data(), inst.c.nuhat, N * sizeof(R), cudaMemcpyDeviceToHost), "cudaMemcpy");
            nuHat.assign(tmp.begin(), tmp.end());
            cudaCheck(cudaMemcpy(tmp.data(), inst.c.nul, N * sizeof(R), cudaMemcpyDeviceToHost), "cudaMemcpy");
            nuL.assign(tmp.begin(), tmp.end());
        });
        auto& eddy = out["Eddy Viscosity"];
        for (long q = 0; q < N; q++) {
            double e = 0.0;
            if (nuHat[q] > 0.0 && nuL[q] > 0.0) {
                const double chi = nuHat[q] / nuL[q];
                const double chi3 = chi * chi * chi;
                const double cv1_3 = 7.1 * 7.1 * 7.1;
                e = chi3 / (chi3 + cv1_3) * U[0][q] * nuHat[q];
            }
            eddy[q] = e;
        }
        out["Nu Tilde"] = nuHat;
    }
    std::array<std::vector<double>, 12> G;
    visit([&](auto& inst, auto&) {
        using R = std::remove_reference_t<decltype(*inst.c.U[0])>;
        std::vector<R> tmp(static_cast<size_t>(N));
        for (int g = 0; g < 12; g++) {
            cudaCheck(cudaMemcpyAsync(tmp.data(), inst.c.G[g], N * sizeof(R), cudaMemcpyDeviceToHost, stream_),
                      "cudaMemcpyAsync");
            cudaCheck(cudaStreamSynchronize(stream_), "cudaStreamSynchronize");
            G[g].assign(tmp.begin(), tmp.end());
        }
    });
    struct Range { long i0, i1, j0, j1, k0, k1; };
    std::vector<std::pair<const BoundaryPatch*, Range>> walls;
    for (const auto& b : boundaries_) {
        if (b.type != kBcNoSlipWall) continue;
        Range r{b.i_min, b.i_max, b.j_min, b.j_max, b.k_min, b.k_max};
        if (r.i0 == r.i1 && r.i0 == 0) r.i1 = 1;
        else if (r.i0 == r.i1 && r.i0 == NI) { r.i0 = NI - 1; r.i1 = NI; }
        else if (r.j0 == r.j1 && r.j0 == 0) r.j1 = 1;
        else if (r.j0 == r.j1 && r.j0 == NJ) { r.j0 = NJ - 1; r.j1 = NJ; }
        else if (r.k0 == r.k1 && r.k0 == 0) r.k1 = 1;
        else { r.k0 = NK - 1; r.k1 = NK; }  // buildWallMask has checked the indices
        walls.push_back({&b, r});
    }
    const auto& P = mesh_.vertices();
    std::map<long, double> memo;
    auto wallDistance = [&](long q) {
        const auto hit = memo.find(q);
        if (hit != memo.end()) return hit->second;
        double best = 1.0E9;
        for (const auto& w : walls) {
            double m = 1.0E9;
            for (long i = w.second.i0; i < w.second.i1; i++)
                for (long j = w.second.j0; j < w.second.j1; j++)
                    for (long k = w.second.k0; k < w.second.k1; k++) {
                        const Vec3& b = P[mesh_.idx(i, j, k)];
                        const double dx = P[q].x - b.x, dy = P[q].y - b.y, dz = P[q].z - b.z;
                        const double d = std::sqrt(dx * dx + dy * dy + dz * dz);
                        if (d < m) m = d;
                    }
            if (m < best) best = m;
        }
        memo[q] = best;
        return best;
    };
    for (const auto& w : walls) {
        const BoundaryPatch& b = *w.first;
        const int o = b.orientation;
        const long si = o == 0 ? 1 : (o == 1 ? -1 : 0), sj = o == 2 ? 1 : (o == 3 ? -1 : 0),
                   sk = o == 4 ? 1 : (o == 5 ? -1 : 0);
        for (long i = w.second.i0; i < w.second.i1; i++)
            for (long j = w.second.j0; j < w.second.j1; j++)
                for (long k = w.second.k0; k < w.second.k1; k++) {
                    const long q = mesh_.idx(i, j, k);
                    const Vec3 gu(G[0][q], G[1][q], G[2][q]), gv(G[3][q], G[4][q], G[5][q]), gw(G[6][q], G[7][q], G[8][q]);
                    const double me = muL[q] + 0.0;
                    const double lam = -2.0 * me / 3.0;
                    const double xx = lam * (gu.x + gv.y + gw.z) + 2.0 * me * gu.x;
                    const double yy = lam * (gu.x + gv.y + gw.z) + 2.0 * me * gv.y;
                    const double zz = lam * (gu.x + gv.y + gw.z) + 2.0 * me * gw.z;
                    const double xy = me * (gu.y + gv.x), xz = me * (gu.z + gw.x), yz = me * (gv.z + gw.y);
                    Vec3 s;
                    switch (o) {
                        case 0: s = mesh_.surfaces(0)[mesh_.faceIdx(0, 0, j, k)]; break;
                        case 1: s = -mesh_.surfaces(0)[mesh_.faceIdx(0, b.i_max, j, k)]; break;
                        case 2: s = mesh_.surfaces(1)[mesh_.faceIdx(1, i, 0, k)]; break;
                        case 3: s = -mesh_.surfaces(1)[mesh_.faceIdx(1, i, b.j_max, k)]; break;
                        case 4: s = mesh_.surfaces(2)[mesh_.faceIdx(2, i, j, 0)]; break;
                        default: s = -mesh_.surfaces(2)[mesh_.faceIdx(2, i, j, b.k_max)]; break;
                    }
                    const double sm = s.magnitude();
                    s = (sm == 0.0) ? Vec3(0, 0, 0) : s / sm;  // Vector3D::normalized
                    Vec3 t(xx * s.x + xy * s.y + xz * s.z, xy * s.x + yy * s.y + yz * s.z, xz * s.x + yz * s.y + zz * s.z);
                    t = t - s * t.dot(s);
                    wx[q] = t.x;
                    wy[q] = t.y;
                    wz[q] = t.z;
                    const double d = wallDistance(mesh_.idx(i + si, j + sj, k + sk)) - wallDistance(q);
                    yp[q] = std::sqrt(t.magnitude() * U[0][q]) * d / muL[q];
                }
    }
}

// Solver::solve starts with preprocessSolution (src/solver.cpp:1323, :3189-3203):
// with viscosity on, the momentum of every no-slip wall node becomes
// density * 0 (walls at rest). Every iteration keeps it there, so doing it
// whenever a state is set gives the reference's states.
void Solver::setState(const double* const in[5]) {
    promo_.reset();
    if (!proto_.viscous) {
        uploadState(in);
        return;
    }
    const long N = mesh_.nodes();
    std::array<std::vector<double>, 3> mom;
    const double* u[5] = {in[0], nullptr, nullptr, nullptr, in[4]};
    for (int v = 0; v < 3; v++) {
        mom[v].assign(in[v + 1], in[v + 1] + N);
        for (long q = 0; q < N; q++)
            if (wall_[static_cast<size_t>(q)]) mom[v][q] = in[0][q] * 0.0;
        u[v + 1] = mom[v].data();
    }
    uploadState(u);
}

void Solver::uploadState(const double* const in[5]) {
    const long N = mesh_.nodes();
    visit([&](auto& inst, auto&) {
        using R = std::remove_reference_t<decltype(*inst.c.U[0])>;
        if (sizeof(R) == sizeof(double)) {
            for (int v = 0; v < 5; v++)
                cudaCheck(cudaMemcpyAsync(inst.c.U[v], in[v], N * sizeof(double), cudaMemcpyHostToDevice, stream_),
                          "cudaMemcpyAsync");
            cudaCheck(cudaStreamSynchronize(stream_), "cudaStreamSynchronize");
        } else {
            // U = float(x), Uc = U - x, so that U - Uc carries x beyond float precision
            std::vector<R> u(N), cc(N);
            for (int v = 0; v < 5; v++) {
                for (long q = 0; q < N; q++) {
                    u[q] = static_cast<R>(in[v][q]);
                    cc[q] = static_cast<R>(static_cast<double>(u[q]) - in[v][q]);
                }
                cudaCheck(cudaMemcpyAsync(inst.c.U[v], u.data(), N * sizeof(R), cudaMemcpyHostToDevice, stream_),
                          "cudaMemcpyAsync");
                cudaCheck(cudaMemcpyAsync(inst.c.Uc[v], cc.data(), N * sizeof(R), cudaMemcpyHostToDevice, stream_),
                          "cudaMemcpyAsync");
                cudaCheck(cudaStreamSynchronize(stream_), "cudaStreamSynchronize");
            }
        }
    });
}

void Solver::getTurbo(double massflow[6], double turbo[4]) {
    visit([&](auto& inst, auto& grp) {
        using R = std::remove_reference_t<decltype(*inst.c.U[0])>;
        cudaCheck(Launcher<R>::boundaryIntegrals(grp.view(), true, 1, stream_), "launch k_bint");
        cudaCheck(Launcher<R>::pre(grp.view(), true, false, false, 1, stream_), "launch k_pre");
    });
    const Control c = control();
    for (int b = 0; b < 6; b++) massflow[b] = c.massflow[b];
    for (int b = 0; b < 4; b++) turbo[b] = c.turbo[b];
}

void Solver::profileKernels(int reps, double* outMs) {
    for (int k = 0; k < kKernelKinds; k++) outMs[k] = 0.0;
    if (reps <= 0) return;
    const Control saved = control();
    visit([&](auto& inst, auto& grp) {
        using R = std::remove_reference_t<decltype(*inst.c.U[0])>;
        using L = Launcher<R>;
        const BatchView<R>& fv = grp.view();
        BatchView<R> v = fv;  // the split stage kernels of every member
        v.fusedMode = 0;
        const long N = mesh_.nodes();
        std::vector<R> dtSaved(N);
        cudaCheck(cudaMemcpy(dtSaved.data(), inst.c.dt, N * sizeof(R), cudaMemcpyDeviceToHost), "cudaMemcpy");
        cudaEvent_t e0, e1;
        cudaCheck(cudaEventCreate(&e0), "cudaEventCreate");
        cudaCheck(cudaEventCreate(&e1), "cudaEventCreate");
        auto timeIt = [&](int kind, auto&& launch) {
            launch();  // warm
            cudaCheck(cudaEventRecord(e0, stream_), "cudaEventRecord");
            for (int r = 0; r < reps; r++) launch();
            cudaCheck(cudaEventRecord(e1, stream_), "cudaEventRecord");
            cudaCheck(cudaEventSynchronize(e1), "cudaEventSynchronize");
            float ms = 0.f;
            cudaCheck(cudaEventElapsedTime(&ms, e0, e1), "cudaEventElapsedTime");
            outMs[kind] = static_cast<double>(ms) / reps;
        };
        const int lastStage = inst.c.nstages - 1;
        // stage 0 reads U^n and writes S1, leaving U^n untouched
        if (inst.c.need_turbo) timeIt(0, [&] { cudaCheck(L::boundaryIntegrals(v, false, 1, stream_), "k_bint"); });
        if (inst.c.dt_method != 2) timeIt(1, [&] { cudaCheck(L::timeStep(v, 1, stream_), "k_dt"); });
        timeIt(2, [&] { cudaCheck(L::pre(v, false, true, false, 1, stream_), "k_pre"); });
        const int dirs = inst.c.topo == 1 ? 3 : 2;
        for (int d = 0; d < dirs; d++) timeIt(3 + d, [&] { cudaCheck(L::faces(v, d, 0, 1, stream_), "k_faces"); });
        timeIt(6, [&] { cudaCheck(L::nodes(v, 0, 1, stream_), "k_nodes"); });
        if (inst.c.periodic) timeIt(7, [&] { cudaCheck(L::periodic(v, 0, 1, stream_), "k_periodic"); });
        timeIt(8, [&] { cudaCheck(L::finalize(v, 1, stream_), "k_finalize"); });
        timeIt(9, [&] { cudaCheck(L::prim(v, 0, 1, stream_), "k_prim"); });
        if (inst.c.fuse_ok) {
            BatchView<R> f = fv;
            f.fusedMode = 1;
            timeIt(10, [&] { cudaCheck(L::fused(f, 0, 1, stream_), "k_stage"); });
        }
        (void)lastStage;
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        cudaCheck(cudaMemcpy(inst.c.dt, dtSaved.data(), N * sizeof(R), cudaMemcpyHostToDevice), "cudaMemcpy");
        *hostCtl_ = saved;
        cudaCheck(cudaMemcpy(inst.c.ctl, hostCtl_, sizeof(Control), cudaMemcpyHostToDevice), "cudaMemcpy");
        cudaCheck(cudaDeviceSynchronize(), "cudaDeviceSynchronize");
    });
}

void Solver::setStatus(int status) {
    Control* d = g64_ ? i64_->c.ctl : i32_->c.ctl;
    cudaCheck(cudaMemcpy(&d->status, &status, sizeof(int), cudaMemcpyHostToDevice), "cudaMemcpy");
}

void Solver::promoteToFP64() {
    preparePromotion();
    commitPromotion();
}

void Solver::preparePromotion() {
    if (prec_ == kFP64 || promo_) return;
    const long N = mesh_.nodes();
    std::array<std::vector<double>, 5> U;
    double* out[5];
    for (int v = 0; v < 5; v++) {
        U[v].resize(N);
        out[v] = U[v].data();
    }
    getState(out);
    auto p = std::make_unique<Promotion>();
    p->ctl = control();
    proto_.compensated = 0;
    p->inst = std::make_unique<InstanceT<double>>();
    InstanceT<double>& inst = *p->inst;
    inst.reserve(2 * i32_->usedBytes() + (size_t(1) << 16));  // float arrays become double
    uploadArrays(inst);
    p->grp = std::make_unique<GroupT<double>>(std::vector<InstanceT<double>*>{&inst});
    p->grp->setFusedMode(fusion_);
    const DevCaseT<float>& f = i32_->c;
    if (proto_.sa) {  // the model's nu hat and laminar viscosity carry over
        std::vector<float> tf(static_cast<size_t>(N));
        std::vector<double> td(static_cast<size_t>(N));
        const std::pair<const float*, double*> pairs[2] = {{f.nuhat, inst.c.nuhat}, {f.nul, inst.c.nul}};
        for (const auto& pr : pairs) {
            cudaCheck(cudaMemcpy(tf.data(), pr.first, N * sizeof(float), cudaMemcpyDeviceToHost), "cudaMemcpy");
            std::copy(tf.begin(), tf.end(), td.begin());
            cudaCheck(cudaMemcpy(pr.second, td.data(), N * sizeof(double), cudaMemcpyHostToDevice), "cudaMemcpy");
        }
    }
    if (proto_.nprofiles)
        cudaCheck(cudaMemcpy(inst.c.prof_p, f.prof_p, profP_.size() * sizeof(double), cudaMemcpyDeviceToDevice),
                  "cudaMemcpy");
    cudaCheck(cudaMemcpy(inst.c.hist, f.hist, static_cast<size_t>(proto_.hist_cap) * kHistWidth * sizeof(double),
                         cudaMemcpyDeviceToDevice),
              "cudaMemcpy");
    // the state (setState: no-slip wall nodes carry no momentum)
    std::array<std::vector<double>, 3> mom;
    const double* in[5] = {U[0].data(), U[1].data(), U[2].data(), U[3].data(), U[4].data()};
    if (proto_.viscous)
        for (int v = 0; v < 3; v++) {
            mom[v] = U[v + 1];
            for (long q = 0; q < N; q++)
                if (wall_[static_cast<size_t>(q)]) mom[v][q] = U[0][q] * 0.0;
            in[v + 1] = mom[v].data();
        }
    for (int v = 0; v < 5; v++)
        cudaCheck(cudaMemcpyAsync(inst.c.U[v], in[v], N * sizeof(double), cudaMemcpyHostToDevice, stream_),
                  "cudaMemcpyAsync");
    cudaCheck(cudaStreamSynchronize(stream_), "cudaStreamSynchronize");
    promo_ = std::move(p);
}

void Solver::commitPromotion() {
    if (prec_ == kFP64) return;
    if (!promo_) preparePromotion();
    Control ctl = promo_->ctl;
    if (ctl.status == 4) ctl.status = 0;  // paused by a server: running again
    i64_ = std::move(promo_->inst);
    g64_ = std::move(promo_->grp);
    promo_.reset();
    prec_ = kFP64;
    *hostCtl_ = ctl;
    cudaCheck(cudaMemcpy(i64_->c.ctl, hostCtl_, sizeof(Control), cudaMemcpyHostToDevice), "cudaMemcpy");
    g32_.reset();
    i32_.reset();
    cudaCheck(cudaStreamSynchronize(cudaStreamLegacy), "cudaStreamSynchronize");
    cudaCheck(cudaStreamSynchronize(stream_), "cudaStreamSynchronize");
}

long long Solver::history(long long maxRows, double* lognorm, double* massflow, double* turbo, double* hub,
                          double* time) {
    const Control c = control();
    const long long cap = proto_.hist_cap;
    long long rows = std::min<long long>(c.it - c.hist_base, cap);
    if (rows < 0) rows = 0;
    if (!lognorm && !massflow && !turbo && !hub && !time) return rows;
    rows = std::min(rows, maxRows);
    std::vector<double> h(static_cast<size_t>(rows) * kHistWidth);
    const double* dh = i64_ ? i64_->c.hist : i32_->c.hist;
    if (rows) cudaCheck(cudaMemcpy(h.data(), dh, h.size() * sizeof(double), cudaMemcpyDeviceToHost), "cudaMemcpy");
    for (long long r = 0; r < rows; r++) {
        const double* row = h.data() + r * kHistWidth;
        if (lognorm) std::copy(row, row + 5, lognorm + 5 * r);
        if (massflow) std::copy(row + 5, row + 11, massflow + 6 * r);
        if (turbo) std::copy(row + 11, row + 15, turbo + 4 * r);
        if (hub) hub[r] = row[15];
        if (time) time[r] = row[16];
    }
    return rows;
}

// The look-up tables on the device: every table in double and as a float copy,
// and the DevLut that points at them.
template <typename R>
const DevLut* Solver::uploadLut(InstanceT<R>& inst) {
    DevLut h{};
    auto fill = [&](DevTable& t, const HostTable& src) {
        t.xmin = src.xmin;
        t.xmax = src.xmax;
        t.ymin = src.ymin;
        t.ymax = src.ymax;
        t.dx = src.dx;
        t.dy = src.dy;
        t.fxmin = static_cast<float>(src.xmin);
        t.fxmax = static_cast<float>(src.xmax);
        t.fymin = static_cast<float>(src.ymin);
        t.fymax = static_cast<float>(src.ymax);
        t.fdx = static_cast<float>(src.dx);
        t.fdy = static_cast<float>(src.dy);
        t.nx = static_cast<int>(src.nx);
        t.ny = static_cast<int>(src.ny);
        t.d = inst.uploadD(src.d);
        std::vector<float> f(src.d.begin(), src.d.end());
        float* df = static_cast<float*>(inst.allocBytes(f.size() * sizeof(float)));
        cudaCheck(cudaMemcpy(df, f.data(), f.size() * sizeof(float), cudaMemcpyHostToDevice), "cudaMemcpy");
        t.f = df;
    };
    for (int q = 0; q < 8; q++) fill(h.re[q], table_->rhoE()[q]);
    for (int q = 0; q < 4; q++) fill(h.pt[q], table_->pT()[q]);
    for (int q = 0; q < 3; q++) fill(h.ps[q], table_->pS()[q]);
    DevLut* d = static_cast<DevLut*>(inst.allocBytes(sizeof(DevLut)));
    cudaCheck(cudaMemcpy(d, &h, sizeof(DevLut), cudaMemcpyHostToDevice), "cudaMemcpy");
    return d;
}

template void Solver::uploadArrays<double>(InstanceT<double>&);
template void Solver::uploadArrays<float>(InstanceT<float>&);
template void Solver::initializeState<double>(InstanceT<double>&, GroupT<double>&);
template void Solver::initializeState<float>(InstanceT<float>&, GroupT<float>&);

}  // namespace ctbfm
