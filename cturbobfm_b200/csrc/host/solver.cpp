// Solver: see solver.hpp.
#include "solver.hpp"

#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstring>
#include <fstream>
#include <sstream>

namespace ctbfm {

namespace {

constexpr int kHistWidth = 16;

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
    if (s == "inlet_supersonic" || s == "outlet_supersonic" || s == "mass_flow" || s == "outlet_mass_flow" ||
        s == "massflow" || s == "mass_flow_rate" || s == "inlet_2d" || s == "no_slip_wall" || s == "transparent" ||
        s == "farfield")
        throw ConfigError("BoundaryType " + s + " is outside this library's scope");
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

void Solver::check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw CudaError(std::string(what) + ": " + cudaGetErrorString(e));
}

double* Solver::alloc(size_t count) {
    void* p = nullptr;
    check(cudaMalloc(&p, std::max<size_t>(count, 1) * sizeof(double)), "cudaMalloc");
    allocations_.push_back(p);
    deviceBytes_ += std::max<size_t>(count, 1) * sizeof(double);
    return static_cast<double*>(p);
}

const double* Solver::upload(const std::vector<double>& v) {
    double* d = alloc(v.size());
    check(cudaMemcpy(d, v.data(), v.size() * sizeof(double), cudaMemcpyHostToDevice), "cudaMemcpy H2D");
    return d;
}

Solver::Solver(Config& config, Mesh& mesh) : config_(config), mesh_(mesh), topo_(config.getTopology()) {
    if (config.isViscosityActive()) throw ConfigError("Viscous fluxes are outside this library's Euler path");
    if (config.parseBool("TURBULENCE_ACTIVE", false)) throw ConfigError("Turbulence models are outside this library's Euler path");
    if (config.parseBool("RESTART_SOLUTION", false)) throw ConfigError("Restart files are outside this library's scope");
    const std::string fluid = config.has("FLUID_MODEL") ? config.get("FLUID_MODEL") : "None";
    if (fluid != "None" && fluid != "Ideal" && fluid != "ideal" && fluid != "IDEAL")
        throw ConfigError("Only the ideal-gas fluid model is supported");
    if (config.isAccelerationActive() && config.getTimeStepMethod() != TimeStepMethod::Fixed)
        throw ConfigError("Rotational speed scaling factor is only active for fixed time step method");
    coeffs_ = config.getTimeIntegrationCoeffs();
    maxIter_ = config.getMaxIterations();
    // every setting and input file is validated before the first CUDA call,
    // so that input errors are reported as such on any machine
    setupModels();
    readBoundaries();
    buildBoundaryStructures();
    validateSettings();
    check(cudaStreamCreateWithFlags(&ownStream_, cudaStreamNonBlocking), "cudaStreamCreate");
    stream_ = ownStream_;
    check(cudaMallocHost(reinterpret_cast<void**>(&hostCtl_), sizeof(Control)), "cudaMallocHost");
    std::memset(hostCtl_, 0, sizeof(Control));
    uploadBoundaryStructures();
    upload();
    initializeSolution();
    initializeProfilesAndPlenum();
}

// Parses every key the device set-up reads (the reference's getters throw on
// the same inputs).
void Solver::validateSettings() {
    const TimeStepMethod m = config_.getTimeStepMethod();
    config_.getCFL();
    if (m == TimeStepMethod::Fixed) config_.getFixedTimeStep();
    config_.getFluidGamma();
    config_.getFluidGasConstant();
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
    if (graph_) cudaGraphExecDestroy(graph_);
    if (ownStream_) cudaStreamSynchronize(ownStream_);
    for (void* p : allocations_) cudaFree(p);
    if (hostCtl_) cudaFreeHost(hostCtl_);
    if (ownStream_) cudaStreamDestroy(ownStream_);
}

// Solver::buildAdvectionModel / buildBfmInfo (src/solver.cpp:185-198, 701-749).
void Solver::setupModels() {
    if (config_.getAdvectionScheme() == Scheme::JST) advection_ = std::make_unique<AdvectionJst>(config_);
    else advection_ = std::make_unique<AdvectionRoe>(config_);
    switch (config_.getBFMModel()) {
        case BfmModel::Hall: bfm_ = std::make_unique<SourceBFMHall>(config_); break;
        case BfmModel::HallThollet: bfm_ = std::make_unique<SourceBFMThollet>(config_); break;
        case BfmModel::LiftDrag: bfm_ = std::make_unique<SourceBFMLiftDrag>(config_); break;
        default: bfm_ = std::make_unique<SourceBFMBase>(config_); break;
    }
}

// Solver::readBoundaryFile (src/solver.cpp:232-294).
void Solver::readBoundaries() {
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
        BoundaryPatch p;
        std::getline(ss, tok, ',');
        tok.erase(std::remove(tok.begin(), tok.end(), ' '), tok.end());
        p.name = tok;
        long v[6];
        for (int q = 0; q < 6; q++) {
            if (!std::getline(ss, tok, ',')) throw ConfigError("bad boundary row for " + p.name);
            tok.erase(std::remove(tok.begin(), tok.end(), ' '), tok.end());
            v[q] = std::stoi(tok);
        }
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
    if (boundaries_.size() > static_cast<size_t>(kMaxPatches))
        throw ConfigError("more than 16 boundary patches");
}

// Solver::buildBoundaryDataStructures, buildBoundaryFluxes,
// buildBoundaryConditionsMap, checkBoundaryConditionsMap
// (src/solver.cpp:296-593).
void Solver::buildBoundaryStructures() {
    const long NI = mesh_.ni(), NJ = mesh_.nj(), NK = mesh_.nk();
    std::vector<double> profP, profR;
    int nprof = 0;
    c_.periodic = 0;
    for (size_t m = 0; m < boundaries_.size(); m++) {
        BoundaryPatch& b = boundaries_[m];
        if (b.type == kBcRadialEq || b.type == kBcThrottle) {
            if (b.i_min != b.i_max) throw ConfigError("Radial equilibrium only supported on j-k patches");
            if (b.i_min == 0) throw ConfigError("Radial equilibrium only supported to the last i-position");
            if (b.j_max <= b.j_min) throw ConfigError("Invalid boundary indices for radial equilibrium patch: " + b.name);
            if (b.j_min != 0) throw ConfigError("radial profiles must start at j = 0 (the profile is indexed by the face's j)");
            if (nprof >= kMaxProfiles) throw ConfigError("too many radial profiles");
            const int n = static_cast<int>(b.j_max - b.j_min);
            c_.prof_off[nprof] = static_cast<int>(profP.size());
            c_.prof_n[nprof] = n;
            c_.prof_type[nprof] = b.type;
            c_.prof_i[nprof] = static_cast<int>(b.i_min > 0 ? b.i_min - 1 : 0);
            c_.prof_j0[nprof] = static_cast<int>(b.j_min);
            c_.prof_kt[nprof] = b.type == kBcThrottle ? (b.values.empty() ? 0.0 : b.values[0]) : 0.0;
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
                c_.periodic = 1;
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
        } else {
            b.flux = std::make_unique<BoundaryFake>(b.type);
        }
        c_.patch[m] = b.flux->toDevice();
    }
    c_.npatches = static_cast<int>(boundaries_.size());
    c_.nprofiles = nprof;
    profiles_ = nprof > 0;

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
    c_.inlet_pt = 0.0;
    for (const auto& b : boundaries_)
        if (b.type == kBcInlet) {
            c_.inlet_pt = b.values[0];
            break;
        }
    c_.throttle_kt = 0.0;
    bool hasThrottle = false;
    for (const auto& b : boundaries_)
        if (b.type == kBcThrottle) {
            hasThrottle = true;
            c_.throttle_kt = b.values.empty() ? 0.0 : b.values[0];
        }
    c_.greitzer = config_.enableGreitzerModeling() ? 1 : 0;
    if (c_.greitzer && !hasThrottle) throw ConfigError("Greitzer modeling enabled but no throttle boundary condition found!");
    if (c_.greitzer || hasThrottle) needTurbo_ = true;
    if (c_.greitzer) {
        profiles_ = true;
        c_.plenum_volume = config_.getGreitzerPlenumVolume();
        c_.ambient_p = config_.getGreitzerAmbientPressure();
    }
    c_.need_turbo = needTurbo_ ? 1 : 0;
    // TURBO_DIRECTION or the inlet orientation (src/solver.cpp:1654-1680)
    std::string dir = config_.has("TURBO_DIRECTION") ? config_.get("TURBO_DIRECTION") : "i";
    if (!config_.has("TURBO_DIRECTION"))
        for (const auto& b : boundaries_)
            if (b.type == kBcInlet) {
                if (b.orientation == 2) { dir = "j"; break; }
                if (b.orientation == 3) { dir = "-j"; break; }
            }
    c_.turbo_dir = dir == "-i" ? 1 : ((dir == "j" || dir == "+j") ? 2 : (dir == "-j" ? 3 : 0));
}

void Solver::uploadBoundaryStructures() {
    auto up8 = [&](const std::vector<signed char>& v) {
        void* d = nullptr;
        check(cudaMalloc(&d, v.size()), "cudaMalloc");
        allocations_.push_back(d);
        check(cudaMemcpy(d, v.data(), v.size(), cudaMemcpyHostToDevice), "cudaMemcpy");
        return static_cast<const signed char*>(d);
    };
    c_.mapI = up8(mapI_);
    c_.mapJ = up8(mapJ_);
    c_.mapK = up8(mapK_);
    if (c_.nprofiles) {
        c_.prof_p = alloc(profP_.size());
        check(cudaMemcpy(c_.prof_p, profP_.data(), profP_.size() * sizeof(double), cudaMemcpyHostToDevice), "cudaMemcpy");
        c_.prof_r = upload(profR_);
    }
}

void Solver::upload() {
    const long NI = mesh_.ni(), NJ = mesh_.nj(), NK = mesh_.nk(), N = mesh_.nodes();
    c_.ni = static_cast<int>(NI);
    c_.nj = static_cast<int>(NJ);
    c_.nk = static_cast<int>(NK);
    c_.n = N;
    c_.topo = static_cast<int>(topo_);
    advection_->configure(c_);
    c_.nstages = static_cast<int>(coeffs_.size());
    for (size_t s = 0; s < coeffs_.size(); s++) c_.coeffs[s] = coeffs_[s];
    c_.dt_method = static_cast<int>(config_.getTimeStepMethod());
    c_.steady = config_.isSimulationSteady() ? 1 : 0;
    c_.drop = config_.getResidualsDropConvergence();
    c_.gamma = config_.getFluidGamma();
    c_.rgas = config_.getFluidGasConstant();
    c_.cp = (c_.gamma * c_.rgas) / (c_.gamma - 1);
    c_.cfl = config_.getCFL();
    c_.fixed_dt = c_.dt_method == 2 ? config_.getFixedTimeStep() : 0.0;
    c_.per_angle_deg = periodicAngleDeg_;
    c_.per_cos_p = std::cos(periodicAngleRad_);
    c_.per_sin_p = std::sin(periodicAngleRad_);
    c_.per_cos_m = std::cos(-periodicAngleRad_);
    c_.per_sin_m = std::sin(-periodicAngleRad_);
    c_.wedge = mesh_.wedgeAngle();
    c_.ramp_iters = config_.getOutletPressureRampMaxIterations();
    c_.init_p = config_.getInitPressure();
    c_.inlet_cyl = config_.isInletCylindrical() ? 1 : 0;
    c_.bfm = config_.isBFMActive() ? 1 : 0;
    bfm_->configure(c_);
    c_.speed_scale = config_.getRotationalSpeedScalingFactor();
    c_.accel = config_.isAccelerationActive() ? 1 : 0;
    if (c_.accel) {
        c_.acc_t0 = config_.parseFloat("ACCELERATION_INITIAL_TIME");
        c_.acc_t1 = config_.parseFloat("ACCELERATION_FINAL_TIME");
        c_.acc_s0 = config_.parseFloat("ROTATIONAL_SPEED_SCALING_FACTOR_INITIAL");
        c_.acc_s1 = config_.parseFloat("ROTATIONAL_SPEED_SCALING_FACTOR_FINAL");
    }
    if (c_.perturb) {
        const auto pc = config_.parseList("PERTURBATION_CENTER");
        if (pc.size() < 3) throw ConfigError("PERTURBATION_CENTER needs 3 values");
        for (int q = 0; q < 3; q++) c_.pert_c[q] = std::stod(pc[q]);
        c_.pert_r = config_.parseFloat("PERTURBATION_RADIAL_EXTENSION");
        c_.pert_s = config_.parseFloat("PERTURBATION_SCALING_FACTOR");
        c_.pert_t0 = config_.parseFloat("PERTURBATION_TIME_START");
        c_.pert_dur = config_.parseFloat("PERTURBATION_TIME_DURATION");
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
        c_.f[d].nx = upload(nx);
        c_.f[d].ny = upload(ny);
        c_.f[d].nz = upload(nz);
        c_.f[d].area = upload(ar);
        for (int v = 0; v < 5; v++) c_.f[d].c[v] = alloc(S.size());
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
    c_.vol = upload(mesh_.volumes());
    c_.cost = upload(cst);
    c_.sint = upload(snt);
    c_.radius = upload(rad);
    c_.areaK0 = upload(aK);
    for (int e = 0; e < 12; e++) c_.edge[e] = upload(edge[e]);
    {
        std::vector<double> vx(N), vy(N), vz(N);
        for (long q = 0; q < N; q++) {
            vx[q] = mesh_.vertices()[q].x;
            vy[q] = mesh_.vertices()[q].y;
            vz[q] = mesh_.vertices()[q].z;
        }
        c_.vx = upload(vx);
        c_.vy = upload(vy);
        c_.vz = upload(vz);
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
        c_.bsx[b] = upload(sx);
        c_.bsy[b] = upload(sy);
        c_.bsz[b] = upload(sz);
    }
    // BFM fields (include/types.hpp:1036-1078 names)
    if (c_.bfm) {
        auto need = [&](const char* name) { return upload(mesh_.field(name)); };
        auto opt = [&](const char* name) -> const double* {
            return mesh_.hasField(name) ? upload(mesh_.field(name)) : nullptr;
        };
        c_.blk = need("blockage");
        const auto& gb = mesh_.blockageGradient();
        std::vector<double> gx(N), gy(N), gz(N);
        for (long q = 0; q < N; q++) {
            gx[q] = gb[q].x;
            gy[q] = gb[q].y;
            gz[q] = gb[q].z;
        }
        c_.gbx = upload(gx);
        c_.gby = upload(gy);
        c_.gbz = upload(gz);
        c_.bpresent = need("bladePresent");
        c_.nblades = need("numberBlades");
        if (c_.bfm_model != 0 && c_.bfm_model != 4) {
            // SourceBFMBase::computeFlowState reads all of these (src/source_bfm_base.cpp:104-149)
            c_.nax = need("normalAxial");
            c_.nrad = need("normalRadial");
            c_.ntan = need("normalTangential");
            c_.rpm = need("rpm");
            need("bladeLeanAngle");
            need("bladeGasPathAngle");
            const auto& metal = mesh_.field("bladeMetalAngle");
            std::vector<double> cm(N);
            for (long q = 0; q < N; q++) cm[q] = std::cos(metal[q]);
            c_.cosmetal = upload(cm);
        } else {
            c_.rpm = opt("rpm");
        }
        if (c_.bfm_model == 2 || c_.bfm_model == 3) c_.stwl = need("streamwiseLength");
        if (c_.bfm_model == 2 && c_.offdesign) c_.devpivot = need("deviationAnglePivot");
        if (c_.stalled) c_.devstall = need("deviationAngleStall");
        if (c_.bfm_model == 3) {
            c_.ldbeta0 = need("liftDragBeta0");
            c_.ldkp = need("liftDragKpEtamax");
            if (c_.le_idx < 0 || c_.le_idx >= NI || c_.te_idx < 0 || c_.te_idx >= NI)
                throw ConfigError("LEADING_EDGE_INDEX / TRAILING_EDGE_INDEX outside the grid");
        }
        if (topo_ == Topology::ThreeD && !c_.rpm) c_.rpm = need("rpm");
    }
    // state, stage buffers, reductions, control block, history
    for (int v = 0; v < 5; v++) {
        c_.U[v] = alloc(N);
        c_.S1[v] = alloc(N);
        c_.S2[v] = alloc(N);
        c_.Rp[v] = alloc(2 * NI * NJ);
        c_.W[v] = alloc(N);
    }
    c_.dt = alloc(N);
    c_.node_blocks = nodeBlocks(N);
    c_.per_blocks = periodicBlocks(NI * NJ);
    c_.dt_blocks = c_.node_blocks;
    c_.partial = alloc(static_cast<size_t>(c_.node_blocks + c_.per_blocks) * 5 + c_.dt_blocks);
    void* ctl = nullptr;
    check(cudaMalloc(&ctl, sizeof(Control)), "cudaMalloc");
    allocations_.push_back(ctl);
    c_.ctl = static_cast<Control*>(ctl);
    c_.hist_cap = std::min<long long>(std::max<long long>(maxIter_, 1024), 1 << 20);
    c_.hist = alloc(static_cast<size_t>(c_.hist_cap) * kHistWidth);
}

// FluidIdeal::computeInitFields (src/fluid_ideal.cpp:155-170) and
// Solver::initializeSolutionFromScratch (src/solver.cpp:777-836).
void Solver::initializeSolution() {
    const double M = config_.getInitMachNumber(), T = config_.getInitTemperature(), p = config_.getInitPressure();
    const double g = c_.gamma, R = c_.rgas;
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
    for (long i = 0; i < NI; i++)
        for (long j = 0; j < NJ; j++)
            for (long k = 0; k < NK; k++) {
                Vec3 dir = d0;
                if (adaptive) {  // Mesh::computeAdaptiveFlowDirection (src/mesh.cpp:637-661)
                    const long ia = i < NI - 1 ? i : NI - 2;
                    const Vec3 dv = V[mesh_.idx(ia + 1, j, k)] - V[mesh_.idx(ia, j, k)];
                    const double m = dv.magnitude();
                    dir = (m == 0) ? Vec3(0, 0, 0) : dv / m;
                }
                const double a = std::sqrt(g * R * T);
                const Vec3 u = (dir / dir.magnitude()) * a * M;
                const double rho = p / (R * T);
                const double e = p / ((g - 1) * rho);
                const double um = u.magnitude();
                const double et = e + 0.5 * (um * um);
                const long q = mesh_.idx(i, j, k);
                U[0][q] = rho;
                U[1][q] = rho * u.x;
                U[2][q] = rho * u.y;
                U[3][q] = rho * u.z;
                U[4][q] = rho * et;
            }
    for (int v = 0; v < 5; v++)
        check(cudaMemcpy(c_.U[v], U[v].data(), N * sizeof(double), cudaMemcpyHostToDevice), "cudaMemcpy");
    std::memset(hostCtl_, 0, sizeof(Control));
    check(cudaMemcpy(c_.ctl, hostCtl_, sizeof(Control), cudaMemcpyHostToDevice), "cudaMemcpy");
}

// Greitzer initial state and initial radial profiles
// (Solver::initializeSolutionArrays, src/solver.cpp:750-776).
void Solver::initializeProfilesAndPlenum() {
    const long N = mesh_.nodes();
    std::array<std::vector<double>, 5> U;
    for (int v = 0; v < 5; v++) {
        U[v].resize(N);
        check(cudaMemcpy(U[v].data(), c_.U[v], N * sizeof(double), cudaMemcpyDeviceToHost), "cudaMemcpy");
    }
    const HostGas gas{c_.gamma, c_.rgas};
    auto prim = [&](long q, double& rho, Vec3& u, double& et) {
        rho = U[0][q];
        u = Vec3(U[1][q] / U[0][q], U[2][q] / U[0][q], U[3][q] / U[0][q]);
        et = U[4][q] / U[0][q];
    };
    if (c_.greitzer) {
        double mf[6], tp[4];
        getTurbo(mf, tp);
        double rho, et;
        Vec3 u;
        prim(mesh_.idx(mesh_.ni() - 1, 0, 0), rho, u, et);
        Control ctl = control();
        ctl.gz_p = gas.pressure(rho, u, et);
        ctl.gz_T = gas.temperature(rho, u, et);
        ctl.gz_min = tp[0];
        ctl.gz_mout = tp[0];
        ctl.gz_t = 0.0;
        ctl.has_turbo = 0;
        *hostCtl_ = ctl;
        check(cudaMemcpy(c_.ctl, hostCtl_, sizeof(Control), cudaMemcpyHostToDevice), "cudaMemcpy");
    }
    if (c_.nprofiles) {
        std::vector<double> profP(c_.prof_off[c_.nprofiles - 1] + c_.prof_n[c_.nprofiles - 1]);
        for (int m = 0; m < c_.nprofiles; m++)
            for (int jj = 0; jj < c_.prof_n[m]; jj++) {
                double rho, et;
                Vec3 u;
                prim(mesh_.idx(c_.prof_i[m], c_.prof_j0[m] + jj, 0), rho, u, et);
                profP[c_.prof_off[m] + jj] = gas.pressure(rho, u, et);
            }
        check(cudaMemcpy(c_.prof_p, profP.data(), profP.size() * sizeof(double), cudaMemcpyHostToDevice), "cudaMemcpy");
    }
}

void Solver::setLimits(long long itStop, long long histBase) {
    check(launchSetLimits(c_, itStop, histBase, stream_), "launch set-limits");
}

// One iteration of the explicit branch of Solver::solve (src/solver.cpp:1337-1398).
void Solver::enqueueIteration() {
    const P5 U{{c_.U[0], c_.U[1], c_.U[2], c_.U[3], c_.U[4]}};
    const P5 A{{c_.S1[0], c_.S1[1], c_.S1[2], c_.S1[3], c_.S1[4]}};
    const P5 B{{c_.S2[0], c_.S2[1], c_.S2[2], c_.S2[3], c_.S2[4]}};
    if (needTurbo_) check(launchBoundaryIntegrals(c_, U, true, stream_), "launch k_bint");
    check(launchTimeStep(c_, U, stream_), "launch k_dt");
    check(launchPre(c_, U, needTurbo_, profiles_, true, stream_), "launch k_pre");
    const int ns = static_cast<int>(coeffs_.size());
    // stage buffers: RK4 U->A->B->A->U, RK3 U->A->B->U (the last stage updates U^n in place)
    const P5 in4[4] = {U, A, B, A}, out4[4] = {A, B, A, U};
    const P5 in3[3] = {U, A, B}, out3[3] = {A, B, U};
    for (int s = 0; s < ns; s++) {
        const P5& in = ns == 4 ? in4[s] : in3[s];
        const P5& out = ns == 4 ? out4[s] : out3[s];
        check(launchStage(c_, in, out, coeffs_[s], s == ns - 1, 0, B, stream_), "launch stage");
    }
    check(launchFinalize(c_, stream_), "launch k_finalize");
}

void Solver::captureGraph() {
    if (graph_) return;
    graphIters_ = 8;
    cudaGraph_t g = nullptr;
    check(cudaStreamBeginCapture(ownStream_, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture");
    cudaStream_t saved = stream_;
    stream_ = ownStream_;
    try {
        for (int i = 0; i < graphIters_; i++) enqueueIteration();
    } catch (...) {
        stream_ = saved;
        cudaStreamEndCapture(ownStream_, &g);
        if (g) cudaGraphDestroy(g);
        throw;
    }
    stream_ = saved;
    check(cudaStreamEndCapture(ownStream_, &g), "cudaStreamEndCapture");
    const cudaError_t e = cudaGraphInstantiate(&graph_, g, 0);
    cudaGraphDestroy(g);
    check(e, "cudaGraphInstantiate");
}

void Solver::enqueue(long long n) {
    if (n <= 0) return;
    setLimits(itHost_ + n, itHost_);
    captureGraph();
    long long left = n;
    while (left >= graphIters_) {
        check(cudaGraphLaunch(graph_, stream_), "cudaGraphLaunch");
        left -= graphIters_;
    }
    for (long long i = 0; i < left; i++) enqueueIteration();
    itHost_ += n;
}

Control Solver::control() {
    check(cudaMemcpyAsync(hostCtl_, c_.ctl, sizeof(Control), cudaMemcpyDeviceToHost, stream_), "cudaMemcpyAsync");
    check(cudaStreamSynchronize(stream_), "cudaStreamSynchronize");
    return *hostCtl_;
}

long long Solver::step(long long n) {
    const Control before = control();
    if (before.status != 0) return 0;
    itHost_ = before.it;
    enqueue(n);
    const Control after = control();
    itHost_ = after.it;
    return after.it - before.it;
}

long long Solver::solve() {
    long long done = 0;
    const long long chunk = 256;
    while (true) {
        const Control c = control();
        if (c.status != 0 || c.it >= maxIter_) break;
        const long long n = std::min<long long>(chunk, maxIter_ - c.it);
        done += step(n);
    }
    return done;
}

void Solver::computeResidual(double* dt, double* const r[5]) {
    const Control c0 = control();
    itHost_ = c0.it;
    DevCase fc = c_;
    fc.force = 1;  // run even after convergence
    const P5 U{{c_.U[0], c_.U[1], c_.U[2], c_.U[3], c_.U[4]}};
    const P5 A{{c_.S1[0], c_.S1[1], c_.S1[2], c_.S1[3], c_.S1[4]}};
    const P5 B{{c_.S2[0], c_.S2[1], c_.S2[2], c_.S2[3], c_.S2[4]}};
    if (needTurbo_) check(launchBoundaryIntegrals(fc, U, true, stream_), "launch k_bint");
    check(launchTimeStep(fc, U, stream_), "launch k_dt");
    check(launchPre(fc, U, needTurbo_, profiles_, true, stream_), "launch k_pre");
    check(launchStage(fc, U, A, 0.0, false, 1, B, stream_), "launch stage");
    const Control c1 = control();
    const long N = mesh_.nodes();
    if (c_.dt_method == 0) {
        check(cudaMemcpy(dt, c_.dt, N * sizeof(double), cudaMemcpyDeviceToHost), "cudaMemcpy");
    } else {
        std::fill(dt, dt + N, c_.dt_method == 2 ? c_.fixed_dt : c1.dt_min);
    }
    for (int v = 0; v < 5; v++)
        check(cudaMemcpy(r[v], c_.S2[v], N * sizeof(double), cudaMemcpyDeviceToHost), "cudaMemcpy");
}

// The residual evaluation of computeResidual with its per-face flux
// contributions kept in the static scratch array of noalloc.cu; nothing is
// allocated on the device (the caller cannot, or must not, call cudaMalloc).
void Solver::computeResidualNoAlloc(double* dt, double* const r[5]) {
    double* scratch = nullptr;
    size_t bytes = 0;
    check(noallocScratch(&scratch, &bytes), "static scratch set-up (cudaGetSymbolAddress)");
    const int dirs = c_.topo == 1 ? 3 : 2;
    size_t faces = 0;
    for (int d = 0; d < dirs; d++) faces += static_cast<size_t>(mesh_.faceCount(d));
    if (faces * 5 * sizeof(double) > bytes)
        throw ConfigError("ctbfm_compute_residual_noalloc: the case has " + std::to_string(faces) +
                          " faces and needs " + std::to_string(faces * 5 * sizeof(double)) +
                          " bytes of face scratch; the static array holds " + std::to_string(bytes) +
                          " bytes (at most " + std::to_string(bytes / (5 * sizeof(double))) + " faces)");
    const Control c0 = control();
    itHost_ = c0.it;
    DevCase fc = c_;
    fc.force = 1;  // run even after convergence
    size_t off = 0;
    for (int d = 0; d < dirs; d++) {
        const size_t nf = static_cast<size_t>(mesh_.faceCount(d));
        for (int v = 0; v < 5; v++) fc.f[d].c[v] = scratch + off + v * nf;
        off += 5 * nf;
    }
    const P5 U{{c_.U[0], c_.U[1], c_.U[2], c_.U[3], c_.U[4]}};
    const P5 A{{c_.S1[0], c_.S1[1], c_.S1[2], c_.S1[3], c_.S1[4]}};
    const P5 B{{c_.S2[0], c_.S2[1], c_.S2[2], c_.S2[3], c_.S2[4]}};
    if (needTurbo_) check(launchBoundaryIntegrals(fc, U, true, stream_), "launch k_bint");
    check(launchTimeStep(fc, U, stream_), "launch k_dt");
    check(launchPre(fc, U, needTurbo_, profiles_, true, stream_), "launch k_pre");
    check(launchStage(fc, U, A, 0.0, false, 1, B, stream_), "launch stage");
    const Control c1 = control();
    const long N = mesh_.nodes();
    if (c_.dt_method == 0) {
        check(cudaMemcpy(dt, c_.dt, N * sizeof(double), cudaMemcpyDeviceToHost), "cudaMemcpy");
    } else {
        std::fill(dt, dt + N, c_.dt_method == 2 ? c_.fixed_dt : c1.dt_min);
    }
    for (int v = 0; v < 5; v++)
        check(cudaMemcpy(r[v], c_.S2[v], N * sizeof(double), cudaMemcpyDeviceToHost), "cudaMemcpy");
}

// Copies run on the solver's stream (asynchronous when the host buffers are
// pinned) and are complete when the call returns.
void Solver::getState(double* const out[5]) {
    for (int v = 0; v < 5; v++)
        check(cudaMemcpyAsync(out[v], c_.U[v], mesh_.nodes() * sizeof(double), cudaMemcpyDeviceToHost, stream_),
              "cudaMemcpyAsync");
    check(cudaStreamSynchronize(stream_), "cudaStreamSynchronize");
}

void Solver::setState(const double* const in[5]) {
    for (int v = 0; v < 5; v++)
        check(cudaMemcpyAsync(c_.U[v], in[v], mesh_.nodes() * sizeof(double), cudaMemcpyHostToDevice, stream_),
              "cudaMemcpyAsync");
    check(cudaStreamSynchronize(stream_), "cudaStreamSynchronize");
}

void Solver::getTurbo(double massflow[6], double turbo[4]) {
    DevCase fc = c_;
    fc.force = 1;
    const P5 U{{c_.U[0], c_.U[1], c_.U[2], c_.U[3], c_.U[4]}};
    check(launchBoundaryIntegrals(fc, U, true, stream_), "launch k_bint");
    check(launchPre(fc, U, true, false, false, stream_), "launch k_pre");
    const Control c = control();
    for (int b = 0; b < 6; b++) massflow[b] = c.massflow[b];
    for (int b = 0; b < 4; b++) turbo[b] = c.turbo[b];
}

void Solver::profileKernels(int reps, double* outMs) {
    for (int k = 0; k < kKernelKinds; k++) outMs[k] = 0.0;
    if (reps <= 0) return;
    const Control saved = control();
    const long N = mesh_.nodes();
    std::vector<double> dtSaved(N);
    check(cudaMemcpy(dtSaved.data(), c_.dt, N * sizeof(double), cudaMemcpyDeviceToHost), "cudaMemcpy");
    DevCase fc = c_;
    fc.force = 1;
    const P5 U{{c_.U[0], c_.U[1], c_.U[2], c_.U[3], c_.U[4]}};
    const P5 A{{c_.S1[0], c_.S1[1], c_.S1[2], c_.S1[3], c_.S1[4]}};
    const P5 B{{c_.S2[0], c_.S2[1], c_.S2[2], c_.S2[3], c_.S2[4]}};
    cudaEvent_t e0, e1;
    check(cudaEventCreate(&e0), "cudaEventCreate");
    check(cudaEventCreate(&e1), "cudaEventCreate");
    auto timeIt = [&](int kind, auto&& launch) {
        launch();  // warm
        check(cudaEventRecord(e0, stream_), "cudaEventRecord");
        for (int r = 0; r < reps; r++) launch();
        check(cudaEventRecord(e1, stream_), "cudaEventRecord");
        check(cudaEventSynchronize(e1), "cudaEventSynchronize");
        float ms = 0.f;
        check(cudaEventElapsedTime(&ms, e0, e1), "cudaEventElapsedTime");
        outMs[kind] = static_cast<double>(ms) / reps;
    };
    if (needTurbo_) timeIt(0, [&] { check(launchBoundaryIntegrals(fc, U, true, stream_), "k_bint"); });
    if (c_.dt_method != 2) timeIt(1, [&] { check(launchTimeStep(fc, U, stream_), "k_dt"); });
    timeIt(2, [&] { check(launchPre(fc, U, needTurbo_, false, true, stream_), "k_pre"); });
    const int dirs = c_.topo == 1 ? 3 : 2;
    for (int d = 0; d < dirs; d++) timeIt(3 + d, [&] { check(launchFaces(fc, d, U, stream_), "k_faces"); });
    timeIt(6, [&] { check(launchNodes(fc, U, A, coeffs_.back(), true, 0, B, stream_), "k_nodes"); });
    if (c_.periodic) timeIt(7, [&] { check(launchPeriodic(fc, A, coeffs_.back(), true, 0, B, stream_), "k_periodic"); });
    timeIt(8, [&] { check(launchFinalize(fc, stream_), "k_finalize"); });
    timeIt(9, [&] { check(launchPrim(fc, U, stream_), "k_prim"); });
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    check(cudaMemcpy(c_.dt, dtSaved.data(), N * sizeof(double), cudaMemcpyHostToDevice), "cudaMemcpy");
    *hostCtl_ = saved;
    check(cudaMemcpy(c_.ctl, hostCtl_, sizeof(Control), cudaMemcpyHostToDevice), "cudaMemcpy");
}

long long Solver::history(long long maxRows, double* lognorm, double* massflow, double* turbo, double* hub) {
    const Control c = control();
    long long rows = std::min<long long>(c.it - c.hist_base, c_.hist_cap);
    if (rows < 0) rows = 0;
    if (!lognorm && !massflow && !turbo && !hub) return rows;
    rows = std::min(rows, maxRows);
    std::vector<double> h(static_cast<size_t>(rows) * kHistWidth);
    if (rows)
        check(cudaMemcpy(h.data(), c_.hist, h.size() * sizeof(double), cudaMemcpyDeviceToHost), "cudaMemcpy");
    for (long long r = 0; r < rows; r++) {
        const double* row = h.data() + r * kHistWidth;
        if (lognorm) std::copy(row, row + 5, lognorm + 5 * r);
        if (massflow) std::copy(row + 5, row + 11, massflow + 6 * r);
        if (turbo) std::copy(row + 11, row + 15, turbo + 4 * r);
        if (hub) hub[r] = row[15];
    }
    return rows;
}

}  // namespace ctbfm
