// Config: input.ini reader with the reference's keys and parsing rules
// (include/config.hpp, src/config.cpp). Keys are exact-case; "KEY = value"
// lines, ';' comments and '[' section lines skipped (src/config.cpp:15-44).
#pragma once

#include <map>
#include <stdexcept>
#include <string>
#include <vector>

namespace ctbfm {

enum class Topology { TwoD = 0, ThreeD = 1, Axisymmetric = 2, OneD = 3 };
enum class Scheme { JST = 0, Roe = 1 };
enum class Limiter { None = 0, VanAlbada = 1, VanLeer = 2, MinMod = 3 };
enum class TimeStepMethod { Local = 0, Global = 1, Fixed = 2 };
enum class BfmModel { None = 0, Hall = 1, HallThollet = 2, LiftDrag = 3, Blockage = 4, Chima = 5, Correlations = 6 };

class ConfigError : public std::runtime_error {
public:
    using std::runtime_error::runtime_error;
};

class Config {
public:
    explicit Config(const std::string& path);
    // Settings given in memory as key/value strings, trimmed as the file
    // reader trims them; files that settings still name resolve against
    // `directory` ("" = the current directory).
    Config(const std::vector<std::pair<std::string, std::string>>& settings, const std::string& directory);

    bool has(const std::string& key) const { return data_.count(key) > 0; }
    std::string get(const std::string& key) const;
    // Overrides one key (the server's FP64 re-run of a diverged float solve).
    void set(const std::string& key, const std::string& value) { data_[key] = value; }
    const std::string& directory() const { return dir_; }

    // typed getters, same names and defaults as the reference's Config
    double parseFloat(const std::string& key) const;
    double parseFloat(const std::string& key, double def) const;
    int parseInt(const std::string& key, int def) const;
    bool parseBool(const std::string& key, bool def) const;
    std::vector<std::string> parseList(const std::string& key) const;

    std::string gridFilePath() const;
    std::string boundaryConditionsFilePath() const;
    Topology getTopology() const;
    Scheme getAdvectionScheme() const;
    bool getMUSCLreconstruction() const { return parseBool("MUSCL_RECONSTRUCTION", false); }
    Limiter getFluxLimiter() const;
    int getRungeKuttaStages() const;  // 4 (RK41A) or 3 (RK31B)
    std::vector<double> getTimeIntegrationCoeffs() const;
    TimeStepMethod getTimeStepMethod() const;
    double getCFL() const;
    double getFixedTimeStep() const { return parseFloat("FIXED_TIME_STEP"); }
    long getMaxIterations() const { return static_cast<long>(parseFloat("N_ITERATIONS")); }
    int getResidualsDropConvergence() const { return parseInt("RESIDUALS_DROP_CONVERGENCE", 16); }
    bool isSimulationSteady() const { return parseBool("SIMULATION_IS_STEADY", true); }
    double getFluidGamma() const { return parseFloat("FLUID_GAMMA"); }
    double getFluidGasConstant() const { return parseFloat("FLUID_R_CONSTANT"); }
    double getInitMachNumber() const { return parseFloat("INIT_MACH_NUMBER"); }
    double getInitPressure() const { return parseFloat("INIT_PRESSURE"); }
    double getInitTemperature() const { return parseFloat("INIT_TEMPERATURE"); }
    bool isBFMActive() const { return parseBool("BFM_ACTIVE", false); }
    bool isBlockageActive() const { return parseBool("BLOCKAGE_ACTIVE", false); }
    BfmModel getBFMModel() const;
    bool isStalledBfmActive() const { return parseBool("STALLED_BFM_ACTIVE", false); }
    bool isPerturbationBodyForceActive() const { return parseBool("PERTURBATION_BODY_FORCE", false); }
    double getRotationalSpeedScalingFactor() const { return parseFloat("ROTATIONAL_SPEED_SCALING_FACTOR", 1.0); }
    bool isAccelerationActive() const { return parseBool("ACCELERATION_ACTIVE", false); }
    bool getHallTholletOffDesignActive() const;
    double getOutletPressureRampMaxIterations() const { return parseFloat("OUTLET_PRESSURE_RAMP_ITERATIONS", 0.0); }
    bool isInletCylindrical() const;
    bool enableGreitzerModeling() const;
    double getGreitzerPlenumVolume() const;
    double getGreitzerAmbientPressure() const { return parseFloat("GREITZER_AMBIENT_PRESSURE", 101325.0); }
    bool saveTurboOutput() const { return parseBool("TURBO_OUTPUT", false); }
    bool isViscosityActive() const { return parseBool("VISCOSITY_ACTIVE", false); }

private:
    std::map<std::string, std::string> data_;
    std::string dir_;
};

}  // namespace ctbfm
