// Config: see config.hpp. Parsing rules follow src/config.cpp of the reference.
#include "config.hpp"

#include <algorithm>
#include <cctype>
#include <fstream>
#include <sstream>

namespace ctbfm {

namespace {

std::string trim(const std::string& s, const char* ws) {
    const size_t a = s.find_first_not_of(ws);
    if (a == std::string::npos) return "";
    const size_t b = s.find_last_not_of(ws);
    return s.substr(a, b - a + 1);
}

std::string lower(std::string s) {
    std::transform(s.begin(), s.end(), s.begin(), [](unsigned char c) { return std::tolower(c); });
    return s;
}

}  // namespace

// Config::load (src/config.cpp:15-44).
Config::Config(const std::string& path) {
    std::ifstream file(path);
    if (!file.is_open()) throw ConfigError("Failed to load configuration file: " + path);
    const size_t slash = path.find_last_of('/');
    dir_ = (slash == std::string::npos) ? "." : path.substr(0, slash);
    std::string line;
    while (std::getline(file, line)) {
        line = trim(line, " \t\r\n");
        if (line.empty() || line[0] == ';' || line[0] == '[') continue;
        const size_t eq = line.find('=');
        if (eq == std::string::npos) continue;
        data_[trim(line.substr(0, eq), " \t")] = trim(line.substr(eq + 1), " \t");
    }
}

Config::Config(const std::vector<std::pair<std::string, std::string>>& settings, const std::string& directory)
    : dir_(directory) {
    for (const auto& kv : settings) {
        const std::string key = trim(kv.first, " \t\r\n");
        if (key.empty()) throw ConfigError("empty setting key");
        data_[key] = trim(kv.second, " \t\r\n");
    }
}

std::string Config::get(const std::string& key) const {
    auto it = data_.find(key);
    return it == data_.end() ? std::string() : it->second;
}

double Config::parseFloat(const std::string& key) const {
    if (!has(key)) throw ConfigError("Not found value for key \"" + key + "\" in configuration.");
    try {
        return std::stod(get(key));
    } catch (const std::exception&) {
        throw ConfigError("Invalid float format for key \"" + key + "\": \"" + get(key) + "\"");
    }
}

double Config::parseFloat(const std::string& key, double def) const {
    return has(key) ? parseFloat(key) : def;
}

int Config::parseInt(const std::string& key, int def) const {
    return has(key) ? static_cast<int>(parseFloat(key)) : def;
}

// Config::parseBool (src/config.cpp:141-159).
bool Config::parseBool(const std::string& key, bool def) const {
    if (!has(key)) return def;
    const std::string v = lower(get(key));
    if (v == "true" || v == "yes" || v == "1") return true;
    if (v == "false" || v == "no" || v == "0") return false;
    throw ConfigError("Invalid value for key \"" + key + "\" in configuration.");
}

// Config::parseVector<std::string> (include/config.hpp:29-51).
std::vector<std::string> Config::parseList(const std::string& key) const {
    if (!has(key)) throw ConfigError("Missing value for key \"" + key + "\" in configuration.");
    std::vector<std::string> out;
    std::stringstream ss(get(key));
    std::string item;
    while (std::getline(ss, item, ',')) {
        item = trim(item, " \t\r\n");
        if (!item.empty()) out.push_back(item);
    }
    return out;
}

std::string Config::gridFilePath() const {
    if (!has("GRID_FILE")) throw ConfigError("Not found value for key \"GRID_FILE\" in configuration.");
    return get("GRID_FILE");
}

std::string Config::boundaryConditionsFilePath() const {
    if (!has("BOUNDARY_CONDITIONS_FILEPATH"))
        throw ConfigError("Not found value for key \"BOUNDARY_CONDITIONS_FILEPATH\" in configuration.");
    return get("BOUNDARY_CONDITIONS_FILEPATH");
}

// Config::getTopology (src/config.cpp:232-248).
Topology Config::getTopology() const {
    if (!has("TOPOLOGY")) throw ConfigError("Not found value for key \"TOPOLOGY\" in configuration.");
    const std::string v = get("TOPOLOGY");
    if (v == "2D" || v == "2d") return Topology::TwoD;
    if (v == "3D" || v == "3d") return Topology::ThreeD;
    if (v == "axisymmetric" || v == "Axisymmetric" || v == "AXISYMMETRIC") return Topology::Axisymmetric;
    if (v == "1D" || v == "1d") return Topology::OneD;
    throw ConfigError("Invalid value for key \"TOPOLOGY\" in configuration.");
}

// Config::getAdvectionScheme (src/config.cpp:371-384).
Scheme Config::getAdvectionScheme() const {
    if (!has("CONVECTION_SCHEME")) throw ConfigError("Not found value for key \"CONVECTION_SCHEME\" in configuration.");
    const std::string v = get("CONVECTION_SCHEME");
    if (v == "JST") return Scheme::JST;
    if (v == "ROE" || v == "roe" || v == "Roe") return Scheme::Roe;
    throw ConfigError("Invalid value for key \"CONVECTION_SCHEME\" in configuration.");
}

// Config::getFluxLimiter (src/config.cpp:453-466); note the spaces in the names.
Limiter Config::getFluxLimiter() const {
    const std::string v = has("FLUX_LIMITER") ? get("FLUX_LIMITER") : "None";
    if (v == "None") return Limiter::None;
    if (v == "van albada") return Limiter::VanAlbada;
    if (v == "van leer") return Limiter::VanLeer;
    if (v == "min mod") return Limiter::MinMod;
    throw ConfigError("Invalid value for key \"FLUX_LIMITER\" in configuration.");
}

// Config::getTimeIntegration (src/config.cpp:250-276), explicit branches only.
int Config::getRungeKuttaStages() const {
    const std::string key = has("TIME_INTEGRATION") ? "TIME_INTEGRATION" : "TIME_INTEGRATION_TYPE";
    if (!has(key)) return 4;
    std::string s;
    for (char c : get(key))
        if (!std::isspace(static_cast<unsigned char>(c))) s.push_back(static_cast<char>(std::tolower(static_cast<unsigned char>(c))));
    if (s == "0" || s == "explicit_rk4" || s == "rk4" || s == "runge_kutta_4") return 4;
    if (s == "1" || s == "explicit_rk3" || s == "rk3" || s == "runge_kutta_3") return 3;
    if (s == "2" || s == "implicit_lu_sgs" || s == "lu_sgs" || s == "lusgs" || s == "3" ||
        s == "implicit_krylov" || s == "krylov" || s == "bicgstab" || s == "implicit_gmres" ||
        s == "gmres" || s == "implicit_fgmres" || s == "fgmres")
        throw ConfigError("Implicit time integration is outside this library's explicit Runge-Kutta path");
    throw ConfigError("Invalid value for TimeIntegration: \"" + get(key) + "\".");
}

// Config::getTimeIntegrationCoeffs (src/config.cpp:400-411).
std::vector<double> Config::getTimeIntegrationCoeffs() const {
    if (getRungeKuttaStages() == 4) return {1.0 / 4.0, 5.0 / 14.0, 14.0 / 25.0, 1.0};
    return {8.0 / 17.0, 17.0 / 20.0, 1.0};
}

// Config::getTimeStepMethod (src/config.cpp:351-369).
TimeStepMethod Config::getTimeStepMethod() const {
    if (!has("TIME_STEP_METHOD")) throw ConfigError("Not found value for key \"TIME_STEP_METHOD\" in configuration.");
    const std::string v = get("TIME_STEP_METHOD");
    if (v == "local") return TimeStepMethod::Local;
    if (v == "global") return TimeStepMethod::Global;
    if (v == "fixed") return TimeStepMethod::Fixed;
    throw ConfigError("Invalid value for key \"TIME_STEP_METHOD\" in configuration.");
}

// Config::getCFL (include/config.hpp:124-133).
double Config::getCFL() const {
    if (has("CFL")) return parseFloat("CFL");
    if (has("CFL_START")) return parseFloat("CFL_START");
    if (has("CFL_MAX")) return parseFloat("CFL_MAX");
    return parseFloat("CFL");
}

// Config::getBFMModel (src/config.cpp:170-190).
BfmModel Config::getBFMModel() const {
    const std::string v = has("BFM_MODEL") ? get("BFM_MODEL") : "None";
    if (v == "Hall-Thollet") return BfmModel::HallThollet;
    if (v == "Hall") return BfmModel::Hall;
    if (v == "None") return BfmModel::None;
    if (v == "Blockage") return BfmModel::Blockage;
    if (v == "Lift-Drag") return BfmModel::LiftDrag;
    if (v == "Chima") return BfmModel::Chima;
    if (v == "Correlations") return BfmModel::Correlations;
    throw ConfigError("Invalid value for key \"BFM_MODEL\" in configuration.");
}

// Config::getHallTholletOffDesignActive (src/config.cpp:441-450): a required key.
bool Config::getHallTholletOffDesignActive() const {
    if (!has("HALL_THOLLET_OFF_DESIGN_ACTIVE"))
        throw ConfigError("Not found value for key \"HALL_THOLLET_OFF_DESIGN_ACTIVE\" in configuration.");
    const std::string v = get("HALL_THOLLET_OFF_DESIGN_ACTIVE");
    if (v == "true" || v == "yes" || v == "1") return true;
    if (v == "false" || v == "no" || v == "0") return false;
    throw ConfigError("Invalid value for key \"HALL_THOLLET_OFF_DESIGN_ACTIVE\" in configuration.");
}

// Config::getInletReferenceFrame (src/config.cpp:604-617).
bool Config::isInletCylindrical() const {
    const std::string v = has("INLET_REFERENCE_FRAME") ? get("INLET_REFERENCE_FRAME") : "None";
    if (v == "Cartesian" || v == "cartesian" || v == "CARTESIAN" || v == "None") return false;
    if (v == "Cylindrical" || v == "cylindrical" || v == "CYLINDRICAL") return true;
    throw ConfigError("Invalid value for key \"INLET_REFERENCE_FRAME\" in configuration.");
}

// Config::enableGreitzerModeling (src/config.cpp:684-693).
bool Config::enableGreitzerModeling() const {
    const bool on = parseBool("ENABLE_GREITZER_MODELING", false);
    if (on && getTimeStepMethod() != TimeStepMethod::Fixed)
        throw ConfigError("Greitzer modeling is only compatible with fixed time step method");
    return on;
}

// Config::getGreitzerPlenumVolume (include/config.hpp:354-356), with the
// reference's misspelled alias.
double Config::getGreitzerPlenumVolume() const {
    return has("GREITZER_PLENUM_VOLUME") ? parseFloat("GREITZER_PLENUM_VOLUME") : parseFloat("GREITZER_PENUM_VOLUME");
}

}  // namespace ctbfm
