// FluidTable: see fluid_table.hpp.
#include "fluid_table.hpp"

#include <cmath>
#include <cstdlib>
#include <fstream>
#include <sstream>

namespace ctbfm {

void HostTable::init(long nx_, long ny_, double x0, double x1, double y0, double y1) {
    nx = nx_;
    ny = ny_;
    xmin = x0;
    xmax = x1;
    ymin = y0;
    ymax = y1;
    dx = (nx > 1) ? (xmax - xmin) / static_cast<double>(nx - 1) : 1.0;
    dy = (ny > 1) ? (ymax - ymin) / static_cast<double>(ny - 1) : 1.0;
    d.assign(static_cast<size_t>(nx * ny), 0.0);
}

double HostTable::interpolate(double x, double y) const {
    const double xc = (x < xmin) ? xmin : ((xmax < x) ? xmax : x);
    const double yc = (y < ymin) ? ymin : ((ymax < y) ? ymax : y);
    const double rx = (xc - xmin) / dx;
    const double ry = (yc - ymin) / dy;
    // size_t conversion; a NaN coordinate lands on the last cell (NaN result)
    size_t i = (rx >= 0.0 && rx < 1e18) ? static_cast<size_t>(rx) : static_cast<size_t>(nx);
    size_t j = (ry >= 0.0 && ry < 1e18) ? static_cast<size_t>(ry) : static_cast<size_t>(ny);
    if (i >= static_cast<size_t>(nx - 1)) i = (nx >= 2) ? static_cast<size_t>(nx - 2) : 0;
    if (j >= static_cast<size_t>(ny - 1)) j = (ny >= 2) ? static_cast<size_t>(ny - 2) : 0;
    const double wx = rx - static_cast<double>(i);
    const double wy = ry - static_cast<double>(j);
    const double f00 = d[i * ny + j];
    const double f10 = d[(i + 1) * ny + j];
    const double f01 = d[i * ny + (j + 1)];
    const double f11 = d[(i + 1) * ny + (j + 1)];
    return (1.0 - wx) * (1.0 - wy) * f00 + wx * (1.0 - wy) * f10 + (1.0 - wx) * wy * f01 + wx * wy * f11;
}

namespace {
void trimRight(std::string& s) { s.erase(s.find_last_not_of(" \t\r\n") + 1); }
void trimLeft(std::string& s) {
    const size_t p = s.find_first_not_of(" \t\r\n");
    s.erase(0, p == std::string::npos ? s.size() : p);
}
bool keyVal(const std::string& line, std::string& key, std::string& val) {
    const size_t c = line.find(':');
    if (c == std::string::npos) return false;
    key = line.substr(0, c);
    val = line.substr(c + 1);
    trimRight(key);
    trimLeft(val);
    return true;
}
// the next data line (empty, '#' and '\r' lines skipped), parsed as n numbers
bool dataRow(std::ifstream& f, std::string& line, double* v, int n) {
    if (!std::getline(f, line)) return false;
    while (line.empty() || line[0] == '#' || line[0] == '\r')
        if (!std::getline(f, line)) break;
    std::istringstream iss(line);
    for (int q = 0; q < n; q++) {
        v[q] = 0.0;
        iss >> v[q];
    }
    return true;
}
}  // namespace

FluidTable::FluidTable(const std::string& path) {
    std::ifstream f(path);
    if (!f.is_open()) throw ConfigError("FluidReal: Could not open table file at: " + path);
    std::string line, key, val;
    int sec = 0;  // 1 RHO_E, 2 P_T, 3 P_S
    long n1 = 0, n2 = 0;
    double x0 = 0, x1 = 0, y0 = 0, y1 = 0;
    while (std::getline(f, line)) {
        if (line.empty() || line[0] == '\r') continue;
        if (line.find("# SECTION: RHO_E") != std::string::npos) { sec = 1; continue; }
        if (line.find("# SECTION: P_T") != std::string::npos) { sec = 2; continue; }
        if (line.find("# SECTION: P_S") != std::string::npos) { sec = 3; continue; }
        if (line[0] == '#') continue;
        if (!keyVal(line, key, val)) continue;
        if (sec == 0) {
            if (key == "MOLAR_MASS") molar_ = std::stod(val);
            else if (key == "GAS_CONSTANT") R_ = std::stod(val);
            else if (key == "CRITICAL_PRESSURE") pcrit_ = std::stod(val);
            else if (key == "CRITICAL_TEMPERATURE") Tcrit_ = std::stod(val);
            else if (key == "CRITICAL_DENSITY") rhocrit_ = std::stod(val);
            else if (key == "NOMINAL_GAMMA") gnom_ = std::stod(val);
            continue;
        }
        const char* kn1 = sec == 1 ? "N_RHO" : "N_P";
        const char* kn2 = sec == 1 ? "N_E" : (sec == 2 ? "N_T" : "N_S");
        const char* kx0 = sec == 1 ? "RHO_MIN" : "P_MIN";
        const char* kx1 = sec == 1 ? "RHO_MAX" : "P_MAX";
        const char* ky0 = sec == 1 ? "E_MIN" : (sec == 2 ? "T_MIN" : "S_MIN");
        const char* ky1 = sec == 1 ? "E_MAX" : (sec == 2 ? "T_MAX" : "S_MAX");
        if (key == kn1) n1 = static_cast<long>(std::stoul(val));
        else if (key == kn2) n2 = static_cast<long>(std::stoul(val));
        else if (key == kx0) x0 = std::stod(val);
        else if (key == kx1) x1 = std::stod(val);
        else if (key == ky0) y0 = std::stod(val);
        else if (key == ky1) {
            y1 = std::stod(val);
            std::vector<HostTable*> t;
            if (sec == 1) for (auto& h : re_) t.push_back(&h);
            else if (sec == 2) for (auto& h : pt_) t.push_back(&h);
            else for (auto& h : ps_) t.push_back(&h);
            for (HostTable* h : t) h->init(n1, n2, x0, x1, y0, y1);
            double v[8];
            bool more = true;
            for (long i = 0; i < n1 && more; i++)
                for (long j = 0; j < n2; j++) {
                    if (!dataRow(f, line, v, static_cast<int>(t.size()))) {
                        more = false;
                        break;
                    }
                    for (size_t q = 0; q < t.size(); q++) t[q]->d[static_cast<size_t>(i * n2 + j)] = v[q];
                }
        }
    }
    for (const auto* tabs : {&re_[0], &pt_[0], &ps_[0]})
        if (tabs->nx < 2 || tabs->ny < 2) throw ConfigError("FluidReal: table " + path + " lacks a section");
}

double FluidTable::staticEnergy_p_rho(double p, double rho) const {
    const HostTable& tp = re_[kReP];
    double eLo = tp.ymin, eHi = tp.ymax;
    const double pLo = tp.interpolate(rho, eLo);
    const double pHi = tp.interpolate(rho, eHi);
    if (p <= pLo) return eLo;
    if (p >= pHi) return eHi;
    for (int it = 0; it < 30; ++it) {
        const double eMid = 0.5 * (eLo + eHi);
        const double pMid = tp.interpolate(rho, eMid);
        if (std::abs(pMid - p) <= 1e-4 * p) return eMid;
        if (pMid < p) eLo = eMid;
        else eHi = eMid;
    }
    return 0.5 * (eLo + eHi);
}

double FluidTable::pressure_rho_T(double rho, double T) const {
    const HostTable& tT = re_[kReT];
    double eLo = tT.ymin, eHi = tT.ymax;
    for (int it = 0; it < 25; ++it) {
        const double eMid = 0.5 * (eLo + eHi);
        if (tT.interpolate(rho, eMid) < T) eLo = eMid;
        else eHi = eMid;
    }
    return pressure_rho_e(rho, 0.5 * (eLo + eHi));
}

double FluidTable::totalPressure_rho_e_et(double rho, double e, double et) const {
    const double p = pressure_rho_e(rho, e);
    const double s = entropy_rho_e(rho, e);
    const double ht = et + p / rho;
    double pLo = p, pHi = ps_[kPsRho].xmax;
    for (int it = 0; it < 25; ++it) {
        const double pMid = 0.5 * (pLo + pHi);
        const double rhoMid = ps_[kPsRho].interpolate(pMid, s);
        const double eMid = ps_[kPsE].interpolate(pMid, s);
        const double hMid = eMid + pMid / rhoMid;
        if (hMid < ht) pLo = pMid;
        else pHi = pMid;
    }
    return 0.5 * (pLo + pHi);
}

std::string fluidTablePath(const Config& config) {
    std::string name = config.has("FLUID_NAME") ? config.get("FLUID_NAME")
                                                : (config.has("FLUID") ? config.get("FLUID") : std::string("CO2"));
    std::string file = config.has("FLUID_TABLE_FILE") ? config.get("FLUID_TABLE_FILE") : "fluid_table_" + name + ".lut";
    if (!file.empty() && file[0] == '/') return file;
    return config.directory().empty() ? file : config.directory() + "/" + file;
}

}  // namespace ctbfm
