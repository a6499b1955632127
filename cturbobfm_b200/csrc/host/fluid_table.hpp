// FluidTable: the real-gas look-up tables of FluidReal (include/fluid_real.hpp,
// src/fluid_real.cpp) on the host, read from the reference's .lut format, for
// the set-up work the reference does on the host (initial fields, the
// initial plenum and radial-profile states) and for the device copy.
#pragma once

#include <array>
#include <string>
#include <vector>

#include "../device/case.cuh"
#include "config.hpp"
#include "mesh.hpp"

namespace ctbfm {

// Table2D (include/fluid_real.hpp:11-58).
struct HostTable {
    long nx = 0, ny = 0;
    double xmin = 0, xmax = 0, ymin = 0, ymax = 0, dx = 1, dy = 1;
    std::vector<double> d;
    void init(long nx_, long ny_, double x0, double x1, double y0, double y1);
    double interpolate(double x, double y) const;
};

class FluidTable {
public:
    // FluidReal::loadTable (src/fluid_real.cpp:12-208); throws ConfigError
    // with the reference's message when the file cannot be opened.
    explicit FluidTable(const std::string& path);

    double gammaNominal() const { return gnom_; }
    double gasConstant() const { return R_; }
    const std::array<HostTable, 8>& rhoE() const { return re_; }
    const std::array<HostTable, 4>& pT() const { return pt_; }
    const std::array<HostTable, 3>& pS() const { return ps_; }

    // FluidBase / FluidReal evaluations used at set-up
    static double staticEnergy_u_et(const Vec3& u, double et) { return et - 0.5 * u.dot(u); }
    double pressure_rho_e(double rho, double e) const { return re_[kReP].interpolate(rho, e); }
    double temperature_rho_e(double rho, double e) const { return re_[kReT].interpolate(rho, e); }
    double soundSpeed_rho_e(double rho, double e) const { return re_[kReA].interpolate(rho, e); }
    double density_p_T(double p, double T) const { return pt_[kPtRho].interpolate(p, T); }
    double energy_p_T(double p, double T) const { return pt_[kPtE].interpolate(p, T); }
    double entropy_rho_e(double rho, double e) const { return re_[kReS].interpolate(rho, e); }
    double temperature_p_s(double p, double s) const { return ps_[kPsT].interpolate(p, s); }
    // FluidReal::computeStaticEnergy_p_rho (src/fluid_real.cpp:227-250)
    double staticEnergy_p_rho(double p, double rho) const;
    // FluidReal::computePressure_rho_T (src/fluid_real.cpp:262-277)
    double pressure_rho_T(double rho, double T) const;
    // FluidReal::computeTotalPressure_rho_u_et (src/fluid_real.cpp:299-321)
    // with e = e(u, et) already formed
    double totalPressure_rho_e_et(double rho, double e, double et) const;

private:
    std::array<HostTable, 8> re_;
    std::array<HostTable, 4> pt_;
    std::array<HostTable, 3> ps_;
    double molar_ = 0, R_ = 287.0, pcrit_ = 0, Tcrit_ = 0, rhocrit_ = 0, gnom_ = 1.3;
};

// Config::getFluidTableFile (src/config.cpp:492-497), resolved against the
// directory of the input file.
std::string fluidTablePath(const Config& config);

}  // namespace ctbfm
