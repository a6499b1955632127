// HostFluid: the fluid evaluations the host does outside the iteration loop
// (restart initialisation and solution output), for the ideal gas of
// FluidIdeal (src/fluid_ideal.cpp) and the look-up tables of FluidReal with
// the FluidBase defaults it inherits (src/fluid_real.cpp,
// include/fluid_base.hpp). Every expression keeps the reference's evaluation
// order; the host sources are compiled with -ffp-contract=off.
#pragma once

#include <cmath>
#include <memory>

#include "fluid_table.hpp"
#include "mesh.hpp"

namespace ctbfm {

class HostFluid {
public:
    virtual ~HostFluid() = default;
    virtual double pressure_rho_u_et(double rho, const Vec3& u, double et) const = 0;
    virtual double temperature_rho_u_et(double rho, const Vec3& u, double et) const = 0;
    virtual double pressure_rho_T(double rho, double T) const = 0;
    virtual double staticEnergy_p_rho(double p, double rho) const = 0;
    virtual double soundSpeed_rho_u_et(double rho, const Vec3& u, double et) const = 0;
    virtual double totalPressure_rho_u_et(double rho, const Vec3& u, double et) const = 0;
    virtual double totalTemperature_rho_u_et(double rho, const Vec3& u, double et) const = 0;
    virtual double entropy_rho_u_et(double rho, const Vec3& u, double et) const = 0;
    // FluidIdeal::computeMachNumber_rho_u_et (src/fluid_ideal.cpp:138-142),
    // FluidBase::computeMachNumber_rho_u_et (include/fluid_base.hpp:111-114)
    double mach_rho_u_et(double rho, const Vec3& u, double et) const {
        const double a = soundSpeed_rho_u_et(rho, u, et);
        return u.magnitude() / a;
    }
};

// FluidIdeal (src/fluid_ideal.cpp).
class IdealFluid final : public HostFluid {
public:
    IdealFluid(double gamma, double R) : g_(gamma), R_(R), cp_((gamma * R) / (gamma - 1)) {}
    // computeStaticEnergy_u_et (:74-77): et - 0.5 * pow(|u|, 2)
    double staticEnergy(const Vec3& u, double et) const {
        const double m = u.magnitude();
        return et - 0.5 * (m * m);
    }
    double pressure_rho_e(double rho, double e) const { return (g_ - 1) * rho * e; }  // :14-16
    double pressure_rho_u_et(double rho, const Vec3& u, double et) const override {  // :89-92
        return pressure_rho_e(rho, staticEnergy(u, et));
    }
    double temperature_rho_u_et(double rho, const Vec3& u, double et) const override {  // :106-109
        const double p = pressure_rho_u_et(rho, u, et);
        return p / (rho * R_);
    }
    double pressure_rho_T(double rho, double T) const override { return rho * R_ * T; }  // :66-68
    double staticEnergy_p_rho(double p, double rho) const override { return p / ((g_ - 1) * rho); }  // :10-12
    double soundSpeed_rho_u_et(double rho, const Vec3& u, double et) const override {  // :83-87, :70-72
        const double p = pressure_rho_u_et(rho, u, et);
        return std::sqrt(g_ * p / rho);
    }
    double totalPressure_rho_u_et(double rho, const Vec3& u, double et) const override {  // :94-98
        const double p = pressure_rho_u_et(rho, u, et);
        const double M = mach_rho_u_et(rho, u, et);
        return p * std::pow(1.0 + (g_ - 1.0) / 2.0 * M * M, g_ / (g_ - 1));
    }
    double totalTemperature_rho_u_et(double rho, const Vec3& u, double et) const override {  // :100-104
        const double T = temperature_rho_u_et(rho, u, et);
        const double M = mach_rho_u_et(rho, u, et);
        return T * (1.0 + (g_ - 1.0) / 2.0 * M * M);
    }
    double entropy_rho_u_et(double rho, const Vec3& u, double et) const override {  // :125-132, :193-196
        const double p = pressure_rho_u_et(rho, u, et);
        const double T = temperature_rho_u_et(rho, u, et);
        return cp_ * std::log(T / 288.15) - R_ * std::log(p / 101325);
    }

private:
    double g_, R_, cp_;
};

// FluidReal (src/fluid_real.cpp:211-328) over a loaded FluidTable.
class RealFluid final : public HostFluid {
public:
    explicit RealFluid(const FluidTable& t) : t_(t) {}
    double pressure_rho_u_et(double rho, const Vec3& u, double et) const override {
        return t_.pressure_rho_e(rho, FluidTable::staticEnergy_u_et(u, et));
    }
    double temperature_rho_u_et(double rho, const Vec3& u, double et) const override {
        return t_.temperature_rho_e(rho, FluidTable::staticEnergy_u_et(u, et));
    }
    double pressure_rho_T(double rho, double T) const override { return t_.pressure_rho_T(rho, T); }
    double staticEnergy_p_rho(double p, double rho) const override { return t_.staticEnergy_p_rho(p, rho); }
    double soundSpeed_rho_u_et(double rho, const Vec3& u, double et) const override {
        return t_.soundSpeed_rho_e(rho, FluidTable::staticEnergy_u_et(u, et));
    }
    double totalPressure_rho_u_et(double rho, const Vec3& u, double et) const override {
        return t_.totalPressure_rho_e_et(rho, FluidTable::staticEnergy_u_et(u, et), et);
    }
    double totalTemperature_rho_u_et(double rho, const Vec3& u, double et) const override {  // :323-328
        const double pt = totalPressure_rho_u_et(rho, u, et);
        const double e = FluidTable::staticEnergy_u_et(u, et);
        const double s = t_.entropy_rho_e(rho, e);
        return t_.temperature_p_s(pt, s);
    }
    double entropy_rho_u_et(double rho, const Vec3& u, double et) const override {
        return t_.entropy_rho_e(rho, FluidTable::staticEnergy_u_et(u, et));
    }

private:
    const FluidTable& t_;
};

}  // namespace ctbfm
