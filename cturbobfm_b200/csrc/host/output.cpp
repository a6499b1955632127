// Solution output: see output.hpp.
#include "output.hpp"

#include <cstdio>
#include <map>
#include <memory>
#include <stdexcept>
#include <vector>

namespace ctbfm {

void writeSolutionCsv(const std::string& path, const Config& config, const Mesh& mesh, const HostFluid& fluid,
                      const double* const U[5], const std::map<std::string, std::vector<double>>* extra) {
    // Config::getOutputFieldsType (src/config.cpp:629-647)
    const std::string t = config.has("OUTPUT_FIELDS_TYPE") ? config.get("OUTPUT_FIELDS_TYPE") : "None";
    // with a turbulence model the secondary fields are written whatever the
    // type (Output::updateOutputArrays, src/output.cpp:141-143)
    const bool primaryOnly = (t == "primary" || t == "Primary" || t == "PRIMARY") &&
                             !(config.parseBool("TURBULENCE_ACTIVE", false) && config.has("TURBULENCE_MODEL") &&
                               config.get("TURBULENCE_MODEL") == "SA");
    const bool turbo = t == "turbo_bfm" || t == "Turbo_bfm" || t == "TURBO_BFM";
    if (turbo && config.isBFMActive())
        throw ConfigError("OUTPUT_FIELDS_TYPE = turbo_bfm (body forces, deviation angle) is not written by this library");

    const long N = mesh.nodes();
    std::map<std::string, std::vector<double>> fields;
    for (const char* name : {"Density", "Velocity X", "Velocity Y", "Velocity Z", "Total Energy", "Pressure",
                             "Temperature"})
        fields[name].resize(static_cast<size_t>(N));
    if (!primaryOnly)
        for (const char* name : {"Mach", "Total Pressure", "Total Temperature", "Entropy"})
            fields[name].resize(static_cast<size_t>(N));
    auto& rho = fields["Density"];
    auto& vx = fields["Velocity X"];
    auto& vy = fields["Velocity Y"];
    auto& vz = fields["Velocity Z"];
    auto& et = fields["Total Energy"];
    auto& p = fields["Pressure"];
    auto& T = fields["Temperature"];
    for (long q = 0; q < N; q++) {
        rho[q] = U[0][q];
        vx[q] = U[1][q] / U[0][q];  // FlowSolution::getVelocityX (include/types.hpp:840-843)
        vy[q] = U[2][q] / U[0][q];
        vz[q] = U[3][q] / U[0][q];
        et[q] = U[4][q] / U[0][q];
        const Vec3 u(vx[q], vy[q], vz[q]);
        p[q] = fluid.pressure_rho_u_et(rho[q], u, et[q]);
        T[q] = fluid.temperature_rho_u_et(rho[q], u, et[q]);
    }
    if (!primaryOnly) {
        auto& M = fields["Mach"];
        auto& pt = fields["Total Pressure"];
        auto& Tt = fields["Total Temperature"];
        auto& s = fields["Entropy"];
        for (long q = 0; q < N; q++) {
            const Vec3 u(vx[q], vy[q], vz[q]);
            const double a = fluid.soundSpeed_rho_u_et(rho[q], u, et[q]);
            M[q] = u.magnitude() / a;
            pt[q] = fluid.totalPressure_rho_u_et(rho[q], u, et[q]);
            Tt[q] = fluid.totalTemperature_rho_u_et(rho[q], u, et[q]);
            s[q] = fluid.entropy_rho_u_et(rho[q], u, et[q]);
        }
    }

    if (extra)
        for (const auto& kv : *extra) fields[kv.first] = kv.second;

    std::unique_ptr<FILE, int (*)(FILE*)> f(std::fopen(path.c_str(), "w"), &std::fclose);
    if (!f) throw std::runtime_error("Failed to open file: " + path);
    std::fprintf(f.get(), "NI=%ld\nNJ=%ld\nNK=%ld\nx,y,z", mesh.ni(), mesh.nj(), mesh.nk());
    for (const auto& kv : fields) std::fprintf(f.get(), ",%s", kv.first.c_str());
    std::fputc('\n', f.get());
    const auto& V = mesh.vertices();
    for (long q = 0; q < N; q++) {
        std::fprintf(f.get(), "%.16g,%.16g,%.16g", V[q].x, V[q].y, V[q].z);
        for (const auto& kv : fields) std::fprintf(f.get(), ",%.16g", kv.second[q]);
        std::fputc('\n', f.get());
    }
    if (std::ferror(f.get())) throw std::runtime_error("Failed to write file: " + path);
}

}  // namespace ctbfm
