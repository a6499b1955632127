// Restart: the initial state read from a solution file (RESTART_SOLUTION =
// yes), as Solver::initializeSolutionFromRestart does it
// (src/solver.cpp:890-966): the file is read by readRestartFile
// (src/solver.cpp:1155-1295), then mapped onto this grid by the standard
// (same dimensions, :968-1000), axisymmetric (same NI x NJ, any NK,
// :1002-1035) or nearest-neighbour (:1037-1153, a k-d tree over (x, r) or
// (x, y, z)) initialisation chosen by RESTART_TYPE and the dimensions. Host
// work at set-up, in FP64 with the reference's operation order.
#pragma once

#include <array>
#include <string>
#include <vector>

#include "config.hpp"
#include "host_fluid.hpp"
#include "mesh.hpp"

namespace ctbfm {

// Fields of a restart file, per node in (i, j, k) order with k fastest;
// coordinates stay (0, 0, 0) when the file has none, as in the reference.
struct RestartFile {
    long ni = 0, nj = 0, nk = 0;
    std::vector<Vec3> xyz;
    std::vector<double> rho, vx, vy, vz, T;
};

// Solver::readRestartFile (src/solver.cpp:1155-1295): three "NAME=value"
// lines (NI, NJ, NK), a header of column names, then one row per node.
// Temperature is computeTemperature_rho_u_et of the row. Throws ConfigError
// for an unreadable file, a missing primary column, a NaN or Inf value (with
// the reference's message) or a row count other than NI*NJ*NK.
RestartFile readRestartFile(const std::string& path, const HostFluid& fluid);

// The conservative initial state U[0..4] (nodes of `mesh`) from the restart
// file named by RESTART_SOLUTION_FILEPATH. `periodic` is whether the grid has
// a periodic patch (Mesh::isPeriodicityActive).
void restartState(const Config& config, const Mesh& mesh, Topology topo, bool periodic, const HostFluid& fluid,
                  std::array<std::vector<double>, 5>& U);

// RESTART_SOLUTION_FILEPATH, a relative path resolved against the directory
// of the input file like the grid and boundary files.
std::string restartPath(const Config& config);

}  // namespace ctbfm
