// Solution output in the reference's volume CSV format (Output::writeHeader
// and Output::writeData, src/output.cpp:416-447): "NI=", "NJ=", "NK=" lines,
// a header "x,y,z,<fields>" with the fields in the order of the reference's
// std::map (sorted by name), then one row per node in (i, j, k) order with
// k fastest, every value printed with 16 significant digits. The fields are
// those of Output::allocateOutputArrays (src/output.cpp:82-132) for
// OUTPUT_FIELDS_TYPE primary (Density, Velocity X/Y/Z, Total Energy,
// Pressure, Temperature) or secondary (the default; adds Mach, Total
// Pressure, Total Temperature, Entropy), computed as
// Output::updatePrimaryFields / updateSecondaryFields do (:152-237).
// A file written here is a valid restart file for this library and for the
// reference.
#pragma once

#include <map>
#include <string>
#include <vector>

#include "config.hpp"
#include "host_fluid.hpp"
#include "mesh.hpp"

namespace ctbfm {

// Throws ConfigError for OUTPUT_FIELDS_TYPE = turbo_bfm on a body-force case
// (its force and deviation-angle fields are not kept by this library) and
// std::runtime_error when the file cannot be written. `extra` adds named
// node fields (the viscous fields of Output::updateViscousFields,
// src/output.cpp:240-306) to the sorted set.
void writeSolutionCsv(const std::string& path, const Config& config, const Mesh& mesh, const HostFluid& fluid,
                      const double* const U[5], const std::map<std::string, std::vector<double>>* extra = nullptr);

}  // namespace ctbfm
