// Replacement for src/implicit_solver_krylov.cpp of the reference, which needs
// Eigen. The explicit Runge-Kutta path never constructs this class; selecting
// TIME_INTEGRATION_TYPE = 3 with this build throws.
#include "implicit_solver_krylov.hpp"
#include <stdexcept>

ImplicitSolverKrylov::ImplicitSolverKrylov(const Config& config, const Mesh& mesh,
                                           const FluidBase& fluid,
                                           const TurbulenceModelBase* turbModel)
    : ImplicitSolverBase(config, mesh, fluid, turbModel) {
    throw std::runtime_error("implicit Krylov solver is not part of this oracle build");
}

void ImplicitSolverKrylov::solveCorrection(const FlowSolution&, const FlowSolution&,
                                           const Matrix3D<FloatType>&, FlowSolution&) {
    throw std::runtime_error("implicit Krylov solver is not part of this oracle build");
}
