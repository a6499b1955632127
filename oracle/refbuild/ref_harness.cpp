// Test harness around the reference solver (CTurboBFM), compiled from the
// reference's own sources by refbuild/Makefile. It is test infrastructure: it gives
// the oracle restatement and the CUDA path a bit-exact target.
//
// Modes
//   ref_harness run      <input.ini> <out.bin>
//       Runs the unmodified Solver::solve() (src/solver.cpp:1296-1424) and dumps
//       the final conservative state at full precision.
//   ref_harness residual <input.ini> <out.bin>
//       Performs the first iteration's preamble and one residual evaluation
//       exactly as Solver::solve() does for it = 1 (src/solver.cpp:1337-1373)
//       and dumps the time-step array and the residual field.
//   ref_harness steps    <input.ini> <n_iter> <out.bin>
//       Calls the reference's own member functions in the order of the explicit
//       Runge-Kutta branch of Solver::solve() (src/solver.cpp:1337-1398) for at
//       most n_iter iterations (stopping on convergence like solve()), and
//       dumps the final state plus, per iteration, the log10 residual norms,
//       the six boundary mass flows, the turbo performance and the hub static
//       pressure at full precision. A NaN/Inf residual norm (the reference's
//       "Solver diverged" exception) ends the loop and is recorded as status 2.
//
// Binary format (little endian): int64 ni, nj, nk, mode-specific payload.

#include <algorithm>
#include <array>
#include <cassert>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <map>
#include <memory>
#include <numeric>
#include <sstream>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>

// Reach the Solver's private members and functions without touching the
// reference's files. Standard headers are already included above, so only the
// reference's own classes are affected.
#define private public
#define protected public
#include "solver.hpp"
#undef private
#undef protected

namespace {

void writeI64(std::ofstream& f, int64_t v) { f.write(reinterpret_cast<const char*>(&v), sizeof v); }
void writeF64(std::ofstream& f, double v) { f.write(reinterpret_cast<const char*>(&v), sizeof v); }
void writeArray(std::ofstream& f, const Matrix3D<FloatType>& m) {
    f.write(reinterpret_cast<const char*>(m.data()), sizeof(double) * m.totalSize());
}
void writeState(std::ofstream& f, const FlowSolution& s) {
    writeArray(f, s._rho);
    writeArray(f, s._rhoU);
    writeArray(f, s._rhoV);
    writeArray(f, s._rhoW);
    writeArray(f, s._rhoE);
}

bool needsTurboPerformance(const Solver& solver, const Config& config) {
    bool need = config.saveTurboOutput() || solver._isGreitzerModelingActive;
    for (const auto& bc : solver._boundaries) {
        if (bc.type == BoundaryType::THROTTLE || bc.type == BoundaryType::MASS_FLOW) need = true;
    }
    if (config.isBFMActive() && config.getBFMModel() == BodyForceModel::CHIMA) need = true;
    return need;
}

}  // namespace

int main(int argc, char** argv) {
    if (argc < 4) {
        std::cerr << "usage: ref_harness run|residual <input.ini> <out.bin>\n"
                     "       ref_harness steps <input.ini> <n_iter> <out.bin>\n";
        return 2;
    }
    const std::string mode = argv[1];
    try {
        Config config(argv[2]);
        Mesh mesh(config);
        Solver solver(config, mesh);
        const int64_t ni = solver._nPointsI, nj = solver._nPointsJ, nk = solver._nPointsK;

        if (mode == "run") {
            solver.solve();
            std::ofstream f(argv[3], std::ios::binary);
            writeI64(f, ni); writeI64(f, nj); writeI64(f, nk);
            writeState(f, solver._conservativeSolution);
            return 0;
        }

        if (mode == "residual") {
            Matrix3D<FloatType> timestep(ni, nj, nk);
            FlowSolution residuals(ni, nj, nk);
            const bool needTurbo = needsTurboPerformance(solver, config);
            solver.preprocessSolution(solver._conservativeSolution, false);
            FlowSolution solutionTmp(solver._conservativeSolution);
            auto gradTmp = solver._solutionGrad;
            solver.updateMassFlows(solutionTmp);
            if (needTurbo) solver.updateTurboPerformance(solutionTmp);
            solver.computeTimestepArray(solutionTmp, timestep);
            solver.preprocessSolution(solutionTmp);
            solver.computeSolutionGradient(solutionTmp, gradTmp);
            solver.computeResiduals(solutionTmp, gradTmp, 1, solver._currentTime, timestep, residuals);
            std::ofstream f(argv[3], std::ios::binary);
            writeI64(f, ni); writeI64(f, nj); writeI64(f, nk);
            writeArray(f, timestep);
            writeState(f, residuals);
            return 0;
        }

        if (mode == "steps") {
            if (argc < 5) { std::cerr << "steps needs n_iter and out.bin\n"; return 2; }
            const long nIter = std::stol(argv[3]);
            Matrix3D<FloatType> timestep(ni, nj, nk);
            FlowSolution residuals(ni, nj, nk);
            const std::vector<FloatType> coeffs = config.getTimeIntegrationCoeffs();
            const bool needTurbo = needsTurboPerformance(solver, config);
            bool exitLoop = false;
            bool diverged = false;
            bool steady = config.isSimulationSteady();

            solver.preprocessSolution(solver._conservativeSolution, false);
            FlowSolution solutionTmp(solver._conservativeSolution);
            auto gradTmp = solver._solutionGrad;

            std::vector<std::array<double, 5>> logres;
            std::vector<std::array<double, 6>> massflows;
            std::vector<std::array<double, 4>> turbo;
            std::vector<double> hubPressure;
            long it = 1;
            for (; it <= nIter; ++it) {
                solver.updateMassFlows(solutionTmp);
                if (needTurbo) solver.updateTurboPerformance(solutionTmp);
                solver.computeTimestepArray(solutionTmp, timestep);
                solver.preprocessSolution(solutionTmp);
                solver.computeSolutionGradient(solutionTmp, gradTmp);
                solver.updateTurbulenceSolution(solutionTmp, gradTmp, 1.0, timestep);
                for (const auto& alpha : coeffs) {
                    solver.computeSolutionGradient(solutionTmp, gradTmp);
                    solver.computeResiduals(solutionTmp, gradTmp, it, solver._currentTime, timestep, residuals);
                    solver.updateSolution(solver._conservativeSolution, solutionTmp, residuals, alpha, timestep);
                    solver.enforcePeriodicityOnSolution(solutionTmp);
                }
                solver._conservativeSolution = solutionTmp;
                solver._currentTime += timestep.min();
                StateVector lr;
                try {
                    lr = solver.computeLogResidualNorm(residuals);
                } catch (const std::runtime_error&) {
                    diverged = true;  // the reference's "Solver diverged" exception
                    break;
                }
                solver._logResiduals.push_back(lr);
                if (!solver._hasInitialLogResiduals) {
                    solver._initialLogResiduals = lr;
                    solver._hasInitialLogResiduals = true;
                } else if (it <= 5) {
                    for (size_t v = 0; v < 5; ++v)
                        solver._initialLogResiduals[v] = std::max(solver._initialLogResiduals[v], lr[v]);
                }
                logres.push_back({lr[0], lr[1], lr[2], lr[3], lr[4]});
                std::array<double, 6> mf{};
                const BoundaryIndex bi[6] = {BoundaryIndex::I_START, BoundaryIndex::I_END,
                                             BoundaryIndex::J_START, BoundaryIndex::J_END,
                                             BoundaryIndex::K_START, BoundaryIndex::K_END};
                for (int b = 0; b < 6; ++b) mf[b] = solver._massFlows[bi[b]];
                massflows.push_back(mf);
                std::array<double, 4> tp{0, 0, 0, 0};
                if (needTurbo) {
                    tp[0] = solver._turboPerformance[TurboPerformance::MASS_FLOW].back();
                    tp[1] = solver._turboPerformance[TurboPerformance::TOTAL_PRESSURE_RATIO].back();
                    tp[2] = solver._turboPerformance[TurboPerformance::TOTAL_TEMPERATURE_RATIO].back();
                    tp[3] = solver._turboPerformance[TurboPerformance::TOTAL_EFFICIENCY].back();
                }
                turbo.push_back(tp);
                hubPressure.push_back(solver._hubStaticPressure);
                solver.checkConvergence(exitLoop, steady, it);
                if (exitLoop && steady) break;
            }
            const long done = static_cast<long>(logres.size());
            std::ofstream f(argv[4], std::ios::binary);
            writeI64(f, ni); writeI64(f, nj); writeI64(f, nk);
            writeI64(f, done);
            writeI64(f, diverged ? 2 : ((exitLoop && steady) ? 1 : 0));
            writeF64(f, solver._currentTime);
            writeState(f, solver._conservativeSolution);
            for (const auto& r : logres) for (double v : r) writeF64(f, v);
            for (const auto& r : massflows) for (double v : r) writeF64(f, v);
            for (const auto& r : turbo) for (double v : r) writeF64(f, v);
            for (double v : hubPressure) writeF64(f, v);
            // the Spalart-Allmaras working variable, when the model is on
            if (config.isTurbulenceActive() && config.getTurbulenceModel() == TurbulenceModel::SPALART_ALLMARAS)
                for (size_t i = 0; i < ni; ++i)
                    for (size_t j = 0; j < nj; ++j)
                        for (size_t k = 0; k < nk; ++k) writeF64(f, solver._turbulenceModel->getWorkingVariable(i, j, k));
            return 0;
        }
        std::cerr << "unknown mode " << mode << "\n";
        return 2;
    } catch (const std::exception& e) {
        std::cerr << "ref_harness: " << e.what() << "\n";
        return 1;
    }
}
