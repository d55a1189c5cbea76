#pragma once
/**
 * @file Suite.hpp
 * @brief The reference's multiple-run mode (dimension continuation):
 *
 *  - SimulationSuite              (reference include/SimulationConfig.hpp:198-323)
 *  - fit_quadratic_least_squares  (reference src/common.cpp:151-198)
 *  - the seeding policy and loop  (reference src/main.cpp:245-378)
 *
 * The reference solves the dimensions of a suite one after the other, each
 * seeded from the converged ones before it.  Here every suite still steps
 * through its dimensions in order, but several suites (for example an
 * ascending and a descending branch from D = 4) step in lockstep: round r
 * solves dimension r of every suite that has one, and those Newton solves
 * share their batch launches (NewtonSolver::runBatched).  A suite's results
 * do not depend on what it runs beside.
 */
#include "Solver.hpp"

struct SimulationSuite {
    json multiInputDict;                     ///< the whole multi-dimension dictionary
    std::vector<std::string> simulationDims; ///< ordered keys to run

    /// Loads the suite file and orders its keys exactly as the reference does:
    /// ascending when reversed, else descending; unless ignoreConverged, the
    /// converged keys are skipped except for up to three of them prepended as
    /// seeds.
    SimulationSuite(const std::string& filePath, bool reversed = false, bool ignoreConverged = false);

    SimulationConfig generateSimulation(const std::string& simDimIn) const;
};

/// y = a x^2 + b x + c through three points, coefficients {a, b, c}, by the
/// Householder QR least-squares solve LAPACK dgels performs on the 3x3
/// design matrix [x^2 x 1].
vec_real fit_quadratic_least_squares(const vec_real& x_vals, const vec_real& y_vals);

/// Initial data of dimension i of a suite (main.cpp:275-354): i = 0 needs its
/// own data; i = 1, 2 borrow the previous converged solution; i >= 3
/// extrapolate quadratically in D from the previous three converged ones.
/// Entries that already hold data keep it.
void seedSuiteEntry(const SimulationSuite& suite, size_t i, SimulationConfig& config);

/// Runs the suites in lockstep (see the file comment).  After every round each
/// suite's dictionary is written back to its path, as the reference writes
/// its file after every dimension.  A suite whose dimension fails stops there
/// (the reference exits; here the other suites go on) and the failure is
/// returned; the result is empty when every suite finished.
std::string runSuites(std::vector<SimulationSuite>& suites, const std::vector<std::string>& paths,
                      bool ignoreConverged, const std::filesystem::path& dataPath);
