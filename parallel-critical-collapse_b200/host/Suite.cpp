// Suite.cpp -- dimension continuation (see Suite.hpp).
#include "Suite.hpp"

#include <algorithm>
#include <cmath>

SimulationSuite::SimulationSuite(const std::string& filePath, bool reversed, bool ignoreConverged)
{
    if (!std::filesystem::exists(filePath))
        throw std::filesystem::filesystem_error("File does not exist!", filePath,
                                                std::make_error_code(std::errc::no_such_file_or_directory));
    std::ifstream in(filePath);
    in >> multiInputDict;
    std::vector<std::string> convergedDims;
    for (const auto& dim : multiInputDict.items()) {
        if (!ignoreConverged && dim.value()["Converged"].get<bool>())
            convergedDims.push_back(dim.key());
        else
            simulationDims.push_back(dim.key());
    }
    auto asc = [](const std::string& a, const std::string& b) { return a < b; };
    auto desc = [](const std::string& a, const std::string& b) { return a > b; };
    if (reversed)
        std::sort(simulationDims.begin(), simulationDims.end(), asc);
    else
        std::sort(simulationDims.begin(), simulationDims.end(), desc);
    if (!ignoreConverged && !convergedDims.empty()) {
        // up to the last three converged keys, in the same order, as seeds
        if (reversed)
            std::sort(convergedDims.begin(), convergedDims.end(), asc);
        else
            std::sort(convergedDims.begin(), convergedDims.end(), desc);
        const size_t k = std::min<size_t>(3, convergedDims.size());
        simulationDims.insert(simulationDims.begin(), convergedDims.end() - k, convergedDims.end());
    }
}

SimulationConfig SimulationSuite::generateSimulation(const std::string& simDimIn) const
{
    if (!multiInputDict.contains(simDimIn))
        throw std::out_of_range("Simulation key '" + simDimIn + "' not found in input dictionary.");
    return SimulationConfig(multiInputDict[simDimIn]);
}

vec_real fit_quadratic_least_squares(const vec_real& x_vals, const vec_real& y_vals)
{
    // A = [x^2 x 1] (row-major 3x3), b = y.  Householder QR column by column
    // (dgeqrf's reflectors H = I - tau v v^T, v[0] = 1, beta = -sign(alpha) ||x||),
    // b <- Q^T b, then back substitution with R.
    double A[3][3], b[3];
    for (int i = 0; i < 3; ++i) {
        A[i][0] = x_vals[i] * x_vals[i];
        A[i][1] = x_vals[i];
        A[i][2] = 1.0;
        b[i] = y_vals[i];
    }
    for (int k = 0; k < 3; ++k) {
        double xnorm = 0.0;
        for (int i = k + 1; i < 3; ++i) xnorm = std::hypot(xnorm, A[i][k]);
        const double alpha = A[k][k];
        if (xnorm == 0.0) continue;  // H = I
        const double beta = -std::copysign(std::hypot(alpha, xnorm), alpha);
        const double tau = (beta - alpha) / beta;
        const double scal = 1.0 / (alpha - beta);
        double v[3] = {0.0, 0.0, 0.0};
        v[k] = 1.0;
        for (int i = k + 1; i < 3; ++i) v[i] = A[i][k] * scal;
        // apply H to the remaining columns and to b
        for (int j = k + 1; j < 3; ++j) {
            double s = 0.0;
            for (int i = k; i < 3; ++i) s += v[i] * A[i][j];
            s *= tau;
            for (int i = k; i < 3; ++i) A[i][j] -= s * v[i];
        }
        double s = 0.0;
        for (int i = k; i < 3; ++i) s += v[i] * b[i];
        s *= tau;
        for (int i = k; i < 3; ++i) b[i] -= s * v[i];
        A[k][k] = beta;
        for (int i = k + 1; i < 3; ++i) A[i][k] = 0.0;
    }
    for (int i = 2; i >= 0; --i) {
        if (A[i][i] == 0.0) throw std::runtime_error("LAPACKE_dgels failed with info = " + std::to_string(i + 1));
        double s = b[i];
        for (int j = i + 1; j < 3; ++j) s -= A[i][j] * b[j];
        b[i] = s / A[i][i];
    }
    return {b[0], b[1], b[2]};
}

void seedSuiteEntry(const SimulationSuite& suite, size_t i, SimulationConfig& config)
{
    const bool empty = config.fc.empty() || config.Up.empty() || config.psic.empty();
    if (!empty) return;
    const std::string& simDim = suite.simulationDims[i];
    if (i == 0)
        throw std::runtime_error("No converged solution as initial conditions available for " + simDim + "!");
    if (i < 3) {
        const std::string prevDim = suite.simulationDims[i - 1];
        SimulationConfig prev = suite.generateSimulation(prevDim);
        if (!prev.Converged)
            throw std::runtime_error("Previous dimension " + prevDim +
                                     " is not converged, hence no initial data for next simulation!");
        config.Delta = prev.Delta;
        config.fc = prev.fc;
        config.Up = prev.Up;
        config.psic = prev.psic;
        return;
    }
    const SimulationConfig p1 = suite.generateSimulation(suite.simulationDims[i - 1]);
    const SimulationConfig p2 = suite.generateSimulation(suite.simulationDims[i - 2]);
    const SimulationConfig p3 = suite.generateSimulation(suite.simulationDims[i - 3]);
    if (!p1.Converged || !p2.Converged || !p3.Converged)
        throw std::runtime_error("Previous dimensions not converged, hence no initial data for next simulation!");
    const vec_real dims = {std::stod(suite.simulationDims[i - 1]), std::stod(suite.simulationDims[i - 2]),
                           std::stod(suite.simulationDims[i - 3])};
    const real_t d = std::stod(simDim);
    const size_t n = p1.fc.size();
    vec_real fc(n, 0.0), Up(n, 0.0), psic(n, 0.0);
    for (size_t j = 0; j < n; ++j) {
        const vec_real cf = fit_quadratic_least_squares(dims, {p1.fc[j], p2.fc[j], p3.fc[j]});
        const vec_real cu = fit_quadratic_least_squares(dims, {p1.Up[j], p2.Up[j], p3.Up[j]});
        const vec_real cp = fit_quadratic_least_squares(dims, {p1.psic[j], p2.psic[j], p3.psic[j]});
        fc[j] = cf[0] * d * d + cf[1] * d + cf[2];
        Up[j] = cu[0] * d * d + cu[1] * d + cu[2];
        psic[j] = cp[0] * d * d + cp[1] * d + cp[2];
    }
    const vec_real cd = fit_quadratic_least_squares(dims, {p1.Delta, p2.Delta, p3.Delta});
    config.Delta = cd[0] * d * d + cd[1] * d + cd[2];
    config.fc = fc;
    config.Up = Up;
    config.psic = psic;
}

std::string runSuites(std::vector<SimulationSuite>& suites, const std::vector<std::string>& paths,
                      bool ignoreConverged, const std::filesystem::path& dataPath)
{
    std::string failures;
    std::vector<bool> stopped(suites.size(), false);
    size_t rounds = 0;
    for (const auto& s : suites) rounds = std::max(rounds, s.simulationDims.size());
    for (size_t k = 0; k < suites.size(); ++k)
        std::cout << "Starting multi run for " << suites[k].simulationDims.size() << " distinct dimensions"
                  << (suites.size() > 1 ? " (suite " + std::to_string(k + 1) + ")" : std::string()) << ".\n\n";
    for (size_t i = 0; i < rounds; ++i) {
        std::vector<std::unique_ptr<NewtonSolver>> solvers;
        std::vector<size_t> owner;
        for (size_t k = 0; k < suites.size(); ++k) {
            SimulationSuite& suite = suites[k];
            if (stopped[k] || i >= suite.simulationDims.size()) continue;
            const std::string& simDim = suite.simulationDims[i];
            std::cout << "Simulation " << i + 1 << "/" << suite.simulationDims.size() << ":\n"
                      << "Starting simulation for D=" << simDim << ".\n\n";
            SimulationConfig config = suite.generateSimulation(simDim);
            try {
                seedSuiteEntry(suite, i, config);
            } catch (const std::exception& e) {
                stopped[k] = true;
                failures += std::string(failures.empty() ? "" : "; ") + e.what();
                continue;
            }
            if (ignoreConverged) config.Converged = false;
            solvers.push_back(std::make_unique<NewtonSolver>(config, dataPath));
            owner.push_back(k);
        }
        std::vector<NewtonSolver*> raw;
        for (auto& s : solvers) raw.push_back(s.get());
        if (raw.empty()) break;
        std::vector<std::string> errs;
        const std::vector<json> results = NewtonSolver::runBatched(raw, &errs);
        for (size_t j = 0; j < raw.size(); ++j) {
            SimulationSuite& suite = suites[owner[j]];
            if (!errs[j].empty()) {
                std::cerr << "ERROR: " << errs[j] << std::endl;
                stopped[owner[j]] = true;
                failures += std::string(failures.empty() ? "" : "; ") + errs[j];
                continue;
            }
            suite.multiInputDict[suite.simulationDims[i]] = results[j];
            std::cout << "Result stored in file: " << paths[owner[j]] << "\n\n";
            SimulationConfig::saveToJson(paths[owner[j]], suite.multiInputDict);
        }
    }
    return failures;
}
