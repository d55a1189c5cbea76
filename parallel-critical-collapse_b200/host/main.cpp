// main.cpp -- cc_b200: the reference's command line (src/main.cpp:19-378) on
// the B200 engine.
//
//   cc_b200 [-s] -i data/simulation_4D_512.json [--ignore-converged]
//   cc_b200 -b --benchmark-repetitions 3 -i ...
//   cc_b200 -m -i suite.json [-r] [--ignore-converged]
//   cc_b200 -m --suite up.json asc --suite down.json desc [--ignore-converged]
//
// Single run: the result dictionary is written back over the input file, as
// the reference does (main.cpp:221-233).  Benchmark mode writes
// benchmark_D=<D>_B200_1.json next to the input with the reference's keys
// (Dim, Ntau, ..., Kind, per-repetition AssembleStep_k / NewtonStep_k /
// OverallTime).  Suite mode (-m) continues through the dimensions of a
// multi-dimension file (-r: ascending, else descending), writing the file
// after every dimension; --suite (repeatable, not in the reference) names
// several such files with their own order, which then run in lockstep with
// their Newton solves batched together.
#include <cstring>

#include "Suite.hpp"

int main(int argc, char** argv)
{
    bool benchmark = false, ignoreConverged = false, multiple = false, reversed = false;
    std::vector<std::pair<std::string, bool>> suiteSpecs;  // --suite path asc|desc
    int reps = 3;
    std::string inputPath = "data/simulation_4D_512.json";
    for (int i = 1; i < argc; ++i) {
        const std::string a = argv[i];
        if (a == "-s" || a == "--single-run") {
        } else if (a == "-m" || a == "--multiple-run") {
            multiple = true;
        } else if (a == "-r" || a == "--reversed-order") {
            reversed = true;
        } else if (a == "--suite") {
            if (i + 2 >= argc || (std::string(argv[i + 2]) != "asc" && std::string(argv[i + 2]) != "desc")) {
                std::cerr << "--suite needs <path> asc|desc\n";
                return 2;
            }
            suiteSpecs.emplace_back(argv[i + 1], std::string(argv[i + 2]) == "asc");
            i += 2;
            multiple = true;
        } else if (a == "--ignore-converged") {
            ignoreConverged = true;
        } else if (a == "-i" || a == "--input-path") {
            if (i + 1 < argc) {
                inputPath = argv[++i];
            } else {
                std::cerr << "Invalid simulation input path!\n";
                return 2;
            }
        } else if (a == "-b" || a == "--benchmark") {
            benchmark = true;
        } else if (a == "--benchmark-repetitions") {
            if (i + 1 < argc) reps = std::stoi(argv[++i]);
        }
    }
    const std::filesystem::path dataPath = std::filesystem::path(inputPath).parent_path();
    try {
        if (multiple) {
            if (suiteSpecs.empty()) suiteSpecs.emplace_back(inputPath, reversed);
            std::vector<SimulationSuite> suites;
            std::vector<std::string> paths;
            for (const auto& sp : suiteSpecs) {
                suites.emplace_back(sp.first, sp.second, ignoreConverged);
                paths.push_back(sp.first);
            }
            const std::string failed = runSuites(suites, paths, ignoreConverged,
                                                 std::filesystem::path(paths[0]).parent_path());
            if (!failed.empty()) {
                std::cerr << "ERROR: " << failed << std::endl;
                return 1;
            }
            return 0;
        }
        SimulationConfig config = SimulationConfig::loadFromJson(inputPath);
        if (ignoreConverged) config.Converged = false;
        if (benchmark) {
            json res;
            res["Dim"] = config.Dim;
            res["Ntau"] = config.Ntau;
            res["XLeft"] = config.XLeft;
            res["XMid"] = config.XMid;
            res["XRight"] = config.XRight;
            res["PrecisionNewton"] = config.PrecisionNewton;
            res["NLeft"] = config.NLeft;
            res["NRight"] = config.NRight;
            res["Repetitions"] = reps;
            res["Kind"] = "B200";
            res["Cores"] = 1;
            std::cout << "Starting benchmark run for D=" << config.Dim << ".\n\n";
            for (int r = 0; r < reps; ++r) {
                std::cout << "Repetition " << r + 1 << "/" << reps << "\n\n";
                NewtonSolver solver(config, dataPath, true);
                solver.run(&res[std::to_string(r)]);
            }
            const auto out = dataPath / ("benchmark_D=" + std::to_string(config.Dim) + "_B200_1.json");
            std::cout << "Benchmark result stored in file: " << out << "\n\n";
            SimulationConfig::saveToJson(out.string(), res);
        } else {
            std::cout << "Starting single run for D=" << config.Dim << ".\n\n";
            NewtonSolver solver(config, dataPath);
            json result = solver.run();
            std::cout << "Result stored in file: " << inputPath << "\n\n";
            SimulationConfig::saveToJson(inputPath, result);
        }
    } catch (const pcc::Error& e) {
        std::cerr << "ERROR: " << e.what() << std::endl;
        return 1;
    } catch (const std::exception& e) {
        std::cerr << "ERROR: " << e.what() << std::endl;
        return 1;
    }
    return 0;
}
