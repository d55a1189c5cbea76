#pragma once
/**
 * @file common.hpp
 * @brief Types shared by the host classes (the reference's include/common.hpp:
 *        real_t, complex_t, vec_real, vec_complex, mat_real, json, Scheme) and
 *        the process-wide device context the classes run on.
 *
 * The host classes keep the reference's interfaces (NewtonSolver,
 * ShootingSolver, ODEStepper, InitialConditionGenerator, SpectralTransformer,
 * SimulationConfig) and do their numerical work through the C ABI of
 * include/pcc.h on a CUDA device.  Where the reference calls std::exit or
 * MPI_Abort (IRK non-convergence, Delta mismatch, singular J, Newton
 * non-convergence) these classes throw pcc::Error carrying the pcc_status.
 */
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdlib>
#include <filesystem>
#include <fstream>
#include <iostream>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include <nlohmann/json.hpp>

#include "pcc.h"

enum class Scheme { IRK1, IRK2, IRK3 };

using real_t = double;
using complex_t = std::complex<real_t>;
using vec_real = std::vector<real_t>;
using vec_complex = std::vector<complex_t>;
using mat_real = std::vector<std::vector<real_t>>;
using json = nlohmann::json;

namespace pcc {

/// A failure the reference would have exited on.
class Error : public std::runtime_error {
  public:
    Error(pcc_status s, const std::string& what) : std::runtime_error(what), status(s) {}
    pcc_status status;
};

/// The process-wide CUDA context (device from $PCC_DEVICE, default 0).
pcc_ctx* device_context();

/// Throws pcc::Error when s != PCC_OK, with the context's last error text.
void check(pcc_status s, const char* where);

}  // namespace pcc
