// Solver.cpp -- the host classes of Solver.hpp over the C ABI (include/pcc.h).
#include "Solver.hpp"

#include <iomanip>

#include <chrono>
#include <cstring>
#include <mutex>

namespace pcc {

pcc_ctx* device_context()
{
    static std::once_flag once;
    static pcc_ctx* ctx = nullptr;
    static pcc_status st = PCC_OK;
    std::call_once(once, [] {
        const char* dev = std::getenv("PCC_DEVICE");
        st = pcc_ctx_create(dev ? std::atoi(dev) : 0, nullptr, &ctx);
    });
    if (st != PCC_OK || !ctx) throw Error(st, "pcc_ctx_create failed: no usable CUDA device");
    return ctx;
}

void check(pcc_status s, const char* where)
{
    if (s != PCC_OK)
        throw Error(s, std::string(where) + ": " + pcc_status_string(s) + " (" + pcc_last_error(device_context()) + ")");
}

}  // namespace pcc

using pcc::check;
using pcc::device_context;

namespace {
double* dp(vec_complex& v) { return reinterpret_cast<double*>(v.data()); }
const double* dp(const vec_complex& v) { return reinterpret_cast<const double*>(v.data()); }
}  // namespace

// ============================================================ SpectralTransformer
// (reference src/SpectralTransformer.cpp)

SpectralTransformer::SpectralTransformer(size_t N_, real_t period_) : N(N_), period(period_), k0(2.0 * M_PI / period_) {}

void SpectralTransformer::dft(const vec_complex& in, vec_complex& out, int sign)
{
    vec_complex tmp(N);
    check(pcc_dft(device_context(), (int)N, 1, sign, dp(in), dp(tmp)), "pcc_dft");
    out.swap(tmp);
}

void SpectralTransformer::forwardFFT(const vec_real& in, vec_complex& out)
{
    vec_complex c(N);
    for (size_t i = 0; i < N; ++i) c[i] = complex_t(in[i], 0.0);
    forwardFFT(c, out);
}

void SpectralTransformer::forwardFFT(const vec_complex& in, vec_complex& out)
{
    dft(in, out, +1);  // the reference's "forward" plan is FFTW_BACKWARD (:33)
    for (auto& v : out) v /= static_cast<real_t>(N);
}

void SpectralTransformer::backwardFFT(const vec_complex& in, vec_real& out)
{
    vec_complex c;
    dft(in, c, -1);
    out.resize(N);
    for (size_t i = 0; i < N; ++i) out[i] = c[i].real();
}

void SpectralTransformer::backwardFFT(const vec_complex& in, vec_complex& out) { dft(in, out, -1); }

void SpectralTransformer::differentiate(const vec_complex& in, vec_complex& out, real_t period_)
{
    const real_t k0c = (period_ == 0.0) ? k0 : 2 * M_PI / period_;
    const size_t size = in.size();
    vec_complex o(size);
    for (size_t k = 0; k < size; ++k) {
        if (k != size / 2) {
            const int m = (k < size / 2) ? static_cast<int>(k) : static_cast<int>(k) - static_cast<int>(size);
            o[k] = -complex_t(0.0, m * k0c) * in[k];
        } else {
            o[k] = complex_t(0.0);
        }
    }
    out.swap(o);
}

void SpectralTransformer::lamIntegrate(const vec_complex& fk, vec_complex& out, complex_t lambda, real_t period_)
{
    const real_t k0c = (period_ == 0.0) ? k0 : 2 * M_PI / period_;
    const size_t size = fk.size();
    vec_complex o(size);
    o[0] = lambda != complex_t(0.0) ? fk[0] / lambda : complex_t(0.0);
    for (size_t k = 1; k < size; ++k) {
        if (k != size / 2) {
            const int m = (k < size / 2) ? static_cast<int>(k) : static_cast<int>(k) - static_cast<int>(size);
            const complex_t denom = lambda - complex_t(0.0, m * k0c);
            o[k] = (std::abs(denom) < 1e-14) ? complex_t(0.0) : fk[k] / denom;
        } else {
            o[k] = lambda / (lambda * lambda + (k0c * size / 2.0) * (k0c * size / 2.0)) * fk[k];
        }
    }
    out.swap(o);
}

void SpectralTransformer::halveModes(const vec_complex& in, vec_complex& out)
{
    const size_t n_out = in.size() / 2;
    vec_complex t(n_out);
    for (size_t k = 0; k < n_out / 2; ++k) t[k] = in[k];
    t[n_out / 2] = in[n_out / 2] + in[3 * n_out / 2];
    for (size_t k = n_out / 2 + 1; k < n_out; ++k) t[k] = in[n_out + k];
    out.swap(t);
}

void SpectralTransformer::doubleModes(const vec_complex& in, vec_complex& out)
{
    // the reference's store order (:231-251): out[3 n/2] ends with the full in[n/2]
    const size_t n_in = in.size();
    vec_complex o(2 * n_in);
    for (size_t k = 0; k < n_in / 2; ++k) o[k] = in[k];
    o[n_in / 2] = 0.5 * in[n_in / 2];
    o[3 * n_in / 2] = 0.5 * in[n_in / 2];
    for (size_t k = n_in / 2; k < n_in; ++k) o[n_in + k] = in[k];
    for (size_t k = n_in / 2 + 1; k < 3 * n_in / 2; ++k) o[k] = complex_t(0.0);
    out.swap(o);
}

void SpectralTransformer::solveInhom(const vec_real& f, const vec_real& g, vec_real& x, real_t period_)
{
    vec_complex f_hat, F_hat, h_hat, H_hat;
    forwardFFT(f, f_hat);
    lamIntegrate(f_hat, F_hat, complex_t(0.0), period_);
    vec_real Fr;
    backwardFFT(F_hat, Fr);
    vec_real h(N);
    for (size_t i = 0; i < N; ++i) h[i] = -g[i] * std::exp(Fr[i]);
    forwardFFT(h, h_hat);
    lamIntegrate(h_hat, H_hat, f_hat[0], period_);
    backwardFFT(H_hat, x);
    for (size_t i = 0; i < N; ++i) x[i] *= std::exp(-Fr[i]);
}

// ====================================================== InitialConditionGenerator
// (reference src/InitialConditionGenerator.cpp)

InitialConditionGenerator::InitialConditionGenerator(size_t Ntau_, real_t Dim_, real_t Delta_)
    : Ntau(Ntau_), Nnewton(3 * Ntau_ / 4), Dim(Dim_), Delta(Delta_), fft(Ntau_, Delta_)
{
}

void InitialConditionGenerator::computeLeftExpansion(real_t XLeft, const vec_real& fc, const vec_real& psic,
                                                     vec_complex& Y, real_t DeltaIn, bool PrintDiagnostics)
{
    Delta = DeltaIn;
    Y.resize(Ntau / 2);
    check(pcc_expansions(device_context(), (int)Ntau, Dim, Delta, XLeft, 0.0, fc.data(), psic.data(), nullptr, dp(Y),
                         nullptr),
          "pcc_expansions");
    if (PrintDiagnostics) std::cout << "[INFO] Left-side 5th-order Taylor expansion at x = " << XLeft << " completed.\n";
}

void InitialConditionGenerator::computeRightExpansion(real_t XRight, const vec_real& Up, vec_complex& Y,
                                                      real_t DeltaIn, bool PrintDiagnostics)
{
    Delta = DeltaIn;
    Y.resize(Ntau / 2);
    check(pcc_expansions(device_context(), (int)Ntau, Dim, Delta, 0.0, XRight, nullptr, nullptr, Up.data(), nullptr,
                         dp(Y)),
          "pcc_expansions");
    if (PrintDiagnostics) std::cout << "[INFO] Right-side 3rd-order Taylor expansion at x = " << XRight << " completed.\n";
}

void InitialConditionGenerator::packSpectralFields(const vec_real& Odd1, const vec_real& Odd2, const vec_real& Even,
                                                   vec_real& Z)
{
    Z.resize(Nnewton);
    check(pcc_pack_fields(device_context(), (int)Ntau, Odd1.data(), Odd2.data(), Even.data(), Z.data()),
          "pcc_pack_fields");
}

void InitialConditionGenerator::unpackSpectralFields(const vec_real& Z, vec_real& Odd1, vec_real& Odd2,
                                                     vec_real& Even)
{
    Odd1.resize(Ntau);
    Odd2.resize(Ntau);
    Even.resize(Ntau);
    check(pcc_unpack_fields(device_context(), (int)Ntau, Z.data(), Odd1.data(), Odd2.data(), Even.data()),
          "pcc_unpack_fields");
}

void InitialConditionGenerator::FieldsToStateVector(const vec_real& U, const vec_real& V, const vec_real& F,
                                                    vec_complex& Y)
{
    Y.resize(Ntau);
    for (size_t j = 0; j < Ntau; ++j) Y[j] = complex_t(U[j], V[j] + F[j]);
    fft.forwardFFT(Y, Y);
    fft.halveModes(Y, Y);
}

void InitialConditionGenerator::StateVectorToFields(vec_complex& Y, vec_real& U, vec_real& V, vec_real& F,
                                                    vec_real& IA2, vec_real& dUdt, vec_real& dVdt, vec_real& dFdt,
                                                    real_t X)
{
    vec_complex c1, c2;
    Delta = Y[2].real();
    fft.doubleModes(Y, c1);
    c1[2] = complex_t(-c1[c1.size() - 2].real(), c1[2].imag());
    fft.differentiate(c1, c2, Delta);
    fft.backwardFFT(c1, c1);
    fft.backwardFFT(c2, c2);
    const size_t h = Ntau / 2;
    for (auto* v : {&U, &V, &F, &IA2, &dUdt, &dVdt, &dFdt}) v->resize(Ntau);
    for (size_t j = 0; j < h; ++j) {
        U[j] = 0.5 * (c1[j].real() - c1[j + h].real());
        V[j] = 0.5 * (c1[j].imag() - c1[j + h].imag());
        F[j] = 0.5 * (c1[j].imag() + c1[j + h].imag());
        dUdt[j] = 0.5 * (c2[j].real() - c2[j + h].real());
        dVdt[j] = 0.5 * (c2[j].imag() - c2[j + h].imag());
        dFdt[j] = 0.5 * (c2[j].imag() + c2[j + h].imag());
        U[j + h] = -U[j];
        V[j + h] = -V[j];
        F[j + h] = F[j];
        dUdt[j + h] = -dUdt[j];
        dVdt[j + h] = -dVdt[j];
        dFdt[j + h] = dFdt[j];
    }
    vec_real k1(Ntau), k2(Ntau);
    for (size_t j = 0; j < Ntau; ++j) {
        k1[j] = -(((X + F[j]) * U[j] * U[j] + (X - F[j]) * V[j] * V[j]) * std::pow((Dim - 2.0), 3) / (8.0 * X) +
                  (Dim - 3.0));
        k2[j] = (Dim - 3.0);
    }
    fft.solveInhom(k1, k2, IA2, Delta);
}

void InitialConditionGenerator::StateVectorToFields(vec_complex& Y, vec_real& U, vec_real& V, vec_real& F)
{
    vec_complex c1;
    Delta = Y[2].real();
    fft.doubleModes(Y, c1);
    c1[2] = complex_t(-c1[c1.size() - 2].real(), c1[2].imag());
    fft.backwardFFT(c1, c1);
    const size_t h = Ntau / 2;
    U.resize(Ntau);
    V.resize(Ntau);
    F.resize(Ntau);
    for (size_t j = 0; j < h; ++j) {
        U[j] = 0.5 * (c1[j].real() - c1[j + h].real());
        V[j] = 0.5 * (c1[j].imag() - c1[j + h].imag());
        F[j] = 0.5 * (c1[j].imag() + c1[j + h].imag());
        U[j + h] = -U[j];
        V[j + h] = -V[j];
        F[j + h] = F[j];
    }
}

// ===================================================================== ODEStepper
// (reference src/ODEStepper.cpp)

ODEStepper::ODEStepper(int Ntau_, real_t Dim_, real_t precision_, Scheme method_, InitialConditionGenerator& initGen_)
    : Ntau(Ntau_), Dim(Dim_), precision(precision_), scheme(method_), initGen(initGen_)
{
}

void ODEStepper::integrate(vec_complex& Yin, vec_complex& Yout, real_t Xin, real_t Xout, bool& converged,
                           int& itsReached, int maxIts)
{
    vec_complex out(Ntau / 2);
    int its = 0;
    check(pcc_irk_step(device_context(), Ntau, Dim, int(scheme) + 1, precision, maxIts, 1, dp(Yin), &Xin, &Xout,
                       dp(out), &its),
          "pcc_irk_step");
    itsReached = its < 0 ? -its : its;
    converged = its > 0;
    Yout.swap(out);
}

// ================================================================= ShootingSolver
// (reference src/ShootingSolver.cpp)

ShootingSolver::ShootingSolver(int Ntau_, real_t Dim_, real_t precision_, InitialConditionGenerator& initGen_,
                               int maxIts_, Scheme SchemeIRK)
    : Ntau(Ntau_), Dim(Dim_), Precision(precision_), initGen(initGen_), maxIts(maxIts_), scheme(SchemeIRK)
{
}

ShootingSolver::~ShootingSolver()
{
    if (solve) pcc_solve_destroy(solve);
}

void ShootingSolver::shoot(vec_complex& YLeft, vec_complex& YRight, const vec_real& gridX, size_t iLeft,
                           size_t iRight, size_t iMid, vec_complex& mismatchOut, SimulationConfig* config,
                           json* fieldVals)
{
    if (iLeft != 0 || iRight + 1 != gridX.size() || iMid <= iLeft || iMid >= iRight)
        throw pcc::Error(PCC_ERR_UNSUPPORTED, "shoot expects iLeft = 0 < iMid < iRight = gridX.size() - 1");
    if (config && config->Debug && fieldVals)
        std::cerr << "[pcc] Debug field snapshots come from NewtonSolver::run (pcc_shoot_debug), not this call\n";
    const size_t nl = iMid - iLeft, nr = iRight - iMid;
    if (!solve || nl != cachedL || nr != cachedR) {
        if (solve) pcc_solve_destroy(solve);
        solve = nullptr;
        pcc_solve_desc d{};
        d.ntau = Ntau;
        d.dim = Dim;
        d.xl = gridX[iLeft];
        d.xm = gridX[iMid];
        d.xr = gridX[iRight];
        d.eps_newton = config ? config->EpsNewton : 1e-8;  // unused by a shoot; kept for reuse
        d.nl = (int)nl;
        d.nr = (int)nr;
        d.prec_irk = Precision;
        d.scheme = int(scheme) + 1;
        d.max_irk = maxIts;
        check(pcc_solve_create(device_context(), &d, &solve), "pcc_solve_create");
        cachedL = nl;
        cachedR = nr;
    }
    check(pcc_solve_set_grid(solve, gridX.data()), "pcc_solve_set_grid");
    vec_complex y(Ntau), out(Ntau);
    std::memcpy(y.data(), YLeft.data(), sizeof(complex_t) * (Ntau / 2));
    std::memcpy(y.data() + Ntau / 2, YRight.data(), sizeof(complex_t) * (Ntau / 2));
    const int sides[2] = {0, 1};
    pcc_stats st{};
    check(pcc_sweep(solve, 2, sides, dp(y), dp(out), &st), "pcc_sweep");
    YLeft.assign(out.begin(), out.begin() + Ntau / 2);
    YRight.assign(out.begin() + Ntau / 2, out.end());
    // computeMismatch (:154-182)
    mismatchOut.resize(Ntau / 2);
    for (int i = 0; i < Ntau / 2; ++i) mismatchOut[i] = YRight[i] - YLeft[i];
    if (mismatchOut[2].real() > Precision) throw pcc::Error(PCC_ERR_DELTA_MISMATCH, "Mismatch in Delta from left and right side");
    mismatchOut[2] = complex_t(YLeft[2].real(), mismatchOut[2].imag());
}

// =================================================================== NewtonSolver
// (reference src/NewtonSolver.cpp, serial/OpenMP build)

NewtonSolver::NewtonSolver(SimulationConfig configIn, std::filesystem::path dataPathIn, bool benchmarkIn)
    : config(configIn), Ntau(configIn.Ntau), Nnewton(3 * configIn.Ntau / 4), maxIts(configIn.MaxIterNewton),
      Dim(configIn.Dim), Delta(configIn.Delta), slowErr(configIn.SlowError), EpsNewton(configIn.EpsNewton),
      TolNewton(configIn.PrecisionNewton), XLeft(configIn.XLeft), XMid(configIn.XMid), XRight(configIn.XRight),
      NLeft(configIn.NLeft), NRight(configIn.NRight), Verbose(configIn.Verbose), Converged(configIn.Converged),
      initGen(configIn.Ntau, configIn.Dim, configIn.Delta), baseFolder(dataPathIn), benchmark(benchmarkIn)
{
    fc = configIn.fc;
    psic = configIn.psic;
    Up = configIn.Up;
    in0.resize(Nnewton);
    out0.resize(Nnewton);
    const char* p = std::getenv("PCC_LU_PRECISION");
    if (p && std::string(p) == "mixed") linearPrecision = PCC_PREC_MIXED;
    const pcc_solve_desc d = config.desc();
    check(pcc_solve_create(device_context(), &d, &solve), "pcc_solve_create");
}

NewtonSolver::~NewtonSolver()
{
    if (solve) pcc_solve_destroy(solve);
}

real_t NewtonSolver::computeL2Norm(const vec_real& vc)
{
    real_t s = 0.0;
    for (real_t x : vc) s += x * x;
    return std::sqrt(s / static_cast<real_t>(vc.size()));
}

void NewtonSolver::shoot(vec_real& inputVec, vec_real& outputVec)
{
    // the fields the shoot starts from (kept for writeFinalOutput, as :408-412 does)
    Delta = inputVec[2 * Nnewton / 3 + 2];
    vec_real z = inputVec;
    z[2 * Nnewton / 3 + 2] = 0.0;
    initGen.unpackSpectralFields(z, Up, psic, fc);
    pcc_stats st{};
    outputVec.resize(Nnewton);
    check(pcc_shoot(solve, inputVec.data(), outputVec.data(), &st), "pcc_shoot");
}

// every n-th element and the last one (common.cpp:201-215)
static vec_real every_nth_element(const vec_real& a, size_t n)
{
    vec_real out;
    for (size_t i = 0; i < a.size(); ++i)
        if (i % n == 0 || i == a.size() - 1) out.push_back(a[i]);
    return out;
}

void NewtonSolver::shootDebug(vec_real& inputVec, vec_real& outputVec, json& fieldVals)
{
    Delta = inputVec[2 * Nnewton / 3 + 2];
    vec_real z = inputVec;
    z[2 * Nnewton / 3 + 2] = 0.0;
    initGen.unpackSpectralFields(z, Up, psic, fc);
    outputVec.resize(Nnewton);
    int count = 0;
    pcc_shoot_debug(solve, inputVec.data(), outputVec.data(), (int)config.DebugNx, 0, &count, nullptr, nullptr,
                    nullptr);  // counts the snapshots
    std::vector<int> idx(count);
    vec_real fields((size_t)count * 4 * Ntau);
    pcc_stats st{};
    check(pcc_shoot_debug(solve, inputVec.data(), outputVec.data(), (int)config.DebugNx, count, &count, idx.data(),
                          fields.data(), &st),
          "pcc_shoot_debug");
    vec_real grid(NLeft + NRight + 1);
    check(pcc_solve_grid(solve, grid.data()), "pcc_solve_grid");
    static const char* names[4] = {"A", "U", "V", "f"};
    for (int k = 0; k < count; ++k) {
        const std::string key = std::to_string(grid[idx[k]]);
        for (int q = 0; q < 4; ++q) {
            const real_t* f = &fields[((size_t)k * 4 + q) * Ntau];
            fieldVals[key][names[q]] = every_nth_element(vec_real(f, f + Ntau), config.DebugNtau);
        }
    }
}

void NewtonSolver::assembleJacobian(const vec_real& baseInput, const vec_real& baseOutput, mat_real& jacobian)
{
    std::cout << "Starting to assemble Jacobian: " << std::endl << std::endl;
    const auto t0 = std::chrono::high_resolution_clock::now();
    vec_real J(Nnewton * Nnewton);
    pcc_stats st{};
    check(pcc_jacobian(solve, baseInput.data(), baseOutput.data(), J.data(), &st), "pcc_jacobian");
    jacobian.assign(Nnewton, vec_real(Nnewton));
    for (size_t r = 0; r < Nnewton; ++r) std::memcpy(jacobian[r].data(), &J[r * Nnewton], Nnewton * sizeof(real_t));
    const auto t1 = std::chrono::high_resolution_clock::now();
    std::cout << "Time for Newton Iteration: " << static_cast<real_t>((t1 - t0).count()) / 1e9 << " s." << std::endl
              << std::endl;
}

void NewtonSolver::solveLinearSystem(const mat_real& A_in, vec_real& rhs, vec_real& dx)
{
    vec_real A((size_t)Nnewton * Nnewton);
    for (size_t i = 0; i < Nnewton; ++i) std::memcpy(&A[i * Nnewton], A_in[i].data(), Nnewton * sizeof(real_t));
    dx.resize(Nnewton);
    pcc_refine_report rep{};
    check(pcc_lu_solve(device_context(), (int)Nnewton, A.data(), rhs.data(), dx.data(), linearPrecision, &rep),
          "pcc_lu_solve");
}

json NewtonSolver::run(json* benchmark_result)
{
    using clk = std::chrono::high_resolution_clock;
    clk::time_point overallStart{}, newtonStart{}, assembleStart{};
    if (benchmark) overallStart = clk::now();
    if (!Converged) {
        real_t fac = 1.0, err = 1.0, errOld = 1.0;
        int mismatch_increase_count = 0;
        initGen.packSpectralFields(Up, psic, fc, in0);
        in0[2 * Nnewton / 3 + 2] = Delta;
        vec_real in0old = in0;
        for (size_t its = 0; its < maxIts; ++its) {
            if (benchmark) newtonStart = clk::now();
            std::cout << "Newton iteration: " << its + 1 << std::endl;
            errOld = err;
            if (config.Debug) {
                // the base shoot with the field export (NewtonSolver.cpp:287-295)
                json fieldVals;
                shootDebug(in0, out0, fieldVals);
                const auto fieldPath = baseFolder / ("fields_" + std::to_string(Dim) + "_" + std::to_string(its) + ".json");
                SimulationConfig::saveToJson(fieldPath.string(), fieldVals);
            } else {
                shoot(in0, out0);
            }
            err = computeL2Norm(out0);
            std::cout << "Mismatch norm: " << err << std::endl;
            if (err < TolNewton) {
                Converged = true;
                std::cout << "The solution has converged!" << std::endl << std::endl;
                writeFinalOutput(its, err);
                break;
            }
            if (std::log10(err) > std::log10(errOld)) mismatch_increase_count++;
            if (mismatch_increase_count >= 5) {
                Converged = true;
                Delta = in0old[2 * Nnewton / 3 + 2];
                in0old[2 * Nnewton / 3 + 2] = 0.0;
                initGen.unpackSpectralFields(in0old, Up, psic, fc);
                writeFinalOutput(its, errOld);
                std::cerr << "Mismatch increased - terminating Newton.\n";
                break;
            }
            mat_real J;
            if (benchmark) assembleStart = clk::now();
            assembleJacobian(in0, out0, J);
            if (config.Debug) {
                // NewtonSolver.cpp:337-341 and OutputWriter::writeMatrix
                const auto jacPath =
                    baseFolder / ("jacobian_" + std::to_string(Dim) + "_" + std::to_string(its + 1) + ".csv");
                std::ofstream outfile(jacPath);
                if (!outfile) throw std::runtime_error("Could not open file for writing: " + jacPath.string());
                outfile << std::setprecision(16);
                for (size_t i = 0; i < J.size(); ++i) {
                    for (size_t j = 0; j + 1 < J[i].size(); ++j) outfile << J[i][j] << ", ";
                    outfile << J[i][J[i].size() - 1] << std::endl;
                }
            }
            if (benchmark)
                (*benchmark_result)["AssembleStep_" + std::to_string(its + 1)] =
                    static_cast<double>((clk::now() - assembleStart).count()) / 1e9;
            vec_real dx(Nnewton), rhs = out0;
            for (auto& e : rhs) e *= -1.0;
            solveLinearSystem(J, rhs, dx);
            fac = std::min(1.0, slowErr / err);
            if (std::log10(err) < std::log10(errOld)) {
                in0old = in0;
                mismatch_increase_count = 0;
            }
            for (size_t i = 0; i < Nnewton; ++i) in0[i] += fac * dx[i];
            if (benchmark)
                (*benchmark_result)["NewtonStep_" + std::to_string(its + 1)] =
                    static_cast<double>((clk::now() - newtonStart).count()) / 1e9;
        }
        if (!Converged)
            throw pcc::Error(PCC_ERR_NEWTON_NO_CONVERGENCE, "Newton method did not converge in " + std::to_string(maxIts) +
                                                                 " iterations. For dimension: " + std::to_string(Dim));
    } else {
        initGen.packSpectralFields(Up, psic, fc, in0);
        in0[2 * Nnewton / 3 + 2] = Delta;
        shoot(in0, out0);
        const real_t err = computeL2Norm(out0);
        std::cout << "The solution is already marked as converged!" << std::endl;
        writeFinalOutput(0, err);
    }
    if (benchmark) (*benchmark_result)["OverallTime"] = static_cast<double>((clk::now() - overallStart).count()) / 1e9;
    return resultDict;
}

std::vector<json> NewtonSolver::runBatched(const std::vector<NewtonSolver*>& solvers,
                                           std::vector<std::string>* errors)
{
    std::vector<json> out(solvers.size());
    if (errors) errors->assign(solvers.size(), std::string());
    std::vector<size_t> idx;
    for (size_t k = 0; k < solvers.size(); ++k) {
        if (solvers[k]->Converged)
            out[k] = solvers[k]->run();  // one shoot to report the stored solution
        else
            idx.push_back(k);
    }
    if (idx.empty()) return out;
    std::vector<pcc_solve*> handles;
    std::vector<vec_real> x(idx.size());
    std::vector<double*> xp;
    for (size_t j = 0; j < idx.size(); ++j) {
        NewtonSolver* a = solvers[idx[j]];
        a->initGen.packSpectralFields(a->Up, a->psic, a->fc, a->in0);
        a->in0[2 * a->Nnewton / 3 + 2] = a->Delta;
        x[j] = a->in0;
        handles.push_back(a->solve);
        xp.push_back(x[j].data());
    }
    std::vector<pcc_newton_state> st(idx.size());
    const pcc_precision prec = solvers[idx[0]]->linearPrecision;
    check(pcc_newton_solve(device_context(), (int)idx.size(), handles.data(), xp.data(), prec, st.data(), nullptr),
          "pcc_newton_solve");
    std::string failures;
    for (size_t j = 0; j < idx.size(); ++j) {
        NewtonSolver* a = solvers[idx[j]];
        const pcc_newton_state& s = st[j];
        std::cout << "D = " << a->Dim << ": " << s.iterations << " Newton iterations, mismatch norm " << s.err << std::endl;
        if (s.code == PCC_NEWTON_CONVERGED || s.code == PCC_NEWTON_STOPPED) {
            // the result iterate (the last improving one when stopped) -> fields, as :306-321
            vec_real z = x[j];
            a->in0 = z;
            a->Delta = z[2 * a->Nnewton / 3 + 2];
            z[2 * a->Nnewton / 3 + 2] = 0.0;
            a->initGen.unpackSpectralFields(z, a->Up, a->psic, a->fc);
            a->Converged = true;
            if (s.code == PCC_NEWTON_CONVERGED) {
                std::cout << "The solution has converged!" << std::endl << std::endl;
                a->writeFinalOutput((size_t)(s.iterations - 1), s.err);
            } else {
                std::cerr << "Mismatch increased - terminating Newton.\n";
                a->writeFinalOutput((size_t)(s.iterations - 1), s.err_old);
            }
            out[idx[j]] = a->resultDict;
        } else {
            const char* what = s.code == PCC_NEWTON_MAX_ITER         ? "Newton method did not converge"
                               : s.code == PCC_NEWTON_IRK_FAILED      ? "IRK iteration did not converge"
                               : s.code == PCC_NEWTON_DELTA_MISMATCH ? "Delta mismatch between the sides"
                                                                      : "singular Jacobian";
            const std::string msg = std::string(what) + " for dimension " + std::to_string(a->Dim);
            if (errors) (*errors)[idx[j]] = msg;
            failures += std::string(failures.empty() ? "" : "; ") + msg;
        }
    }
    if (!failures.empty() && !errors) throw pcc::Error(PCC_ERR_NEWTON_NO_CONVERGENCE, failures);
    return out;
}

void NewtonSolver::writeFinalOutput(size_t newtonIts, real_t mismatchNorm)
{
    resultDict["Ntau"] = Ntau;
    resultDict["Dim"] = Dim;
    resultDict["XLeft"] = XLeft;
    resultDict["XMid"] = XMid;
    resultDict["XRight"] = XRight;
    resultDict["EpsNewton"] = EpsNewton;
    resultDict["PrecisionNewton"] = TolNewton;
    resultDict["SlowError"] = slowErr;
    resultDict["MaxIterNewton"] = maxIts;
    resultDict["Verbose"] = Verbose;
    resultDict["Debug"] = config.Debug;
    if (config.Debug) {
        resultDict["DebugNx"] = config.DebugNx;
        resultDict["DebugNtau"] = config.DebugNtau;
    }
    resultDict["Converged"] = true;
    resultDict["NLeft"] = NLeft;
    resultDict["NRight"] = NRight;
    resultDict["SchemeIRK"] = int(config.SchemeIRK) + 1;
    resultDict["PrecisionIRK"] = config.PrecisionIRK;
    resultDict["MaxIterIRK"] = config.MaxIterIRK;
    resultDict["IterNewton"] = newtonIts;
    resultDict["mismatchNorm"] = mismatchNorm;
    resultDict["Initial_Conditions"]["Delta"] = Delta;
    resultDict["Initial_Conditions"]["fc"] = fc;
    resultDict["Initial_Conditions"]["psic"] = psic;
    resultDict["Initial_Conditions"]["Up"] = Up;
    std::cout << "Final result stored in simulation dictionary for dimension D = " << Dim << "." << std::endl << std::endl;
}
