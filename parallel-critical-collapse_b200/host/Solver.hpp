#pragma once
/**
 * @file Solver.hpp
 * @brief The reference's solver classes with their interfaces kept, computing
 *        on the GPU through include/pcc.h:
 *
 *  - SpectralTransformer      (reference include/SpectralTransformer.hpp:29-102)
 *  - InitialConditionGenerator(reference include/InitialConditionGenerator.hpp:46-209)
 *  - ODEStepper               (reference include/ODEStepper.hpp:38-111)
 *  - ShootingSolver           (reference include/ShootingSolver.hpp:36-118)
 *  - NewtonSolver             (reference include/NewtonSolver.hpp:42-170)
 *
 * Work placement.  Transforms, boundary expansions, packing, IRK steps, the
 * sweeps, the Jacobian and the LU run on the device.  SpectralTransformer's
 * O(N) mode bookkeeping (differentiate, lamIntegrate, halve/doubleModes)
 * runs in the host class around device DFTs; it serves callers that use the
 * class directly and is not on the Newton-shooting path.
 */
#include "SimulationConfig.hpp"

class SpectralTransformer {
  public:
    SpectralTransformer(size_t N, real_t period);
    void forwardFFT(const vec_real& in, vec_complex& out);     // e^{+i}, scaled 1/N
    void backwardFFT(const vec_complex& in, vec_real& out);    // e^{-i}, real part
    void forwardFFT(const vec_complex& in, vec_complex& out);
    void backwardFFT(const vec_complex& in, vec_complex& out);
    void differentiate(const vec_complex& in, vec_complex& out, real_t period_ = 0.0);
    void lamIntegrate(const vec_complex& fk, vec_complex& out, complex_t lambda = complex_t(0.0),
                      real_t period_ = 0.0);
    void halveModes(const vec_complex& in, vec_complex& out);
    void doubleModes(const vec_complex& in, vec_complex& out);
    void solveInhom(const vec_real& f, const vec_real& g, vec_real& x, real_t period_ = 0.0);

  private:
    size_t N;
    real_t period, k0;
    void dft(const vec_complex& in, vec_complex& out, int sign);
};

class InitialConditionGenerator {
  public:
    InitialConditionGenerator(size_t Ntau, real_t Dim, real_t Delta);
    void computeLeftExpansion(real_t XLeft, const vec_real& fc, const vec_real& psic, vec_complex& Y,
                              real_t DeltaIn, bool PrintDiagnostics = false);
    void computeRightExpansion(real_t XRight, const vec_real& Up, vec_complex& Y, real_t DeltaIn,
                               bool PrintDiagnostics = false);
    void packSpectralFields(const vec_real& Odd1, const vec_real& Odd2, const vec_real& Even, vec_real& Z);
    void unpackSpectralFields(const vec_real& Z, vec_real& Odd1, vec_real& Odd2, vec_real& Even);
    void FieldsToStateVector(const vec_real& U, const vec_real& V, const vec_real& F, vec_complex& Y);
    void StateVectorToFields(vec_complex& Y, vec_real& U, vec_real& V, vec_real& F, vec_real& IA2, vec_real& dUdt,
                             vec_real& dVdt, vec_real& dFdt, real_t X);
    void StateVectorToFields(vec_complex& Y, vec_real& U, vec_real& V, vec_real& F);

    size_t Ntau, Nnewton;
    real_t Dim, Delta;

  private:
    SpectralTransformer fft;
};

class ODEStepper {
  public:
    ODEStepper(int Ntau, real_t Dim, real_t precision, Scheme method, InitialConditionGenerator& initGen);
    void integrate(vec_complex& Yin, vec_complex& Yout, real_t Xin, real_t Xout, bool& converged, int& itsReached,
                   int maxIts);

  private:
    int Ntau;
    real_t Dim, precision;
    Scheme scheme;
    InitialConditionGenerator& initGen;
};

class ShootingSolver {
  public:
    ShootingSolver(int Ntau, real_t Dim, real_t precision, InitialConditionGenerator& initGen, int maxIts,
                   Scheme SchemeIRK = Scheme::IRK2);
    ~ShootingSolver();
    void shoot(vec_complex& YLeft, vec_complex& YRight, const vec_real& gridX, size_t iLeft, size_t iRight,
               size_t iMid, vec_complex& mismatchOut, SimulationConfig* config = nullptr, json* fieldVals = nullptr);

  private:
    int Ntau;
    real_t Dim, Precision;
    InitialConditionGenerator& initGen;
    int maxIts;
    Scheme scheme;
    pcc_solve* solve = nullptr;  // cached for one grid shape
    size_t cachedL = 0, cachedR = 0;
};

class NewtonSolver {
  public:
    NewtonSolver(SimulationConfig configIn, std::filesystem::path dataPathIn, bool benchmarkIn = false);
    ~NewtonSolver();
    NewtonSolver(const NewtonSolver&) = delete;
    NewtonSolver& operator=(const NewtonSolver&) = delete;

    json run(json* benchmark_result = nullptr);
    void writeFinalOutput(size_t newtonIts, real_t mismatchNorm);

    /// run() for several solvers at once through the device-resident Newton
    /// loop (pcc_newton_solve): every iteration's shoots of all solvers still
    /// running share one batch launch, and the loop state (mismatch history,
    /// divergence counter, last improving iterate) stays on the device.  The
    /// result dictionaries are those run() writes.  Failures throw pcc::Error
    /// after every solver has finished, unless `errors` is given: then
    /// errors[k] describes solver k's failure ("" when it converged).
    static std::vector<json> runBatched(const std::vector<NewtonSolver*>& solvers,
                                        std::vector<std::string>* errors = nullptr);

    /// Precision of the dense Newton solve: PCC_PREC_FP64 (dgesv semantics,
    /// the default) or PCC_PREC_MIXED ($PCC_LU_PRECISION=mixed).
    pcc_precision linearPrecision = PCC_PREC_FP64;

  private:
    SimulationConfig config;
    size_t Ntau, Nnewton, maxIts;
    real_t Dim, Delta, slowErr, EpsNewton, TolNewton, XLeft, XMid, XRight;
    size_t NLeft, NRight;
    bool Verbose, Converged;
    InitialConditionGenerator initGen;
    vec_real fc, psic, Up, in0, out0;
    json resultDict;
    std::filesystem::path baseFolder;
    bool benchmark;
    pcc_solve* solve = nullptr;

    void shoot(vec_real& inputVec, vec_real& outputVec);
    /// shoot with the Debug field export (ShootingSolver.cpp:85-97, 128-138)
    void shootDebug(vec_real& inputVec, vec_real& outputVec, json& fieldVals);
    void assembleJacobian(const vec_real& baseInput, const vec_real& baseOutput, mat_real& jacobian);
    void solveLinearSystem(const mat_real& A, vec_real& rhs, vec_real& dx);
    real_t computeL2Norm(const vec_real& vc);
};
