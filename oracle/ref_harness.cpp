// ref_harness.cpp -- TEST INFRASTRUCTURE ONLY.
//
// A C-ABI over the *compiled reference* (tobjec/parallel-critical-collapse,
// built unmodified by oracle/build_ref.sh except the one-line null-config fix
// at src/NewtonSolver.cpp:456).  Nothing here re-implements the algorithm: each
// entry point constructs the reference's own classes and calls the method that
// the named reference line defines.  It exists so that tests and the CPU
// reference arm of bench.py can call the reference from Python via ctypes.
//
// Private members are reached by compiling this one translation unit with
// `private` redefined to `public`; the reference objects themselves are
// compiled normally.
#include <any>
#include <cstdio>
#include <map>
#include <string>

#include "common.hpp"  // all standard and third-party headers, before the redefinition

#define private public
#include "InitialConditionGenerator.hpp"
#include "NewtonSolver.hpp"
#include "ODEStepper.hpp"
#include "ShootingSolver.hpp"
#include "SimulationConfig.hpp"
#include "SpectralTransformer.hpp"
#undef private

namespace {

void to_complex(const double* re_im, size_t n, vec_complex& out)
{
    out.resize(n);
    for (size_t i = 0; i < n; ++i) out[i] = complex_t(re_im[2 * i], re_im[2 * i + 1]);
}

void from_complex(const vec_complex& in, double* re_im)
{
    for (size_t i = 0; i < in.size(); ++i) {
        re_im[2 * i] = in[i].real();
        re_im[2 * i + 1] = in[i].imag();
    }
}

Scheme scheme_of(int s) { return s == 1 ? Scheme::IRK1 : (s == 3 ? Scheme::IRK3 : Scheme::IRK2); }

// Parses the reference's SimulationConfig JSON (include/SimulationConfig.hpp:73-137).
SimulationConfig parse_cfg(const char* cfg_json) { return SimulationConfig(json::parse(cfg_json)); }

}  // namespace

extern "C" {

// InitialConditionGenerator::packSpectralFields (src/InitialConditionGenerator.cpp:678-711)
int ref_pack(int ntau, double dim, double delta, const double* up, const double* psic, const double* fc,
             double* z_out)
{
    InitialConditionGenerator g(ntau, dim, delta);
    vec_real a(up, up + ntau), b(psic, psic + ntau), c(fc, fc + ntau), z;
    g.packSpectralFields(a, b, c, z);
    for (size_t i = 0; i < z.size(); ++i) z_out[i] = z[i];
    return (int)z.size();
}

// InitialConditionGenerator::unpackSpectralFields (src/InitialConditionGenerator.cpp:719-758)
int ref_unpack(int ntau, double dim, double delta, const double* z, double* up, double* psic, double* fc)
{
    InitialConditionGenerator g(ntau, dim, delta);
    vec_real zz(z, z + 3 * ntau / 4), a(ntau), b(ntau), c(ntau);
    g.unpackSpectralFields(zz, a, b, c);
    for (int i = 0; i < ntau; ++i) {
        up[i] = a[i];
        psic[i] = b[i];
        fc[i] = c[i];
    }
    return 0;
}

// InitialConditionGenerator::computeLeftExpansion (src/InitialConditionGenerator.cpp:37-239)
// y_out: Ntau/2 complex values interleaved (re, im).
int ref_left_expansion(int ntau, double dim, double xl, const double* fc, const double* psic, double delta,
                       double* y_out)
{
    InitialConditionGenerator g(ntau, dim, delta);
    vec_real f(fc, fc + ntau), p(psic, psic + ntau);
    vec_complex y(ntau);
    g.computeLeftExpansion(xl, f, p, y, delta, false);
    from_complex(y, y_out);
    return (int)y.size();
}

// InitialConditionGenerator::computeRightExpansion (src/InitialConditionGenerator.cpp:252-667)
int ref_right_expansion(int ntau, double dim, double xr, const double* up, double delta, double* y_out)
{
    InitialConditionGenerator g(ntau, dim, delta);
    vec_real u(up, up + ntau);
    vec_complex y(ntau);
    g.computeRightExpansion(xr, u, y, delta, false);
    from_complex(y, y_out);
    return (int)y.size();
}

// InitialConditionGenerator::StateVectorToFields with derivatives and IA2
// (src/InitialConditionGenerator.cpp:791-884).  Outputs are Ntau reals each.
int ref_state_to_fields(int ntau, double dim, const double* y, double x, double* u, double* v, double* f,
                        double* ia2, double* dudt, double* dvdt, double* dfdt)
{
    InitialConditionGenerator g(ntau, dim, y[4]);
    vec_complex yy;
    to_complex(y, ntau / 2, yy);
    vec_real U(ntau), V(ntau), F(ntau), A(ntau), dU(ntau), dV(ntau), dF(ntau);
    g.StateVectorToFields(yy, U, V, F, A, dU, dV, dF, x);
    for (int i = 0; i < ntau; ++i) {
        u[i] = U[i];
        v[i] = V[i];
        f[i] = F[i];
        ia2[i] = A[i];
        dudt[i] = dU[i];
        dvdt[i] = dV[i];
        dfdt[i] = dF[i];
    }
    return 0;
}

// ODEStepper::computeDerivatives (src/ODEStepper.cpp:92-136).  y and dy are the
// interleaved real storage of Ntau/2 complex modes (Ntau reals).
int ref_rhs(int ntau, double dim, const double* y, double x, double* dy)
{
    InitialConditionGenerator g(ntau, dim, y[4]);
    ODEStepper st(ntau, dim, 1e-15, Scheme::IRK2, g);
    vec_real yy(y, y + ntau), d(ntau);
    st.computeDerivatives(yy, d, x);
    for (int i = 0; i < ntau; ++i) dy[i] = d[i];
    return 0;
}

// ODEStepper::stepIRK (src/ODEStepper.cpp:163-292).
int ref_irk_step(int ntau, double dim, int scheme, double precision, int max_its, const double* y_in, double x_in,
                 double x_out, double* y_out, int* its, int* converged)
{
    InitialConditionGenerator g(ntau, dim, y_in[4]);
    ODEStepper st(ntau, dim, precision, scheme_of(scheme), g);
    vec_complex yi, yo(ntau / 2);
    to_complex(y_in, ntau / 2, yi);
    bool conv = false;
    int it = 0;
    st.integrate(yi, yo, x_in, x_out, conv, it, max_its);
    from_complex(yo, y_out);
    *its = it;
    *converged = conv ? 1 : 0;
    return 0;
}

// ShootingSolver::integrateToMatchPoint (src/ShootingSolver.cpp:53-145) on the
// grid of the given config; forward=1 marches iL->iM, forward=0 marches iR->iM.
int ref_sweep(const char* cfg_json, const double* y_init, int forward, double* y_final)
{
    SimulationConfig cfg = parse_cfg(cfg_json);
    NewtonSolver solver(cfg, ".", false);
    solver.generateGrid();
    InitialConditionGenerator g(cfg.Ntau, cfg.Dim, y_init[4]);
    ShootingSolver sh((int)cfg.Ntau, cfg.Dim, cfg.PrecisionIRK, g, cfg.MaxIterIRK, cfg.SchemeIRK);
    vec_complex yi, yo;
    to_complex(y_init, cfg.Ntau / 2, yi);
    cfg.Debug = false;
    if (forward)
        sh.integrateToMatchPoint(yi, solver.XGrid, solver.iL, solver.iM, true, yo, &cfg, nullptr);
    else
        sh.integrateToMatchPoint(yi, solver.XGrid, solver.iR, solver.iM, false, yo, &cfg, nullptr);
    from_complex(yo, y_final);
    return 0;
}

// NewtonSolver::generateGrid (src/NewtonSolver.cpp:477-519); grid_out has NLeft+NRight+1 entries.
int ref_grid(const char* cfg_json, double* grid_out)
{
    SimulationConfig cfg = parse_cfg(cfg_json);
    NewtonSolver solver(cfg, ".", false);
    solver.generateGrid();
    for (size_t i = 0; i < solver.XGrid.size(); ++i) grid_out[i] = solver.XGrid[i];
    return (int)solver.XGrid.size();
}

// NewtonSolver::shoot (src/NewtonSolver.cpp:403-423): in0 -> out0 (Nnewton reals each).
int ref_shoot(const char* cfg_json, const double* in0, double* out0)
{
    SimulationConfig cfg = parse_cfg(cfg_json);
    cfg.Debug = false;
    cfg.Verbose = false;
    NewtonSolver solver(cfg, ".", false);
    solver.generateGrid();
    vec_real in(in0, in0 + solver.Nnewton), out(solver.Nnewton);
    solver.shoot(in, out);
    for (size_t i = 0; i < solver.Nnewton; ++i) out0[i] = out[i];
    return 0;
}

// The OpenMP branch of NewtonSolver::assembleJacobian (src/NewtonSolver.cpp:619-666)
// restricted to columns [c0, c1): thread-local generator and shooter, the
// reference's own per-thread shoot (:439-459).  cols_out is column-major:
// cols_out[(c - c0) * Nnewton + row] = J[row][c].
int ref_jacobian_columns(const char* cfg_json, const double* in0, const double* out0, int c0, int c1,
                         double* cols_out, int nthreads)
{
    SimulationConfig cfg = parse_cfg(cfg_json);
    cfg.Debug = false;
    cfg.Verbose = false;
    NewtonSolver solver(cfg, ".", false);
    solver.generateGrid();
    const size_t nn = solver.Nnewton;
    const size_t ntau = cfg.Ntau;
    vec_real base_in(in0, in0 + nn), base_out(out0, out0 + nn);
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel
    {
        vec_complex yl(ntau), yr(ntau), mm(ntau);
        InitialConditionGenerator g(ntau, cfg.Dim, cfg.Delta);
        ShootingSolver sh((int)ntau, cfg.Dim, cfg.PrecisionIRK, g, cfg.MaxIterIRK, cfg.SchemeIRK);
#pragma omp for schedule(static)
        for (int c = c0; c < c1; ++c) {
            vec_real pin = base_in;
            pin[c] += cfg.EpsNewton;
            vec_real pout(nn);
            solver.shoot(pin, pout, sh, g, yl, yr, mm);
            for (size_t j = 0; j < nn; ++j) cols_out[(size_t)(c - c0) * nn + j] = (pout[j] - base_out[j]) / cfg.EpsNewton;
        }
    }
    return 0;
}

// NewtonSolver::solveLinearSystem (src/NewtonSolver.cpp:739-757): LAPACKE_dgesv
// on the row-major matrix a (n*n), right-hand side rhs; x receives the solution.
int ref_solve(int n, const double* a, const double* rhs, double* x)
{
    mat_real A(n, vec_real(n));
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) A[i][j] = a[(size_t)i * n + j];
    vec_real b(rhs, rhs + n), dx(n);
    // solveLinearSystem only reads Nnewton from the object; build a minimal one.
    json j = {{"Ntau", 4 * n / 3}, {"Dim", 4.0}, {"XLeft", 0.001}, {"XMid", 0.1}, {"XRight", 0.999},
              {"EpsNewton", 1e-8}, {"PrecisionNewton", 1e-14}, {"SlowError", 1e-3}, {"MaxIterNewton", 1},
              {"Verbose", false}, {"Debug", false}, {"Converged", false}, {"NLeft", 2}, {"NRight", 2},
              {"PrecisionIRK", 1e-15}, {"SchemeIRK", 2}, {"MaxIterIRK", 10}, {"DebugNx", nullptr},
              {"DebugNtau", nullptr},
              {"Initial_Conditions", {{"Delta", 3.0}, {"fc", nullptr}, {"psic", nullptr}, {"Up", nullptr}}}};
    SimulationConfig cfg(j);
    NewtonSolver solver(cfg, ".", false);
    solver.Nnewton = (size_t)n;
    solver.solveLinearSystem(A, b, dx);
    for (int i = 0; i < n; ++i) x[i] = dx[i];
    return 0;
}

}  // extern "C"
