/*
 * pcc_oracle.h -- CPU restatement of the reference's Newton-shooting path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the oracle that the CUDA path is checked
 * against: a plain-C restatement of tobjec/parallel-critical-collapse's
 * SpectralTransformer, InitialConditionGenerator, ODEStepper, ShootingSolver
 * and NewtonSolver (Jacobian + dense solve), each function citing the
 * reference file:line it follows.  It is pinned against the reference's own
 * golden vectors (test/test_init_gen.cpp) and against the compiled reference
 * (oracle/_ref, built by oracle/build_ref.sh) through tests/golden fixtures.
 * Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg may
 * load it; the product never does.
 *
 * Conventions: real_t = double; complex values are {re, im} pairs; a state Y
 * of the shooting march holds Ntau/2 complex Fourier modes, stored interleaved
 * as Ntau reals ("Yreal" in ODEStepper.cpp:92-136) with Re Y[2] = Delta.
 */
#pragma once
#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int ntau;            /* Ntau, power of two */
    double dim;          /* D */
    double xl, xm, xr;   /* XLeft, XMid, XRight */
    double eps_newton;   /* EpsNewton */
    int nl, nr;          /* NLeft, NRight */
    double prec_irk;     /* PrecisionIRK */
    int scheme;          /* SchemeIRK: 1, 2 or 3 stages */
    int max_irk;         /* MaxIterIRK */
} orc_cfg;

/* status codes (the reference calls std::exit on each of these) */
enum { ORC_OK = 0, ORC_IRK_NO_CONVERGENCE = 1, ORC_DELTA_MISMATCH = 2, ORC_SINGULAR = 3, ORC_BAD_ARG = 4 };

/* SpectralTransformer (src/SpectralTransformer.cpp) ------------------------ */
void orc_dft(int n, double* data, int sign);                       /* FFTW-style unnormalised DFT, in place */
void orc_forward_real(int n, const double* in, double* out);      /* :57-72, e^{+i}, /N */
void orc_backward_real(int n, const double* in, double* out);     /* :77-92, e^{-i}, real part */
void orc_differentiate(int n, const double* in, double* out, double period);       /* :140-158 */
void orc_lam_integrate(int n, const double* fk, double* out, const double* lambda, double period); /* :165-189 */
void orc_halve_modes(int n_in, const double* in, double* out);    /* :196-217 */
void orc_double_modes(int n_in, const double* in, double* out);   /* :224-252 */
void orc_solve_inhom(int n, const double* f, const double* g, double* x, double period); /* :264-292 */

/* InitialConditionGenerator (src/InitialConditionGenerator.cpp) ----------- */
void orc_left_expansion(int n, double dim, double xl, const double* fc, const double* psic, double delta,
                        double* y);                                /* :37-239 */
void orc_right_expansion(int n, double dim, double xr, const double* up, double delta, double* y); /* :252-667 */
void orc_pack(int n, const double* odd1, const double* odd2, const double* even, double* z);      /* :678-711 */
void orc_unpack(int n, const double* z, double* odd1, double* odd2, double* even);               /* :719-758 */
void orc_fields_to_state(int n, const double* u, const double* v, const double* f, double* y);   /* :766-778 */
void orc_state_to_fields(int n, double dim, const double* y, double x, double* u, double* v, double* f,
                         double* ia2, double* dudt, double* dvdt, double* dfdt);                  /* :791-884 */
void orc_state_to_fields_light(int n, const double* y, double* u, double* v, double* f);        /* :891-932 */

/* ODEStepper (src/ODEStepper.cpp) ----------------------------------------- */
void orc_rhs(int n, double dim, const double* yreal, double x, double* dyreal); /* :92-136 */
int orc_irk_step(int n, double dim, int scheme, double precision, int max_its, const double* yin,
                 double xin, double xout, double* yout, int* its); /* :163-292; returns 1 if converged */

/* ShootingSolver (src/ShootingSolver.cpp) --------------------------------- */
int orc_sweep(const orc_cfg* c, const double* grid, int start, int end, int forward, const double* yinit,
              double* yfinal, int* fail_index, long long* rhs_evals); /* :53-145 */
int orc_mismatch(int n, const double* yl, const double* yr, double precision, double* out); /* :154-182 */

/* NewtonSolver (src/NewtonSolver.cpp) ------------------------------------- */
void orc_grid(const orc_cfg* c, double* grid);                              /* :477-519 */
int orc_shoot(const orc_cfg* c, const double* grid, const double* in0, double* out0,
              long long* rhs_evals);                                        /* :403-423 */
int orc_jacobian_columns(const orc_cfg* c, const double* grid, const double* in0, const double* out0, int c0,
                         int c1, double* cols, long long* rhs_evals);       /* :615-702, column-major */
int orc_dgesv(int n, double* a_rowmajor, double* b);                        /* :739-757 (LAPACK dgesv) */
double orc_rms(int n, const double* v);                                     /* :763-768 */

#ifdef __cplusplus
}
#endif
