// pcc_internal.h -- declarations shared by the CUDA translation units.
#pragma once
#include <cuda_runtime.h>

#include "boundary.cuh"
#include "march.cuh"

namespace pcc {

cudaError_t launch_prologue(const BoundaryParams& P, int ctas, cudaStream_t st);
cudaError_t launch_epilogue(const BoundaryParams& P, int ctas, cudaStream_t st);
cudaError_t launch_pack(int ntau, const double2* tw, double* scratch, double* up, double* psic, double* fc, double* z,
                        int dir, cudaStream_t st);
cudaError_t launch_expansions(int ntau, double dim, double delta, double xl, double xr, const double2* tw,
                              double* scratch, const double* fc, const double* psic, const double* up, double* yl,
                              double* yr, cudaStream_t st);
cudaError_t launch_dft(int n, int count, int sign, const double2* tw, const double2* in, double2* out,
                       cudaStream_t st);
// One spectral doubling of count periodic fields of n samples (resample.cu):
// out has count x 2n values; tw_n / tw_2n are exp(+2 pi i k/m) tables and
// w0, w1 work arrays of count x 2n complex values.
cudaError_t launch_double_fields(int n, int count, const double* in, double* out, const double2* tw_n,
                                 const double2* tw_2n, double2* w0, double2* w1, cudaStream_t st);
// Debug field export: count state snapshots at xs -> fields [count][4][ntau] = A, U, V, f.
cudaError_t launch_debug_fields(int ntau, double dim, double dm2c, int count, const double* states, const double* xs,
                                double* fields, double* scratch, int ctas, const double2* tw, cudaStream_t st);
cudaError_t launch_fd_cols(const double* outc, const double* out0, double* cols, int nn, int ncols, double eps,
                           cudaStream_t st);
cudaError_t launch_fd(const double* outc, const double* out0, double* J, int nn, int c0, int ncols, double eps,
                      cudaStream_t st);

struct MarchLaunchInfo {
    int ctas;            // persistent CTAs launched
    int sweeps_per_cta;  // sweep slots per CTA
    int threads;         // threads per CTA
    size_t smem;         // dynamic shared memory per CTA
    int ctas_per_sm;     // resident CTAs per SM at this shape
};

// Launches the IRK march for Ntau in {128,...,2048} and 1..3 stages.
// max_ctas <= 0 means one wave of resident CTAs on every SM.
cudaError_t launch_march(int ntau, int stages, const MarchParams& P, int max_ctas, cudaStream_t st,
                         MarchLaunchInfo* info);
bool march_supported(int ntau, int stages);

// The autotuned transform schedule of the march for one (device, Ntau,
// stages): paired transforms (dft_m2) or single ones, with the probe times.
struct MarchTuning {
    int pair;          // 0 single, 1 paired, 2 paired with the warp-exchange transforms (Ntau 1024)
    double ms_pair;    // probe time of each schedule (ms), 0 when set from a cache or not available
    double ms_single;
    double ms_wx;
};
bool march_tuning(int device, int ntau, int stages, MarchTuning* out);
void march_set_tuning(int device, int ntau, int stages, const MarchTuning& t);
// Times the schedules on the current device and records the choice.
cudaError_t march_autotune(int ntau, int stages, const double2* tw, cudaStream_t st, MarchTuning* out);

// Sweeps of several solves in one persistent launch (march_batch_kernel):
// Ntau in {128, 256, 512, 1024} with 2 stages.  B.cls_counter must be zero.
cudaError_t launch_march_batch(const BatchParams& B, int max_ctas, cudaStream_t st, MarchLaunchInfo* info);
bool march_batch_supported(int ntau, int stages);

// Device-resident Newton state of one solve (newton.cu).
enum NewtonStateCode {
    kNewtonRunning = 0,
    kNewtonConverged = 1,     // err < PrecisionNewton
    kNewtonStopped = 2,       // five mismatch increases: the last improving iterate is the result
    kNewtonMaxIter = 3,       // MaxIterNewton iterations without convergence
    kNewtonIrkFailed = 4,     // a sweep's IRK iteration did not converge
    kNewtonDeltaMismatch = 5, // the two sides' Delta differ
    kNewtonSingular = 6       // zero pivot in the Newton solve
};

struct NewtonDev {
    double err;       // mismatch RMS of the last base shoot
    double err_old;   // of the one before
    int its;          // iterations whose base shoot was evaluated
    int inc_count;    // mismatch increases since the last improvement
    int state;        // NewtonStateCode
    int fail_item;
};

cudaError_t launch_newton_reset(NewtonDev* nd, const double* in0, double* in0old, int nn, cudaStream_t st);
cudaError_t launch_newton_check(NewtonDev* nd, const double* out0, int nn, const int* sweep_status,
                                const int* col_status, double tol, double* rhs, cudaStream_t st);
cudaError_t launch_newton_update(NewtonDev* nd, double* in0, double* in0old, const double* dx, const int* lu_info,
                                 int nn, double slow_error, int max_its, cudaStream_t st);

// LU helpers (lu.cu)
cudaError_t lu_solve_fp64(const double* dA, const double* db, double* dx, int n, double* work, int* ipiv,
                          int* info, cudaStream_t st);
cudaError_t lu_solve_mixed(const double* dA, const double* db, double* dx, int n, void* work, size_t work_bytes,
                           int* ipiv, int* info, int max_refine, double tol, int* steps_out, double* resid_out,
                           cudaStream_t st);
size_t lu_mixed_work_bytes(int n);
int lu_max_order();  // largest n the LU takes (its panel lives in shared memory)

cudaError_t fp64_peak_probe(double* tflops, cudaStream_t st);

}  // namespace pcc

// accessors of the opaque context (pcc_abi.cu)
struct pcc_ctx;
cudaStream_t pcc_ctx_stream(pcc_ctx* ctx);
int pcc_ctx_device(pcc_ctx* ctx);
void pcc_ctx_set_error(pcc_ctx* ctx, const char* msg);
