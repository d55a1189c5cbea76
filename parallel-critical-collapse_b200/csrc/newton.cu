// newton.cu -- the Newton iteration of NewtonSolver::run (NewtonSolver.cpp:
// 279-366) kept on the device: the mismatch norm and convergence test of the
// base shoot, the divergence safeguard (five mismatch increases stop the solve
// at the last improving iterate), the right-hand side -out0 and the damped
// update in0 += min(1, SlowError/err) dx.  The host only reads the small
// NewtonDev record of each solve to decide whether to continue.
#include "pcc_internal.h"

namespace pcc {

namespace {

constexpr int kNewtonThreads = 1024;

// Sum of squares in index order per thread, then a fixed-shape tree: the same
// inputs always give the same bits.
__device__ double block_sum_sq(const double* __restrict__ v, int n, double* red)
{
    double s = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) s = fma(v[i], v[i], s);
    red[threadIdx.x] = s;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    const double r = red[0];
    __syncthreads();
    return r;
}

__device__ int block_any(const int* __restrict__ v, int n, int* flag)
{
    if (threadIdx.x == 0) *flag = 0;
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x)
        if (v[i] != 0) *flag = 1;
    __syncthreads();
    const int r = *flag;
    __syncthreads();
    return r;
}

__global__ void __launch_bounds__(kNewtonThreads) newton_reset_kernel(NewtonDev* nd, const double* __restrict__ in0,
                                                                     double* __restrict__ in0old, int nn)
{
    if (threadIdx.x == 0) {
        nd->err = 1.0;  // fac = 1, err = 1, errOld = 1 (NewtonSolver.cpp:270)
        nd->err_old = 1.0;
        nd->its = 0;
        nd->inc_count = 0;
        nd->state = kNewtonRunning;
        nd->fail_item = -1;
    }
    for (int i = threadIdx.x; i < nn; i += blockDim.x) in0old[i] = in0[i];
}

// After the shoots of one iteration: march and epilogue statuses, then
// NewtonSolver.cpp:285-325 on the base shoot out0.
__global__ void __launch_bounds__(kNewtonThreads) newton_check_kernel(NewtonDev* nd, const double* __restrict__ out0,
                                                                     int nn, const int* __restrict__ sweep_status,
                                                                     const int* __restrict__ col_status,
                                                                     double tol, double* __restrict__ rhs)
{
    __shared__ double red[kNewtonThreads];
    __shared__ int flag;
    if (nd->state != kNewtonRunning) return;
    const int bad_sweep = block_any(sweep_status, 2 * (nn + 1), &flag);
    const int bad_col = block_any(col_status, nn + 1, &flag);
    const double err = sqrt(block_sum_sq(out0, nn, red) / (double)nn);  // computeL2Norm (:763-768)
    for (int i = threadIdx.x; i < nn; i += blockDim.x) rhs[i] = -out0[i];
    if (threadIdx.x == 0) {
        nd->its += 1;
        if (bad_sweep || bad_col) {
            nd->state = bad_sweep ? kNewtonIrkFailed : kNewtonDeltaMismatch;
            return;
        }
        const double err_old = nd->err;
        nd->err_old = err_old;
        nd->err = err;
        if (err < tol) {
            nd->state = kNewtonConverged;
        } else {
            if (log10(err) > log10(err_old)) nd->inc_count += 1;
            if (nd->inc_count >= 5) nd->state = kNewtonStopped;
        }
    }
}

// NewtonSolver.cpp:344-358 for a solve still running after its check.
__global__ void __launch_bounds__(kNewtonThreads) newton_update_kernel(NewtonDev* nd, double* __restrict__ in0,
                                                                      double* __restrict__ in0old,
                                                                      const double* __restrict__ dx,
                                                                      const int* __restrict__ lu_info, int nn,
                                                                      double slow_error, int max_its)
{
    if (nd->state != kNewtonRunning) return;
    if (lu_info[0] != 0) {
        __syncthreads();
        if (threadIdx.x == 0) nd->state = kNewtonSingular;
        return;
    }
    const double err = nd->err, err_old = nd->err_old;
    const double fac = fmin(1.0, slow_error / err);
    const bool improved = log10(err) < log10(err_old);
    for (int i = threadIdx.x; i < nn; i += blockDim.x) {
        if (improved) in0old[i] = in0[i];
        in0[i] += fac * dx[i];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        if (improved) nd->inc_count = 0;
        if (nd->its >= max_its) nd->state = kNewtonMaxIter;
    }
}

}  // namespace

cudaError_t launch_newton_reset(NewtonDev* nd, const double* in0, double* in0old, int nn, cudaStream_t st)
{
    newton_reset_kernel<<<1, kNewtonThreads, 0, st>>>(nd, in0, in0old, nn);
    return cudaGetLastError();
}

cudaError_t launch_newton_check(NewtonDev* nd, const double* out0, int nn, const int* sweep_status,
                                const int* col_status, double tol, double* rhs, cudaStream_t st)
{
    newton_check_kernel<<<1, kNewtonThreads, 0, st>>>(nd, out0, nn, sweep_status, col_status, tol, rhs);
    return cudaGetLastError();
}

cudaError_t launch_newton_update(NewtonDev* nd, double* in0, double* in0old, const double* dx, const int* lu_info,
                                 int nn, double slow_error, int max_its, cudaStream_t st)
{
    newton_update_kernel<<<1, kNewtonThreads, 0, st>>>(nd, in0, in0old, dx, lu_info, nn, slow_error, max_its);
    return cudaGetLastError();
}

}  // namespace pcc
