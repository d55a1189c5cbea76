// static_scratch.cu -- pcc_expansions_static: the boundary Taylor expansions
// (InitialConditionGenerator::computeLeftExpansion / computeRightExpansion)
// without any device allocation.
//
// Who needs this: callers that reserve all of their device memory up front and
// may not call cudaMalloc/cudaFree afterwards -- for example a long-running
// solver service that sizes its memory pool at start-up, or a host library that
// must not trigger the implicit device-wide synchronisation cudaFree can cause.
// pcc_expansions allocates its work arrays per call; this entry point instead
// uses a fixed work area compiled into the library.
//
// The work area is the file-scope array below.  In host code its name is only a
// host-side stand-in, not a device address, so the address kernels receive is
// obtained once per device with cudaGetSymbolAddress (with that device current)
// and cached.  The array holds the two CTAs' expansion work arrays plus the
// twiddle table, for Ntau up to kStaticMaxNtau; every GPU that loads the library
// keeps it (1.3 MiB) until the process exits.
#include <mutex>

#include "pcc.h"
#include "pcc_internal.h"

namespace pcc {

namespace {

constexpr int kStaticMaxNtau = 2048;
constexpr size_t kStaticWork = 2 * (size_t)kBoundaryArrays * kStaticMaxNtau;  // doubles: 2 CTAs
constexpr size_t kStaticTw = 2 * (size_t)kStaticMaxNtau;                       // doubles: Ntau complex

static __device__ __align__(256) double g_static_scratch[kStaticWork + kStaticTw];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
double* g_addr[kMaxDevices] = {};

// exp(+2 pi i k/n) for k < n, written by the device into the static area.
// pcc_expansions takes the same table from the host (computed in long double
// and rounded); sincospi's results differ from it by at most about one ulp,
// which the 1e-12 parity check of the two entry points covers.
__global__ void static_twiddle_kernel(double2* tw, int n)
{
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        double s, c;
        sincospi(2.0 * (double)k / (double)n, &s, &c);
        tw[k] = make_double2(c, s);
    }
}

}  // namespace

}  // namespace pcc

using namespace pcc;

extern "C" pcc_status pcc_expansions_static(pcc_ctx* ctx, int ntau, double dim, double delta, double x_l, double x_r,
                                            const double* d_fc, const double* d_psic, const double* d_up,
                                            double* d_y_left, double* d_y_right)
{
    if (!ctx || (!d_y_left && !d_y_right) || (d_y_left && (!d_fc || !d_psic)) || (d_y_right && !d_up))
        return PCC_ERR_INVALID_ARG;
    if (ntau > kStaticMaxNtau) {
        pcc_ctx_set_error(ctx, "pcc_expansions_static: Ntau exceeds the static work area (2048)");
        return PCC_ERR_INVALID_ARG;
    }
    if (!march_supported(ntau, 2)) {
        pcc_ctx_set_error(ctx, "pcc_expansions_static: Ntau must be 128..2048, power of two");
        return PCC_ERR_INVALID_ARG;
    }
    const int dev = pcc_ctx_device(ctx);
    if (dev < 0 || dev >= kMaxDevices) {
        pcc_ctx_set_error(ctx, "pcc_expansions_static: device index out of range");
        return PCC_ERR_INVALID_ARG;
    }
    // the context's device is made current for the call and the caller's
    // current device is restored before returning
    int prev = -1;
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    struct Restore {
        int d;
        ~Restore()
        {
            if (d >= 0) cudaSetDevice(d);
        }
    } restore{prev};
    cudaError_t e = cudaSetDevice(dev);
    if (e != cudaSuccess) {
        pcc_ctx_set_error(ctx, cudaGetErrorString(e));
        return PCC_ERR_CUDA;
    }
    double* base = nullptr;
    {
        // set-up, once per device, with that device current: the device
        // address of the static array (its host-side name is not one)
        std::lock_guard<std::mutex> lock(g_mu);
        if (!g_addr[dev]) {
            void* p = nullptr;
            e = cudaGetSymbolAddress(&p, g_static_scratch);
            if (e != cudaSuccess || !p) {
                pcc_ctx_set_error(ctx, cudaGetErrorString(e));
                return PCC_ERR_CUDA;
            }
            g_addr[dev] = static_cast<double*>(p);
        }
        base = g_addr[dev];
    }
    cudaStream_t st = pcc_ctx_stream(ctx);
    double2* tw = reinterpret_cast<double2*>(base + kStaticWork);
    static_twiddle_kernel<<<(ntau + 255) / 256, 256, 0, st>>>(tw, ntau);
    e = cudaGetLastError();
    if (e == cudaSuccess) {
        // every work array is written before it is read, so nothing needs clearing
        e = launch_expansions(ntau, dim, delta, x_l, x_r, tw, base, d_fc, d_psic, d_up, d_y_left, d_y_right, st);
    }
    if (e != cudaSuccess) {
        pcc_ctx_set_error(ctx, cudaGetErrorString(e));
        return PCC_ERR_CUDA;
    }
    return PCC_OK;
}
