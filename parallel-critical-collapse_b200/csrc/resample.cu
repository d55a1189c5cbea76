// resample.cu -- spectral doubling of periodic fields: the reference's
// scripts/create_simulation_data.py:37-58 (double), which refines initial data
// from Ntau to 2 Ntau points for convergence studies.  Per doubling:
//   F = DFT_n(x) (e^{-i} convention), mode map n -> 2n, x' = 2 Re IDFT_2n(F')/(2n).
// The mode map is the script's, including its omission of mode n/2-1.
#include "pcc_internal.h"

namespace pcc {

namespace {

__global__ void real_to_complex_kernel(const double* __restrict__ in, double2* __restrict__ out, int total)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x)
        out[i] = make_double2(in[i], 0.0);
}

// doubled[:n/2-1] = F[:n/2-1]; doubled[n/2] = doubled[3n/2] = F[n/2]/2;
// doubled[3n/2+1:] = F[n/2+1:]; everything else zero.
__global__ void double_modes_kernel(const double2* __restrict__ F, double2* __restrict__ D, int n, int count)
{
    const int m = 2 * n;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count * m; i += gridDim.x * blockDim.x) {
        const int f = i / m, k = i % m;
        const double2* src = F + (size_t)f * n;
        double2 v = make_double2(0.0, 0.0);
        if (k < n / 2 - 1) {
            v = src[k];
        } else if (k == n / 2 || k == 3 * n / 2) {
            v = make_double2(src[n / 2].x / 2.0, src[n / 2].y / 2.0);
        } else if (k > 3 * n / 2) {
            v = src[k - n];
        }
        D[i] = v;
    }
}

__global__ void real_scale_kernel(const double2* __restrict__ X, double* __restrict__ out, int total, double scale)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x)
        out[i] = scale * X[i].x;
}

int blocks_for(int total) { return total < 256 ? 1 : (total + 255) / 256 > 4096 ? 4096 : (total + 255) / 256; }

}  // namespace

cudaError_t launch_double_fields(int n, int count, const double* in, double* out, const double2* tw_n,
                                 const double2* tw_2n, double2* w0, double2* w1, cudaStream_t st)
{
    const int tn = n * count, t2 = 2 * n * count;
    real_to_complex_kernel<<<blocks_for(tn), 256, 0, st>>>(in, w0, tn);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = launch_dft(n, count, -1, tw_n, w0, w1, st);
    if (e != cudaSuccess) return e;
    double_modes_kernel<<<blocks_for(t2), 256, 0, st>>>(w1, w0, n, count);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if ((e = launch_dft(2 * n, count, 1, tw_2n, w0, w1, st)) != cudaSuccess) return e;
    // np.sqrt(4) * ifft = 2 / (2n) * unscaled inverse transform, real part
    real_scale_kernel<<<blocks_for(t2), 256, 0, st>>>(w1, out, t2, 2.0 / (2.0 * n));
    return cudaGetLastError();
}

}  // namespace pcc
