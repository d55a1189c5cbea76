// boundary.cuh -- the cold kernels around the IRK march: boundary data before
// it (unpackSpectralFields + the left/right Taylor expansions, as
// NewtonSolver::shoot runs them, NewtonSolver.cpp:403-432) and the mismatch,
// field reconstruction, packing and finite differencing after it
// (ShootingSolver::computeMismatch, ShootingSolver.cpp:154-182;
// NewtonSolver.cpp:421-422 and :642-645).
//
// These follow the reference algorithm literally with full-length (Ntau-point)
// transforms: about 45 FFTs per shoot against ~10^5-10^6 in the march, so they
// are a fraction of a percent of the time.  One CTA per work item; a
// radix-2 Stockham FFT in shared memory; N-length work arrays in a per-CTA
// global scratch slab (L2 resident).
#pragma once
#include "pcc_device.cuh"

namespace pcc {

// number of N-length real work arrays a CTA of the boundary kernels uses
constexpr int kBoundaryArrays = 40;

struct Blk {
    int n;
    const double2* __restrict__ tw;  // exp(+2 pi i k/n)
    double2* sa;                     // shared, n complex: transform data
    double2* sb;                     // shared, n complex: Stockham partner
    double* scr;                     // global slab, kBoundaryArrays * n doubles

    __device__ double* arr(int i) const { return scr + (size_t)i * n; }
    __device__ static void sync() { __syncthreads(); }

    // unnormalised DFT of sa in place: sa[k] = sum_j sa[j] exp(sign 2 pi i jk/n)
    __device__ void fft(int sign) const
    {
        double2* src = sa;
        double2* dst = sb;
        const int h = n / 2;
        for (int l = 1; l < n; l <<= 1) {
            const int step = n / (2 * l);
            for (int j = threadIdx.x; j < h; j += blockDim.x) {
                const int k = j & (l - 1);
                const int g = j / l;
                double2 w = tw[k * step];
                if (sign < 0) w.y = -w.y;
                const double2 a = src[j];
                const double2 b = cmul(w, src[j + h]);
                dst[g * 2 * l + k] = cadd(a, b);
                dst[g * 2 * l + k + l] = csub(a, b);
            }
            sync();
            double2* t = src;
            src = dst;
            dst = t;
        }
        if (src != sa) {
            for (int j = threadIdx.x; j < n; j += blockDim.x) sa[j] = src[j];
            sync();
        }
    }
    // SpectralTransformer::forwardFFT (SpectralTransformer.cpp:57-72, 97-112): e^{+i}, / N
    __device__ void forward() const
    {
        fft(+1);
        const double inv = 1.0 / n;
        for (int j = threadIdx.x; j < n; j += blockDim.x) sa[j] = cscale(sa[j], inv);
        sync();
    }
    // SpectralTransformer::backwardFFT (:77-92, 117-132): e^{-i}, unscaled
    __device__ void backward() const { fft(-1); }
    __device__ void load_real(const double* x) const
    {
        for (int j = threadIdx.x; j < n; j += blockDim.x) sa[j] = make_double2(x[j], 0.0);
        sync();
    }
    __device__ void store_real(double* x) const
    {
        for (int j = threadIdx.x; j < n; j += blockDim.x) x[j] = sa[j].x;
        sync();
    }
    // SpectralTransformer::differentiate (:140-158)
    __device__ void differentiate(double period) const
    {
        const double k0c = 2.0 * kPi / period;
        for (int k = threadIdx.x; k < n; k += blockDim.x) {
            if (k != n / 2) {
                const int m = k < n / 2 ? k : k - n;
                const double s = m * k0c;
                const double2 a = sa[k];
                sa[k] = make_double2(s * a.y, -(s * a.x));
            } else {
                sa[k] = make_double2(0.0, 0.0);
            }
        }
        sync();
    }
    // SpectralTransformer::lamIntegrate (:165-189) with real lambda
    __device__ void lam_integrate(double lam, double period) const
    {
        const double k0c = 2.0 * kPi / period;
        for (int k = threadIdx.x; k < n; k += blockDim.x) {
            const double2 f = sa[k];
            double2 o;
            if (k == 0) {
                o = lam != 0.0 ? cdiv(f.x, f.y, lam, 0.0) : make_double2(0.0, 0.0);
            } else if (k != n / 2) {
                const int m = k < n / 2 ? k : k - n;
                const double dr = lam - 0.0, di = 0.0 - m * k0c;
                o = hypot(dr, di) < 1e-14 ? make_double2(0.0, 0.0) : cdiv(f.x, f.y, dr, di);
            } else {
                const double s = k0c * n / 2.0;
                const double2 q = cdiv(lam, 0.0, lam * lam - 0.0 * 0.0 + s * s, lam * 0.0 + 0.0 * lam);
                o = cmul(q, f);
            }
            sa[k] = o;
        }
        sync();
    }
    // forwardFFT -> differentiate -> backwardFFT of a real series
    __device__ void tau_derivative(const double* in, double* out, double period) const
    {
        load_real(in);
        forward();
        differentiate(period);
        backward();
        store_real(out);
    }
    // SpectralTransformer::solveInhom (:264-292); uses work arrays fr, hh
    __device__ void solve_inhom(const double* f, const double* g, double* x, double period, double* fr) const
    {
        load_real(f);
        forward();
        const double lam = sa[0].x;  // f_hat[0]; its imaginary part is exactly zero
        sync();
        lam_integrate(0.0, period);
        backward();
        store_real(fr);
        for (int j = threadIdx.x; j < n; j += blockDim.x) sa[j] = make_double2(-g[j] * exp(fr[j]), 0.0);
        sync();
        forward();
        lam_integrate(lam, period);
        backward();
        for (int j = threadIdx.x; j < n; j += blockDim.x) x[j] = sa[j].x * exp(-fr[j]);
        sync();
    }
    // InitialConditionGenerator::FieldsToStateVector (InitialConditionGenerator.cpp:766-778)
    // y: n/2 complex, interleaved
    __device__ void fields_to_state(const double* u, const double* v, const double* f, double* y) const
    {
        for (int j = threadIdx.x; j < n; j += blockDim.x) sa[j] = make_double2(u[j], v[j] + f[j]);
        sync();
        forward();
        const int no = n / 2;
        for (int k = threadIdx.x; k < no; k += blockDim.x) {
            double2 val;
            if (k < no / 2)
                val = sa[k];
            else if (k == no / 2)
                val = cadd(sa[no / 2], sa[3 * no / 2]);
            else
                val = sa[no + k];
            y[2 * k] = val.x;
            y[2 * k + 1] = val.y;
        }
        sync();
    }
};

// SpectralTransformer::doubleModes (SpectralTransformer.cpp:224-252), element k
// of the doubled spectrum of `in` (n_in complex), with its store order: the
// upper-half copy overwrites out[3 n_in/2] with the full in[n_in/2].
__device__ __forceinline__ double2 double_modes_at(const double2* in, int n_in, int k)
{
    if (k < n_in / 2) return in[k];
    if (k == n_in / 2) return make_double2(0.5 * in[k].x, 0.5 * in[k].y);
    if (k < 3 * n_in / 2) return make_double2(0.0, 0.0);
    return in[k - n_in];
}

// Which sides of the shoot of column col read the perturbed free datum: the
// left expansion reads the psi_c and f_c blocks z[nn/3, nn) and Delta, the
// right expansion the U_p block z[0, nn/3) and Delta (Delta sits at
// z[2 nn/3 + 2]); column nn is the unperturbed base shoot.  A side that does
// not read the datum starts from the base shoot's boundary state bit for bit,
// so its final state is the base shoot's.
__host__ __device__ __forceinline__ bool column_moves_left(int col, int nn) { return col >= nn / 3; }
__host__ __device__ __forceinline__ bool column_moves_right(int col, int nn)
{
    return col < nn / 3 || col == 2 * nn / 3 + 2 || col >= nn;
}

struct BoundaryParams {
    int n_items;        // prologue: sweeps (2 per column, or sweeps[] entries); epilogue: 1 per column
    int ntau, nn;       // Ntau, Nnewton
    int c0;             // first column of this batch (Nnewton = the unperturbed base shoot)
    double dim, xl, xr, eps, prec;
    double dim_m2_cubed;
    const double* __restrict__ in0;   // Nnewton
    const double* __restrict__ out0;  // Nnewton (finite differencing)
    // Sweep slots.  Prologue: with sweeps == null item i is column c0 + i/2,
    // side i & 1, at slot i; else item i is slot sweeps[i] (2 column + side,
    // absolute).  Epilogue: with abs_slots == 0 column c0 + i reads slots 2i
    // and 2i + 1; else column col reads slots 2 col (left) and 2 col + 1
    // (right), or, with reuse set, the base column's slot of each side col
    // does not move.
    const int* sweeps;
    int abs_slots, reuse;
    double* yinit;                    // [slot][N]   (prologue output)
    const double* yfinal;             // [slot][N]   (epilogue input)
    double* outc;                     // [col][Nnewton] packed mismatch per column
    int* status;                      // [col] epilogue: 0 or PCC_ERR_DELTA_MISMATCH
    double* scratch;                  // gridDim.x * kBoundaryArrays * N
    const double2* __restrict__ tw;
    int* work_counter;
};

}  // namespace pcc
