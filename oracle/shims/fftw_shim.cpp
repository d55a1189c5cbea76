// fftw_shim.cpp -- TEST INFRASTRUCTURE ONLY (see fftw3.h).
// Implements the FFTW3 calls the reference's SpectralTransformer makes
// (SpectralTransformer.cpp:25-50): plan creation bound to fixed in/out arrays,
// execution, destruction and aligned allocation.  Radix-2 decimation in time
// for powers of two, with twiddles rounded from long-double cos/sin.
#include "fftw3.h"

#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

struct pcc_fftw_plan_s {
    int n;
    int sign;
    fftw_complex* in;
    fftw_complex* out;
    std::vector<double> twr, twi;  // exp(sign*2*pi*i*k/n), k < n/2
    std::vector<int> rev;          // bit reversal permutation
    std::vector<double> scratch;   // for the in==out case
};

extern "C" fftw_complex* fftw_alloc_complex(size_t n)
{
    void* p = nullptr;
    if (posix_memalign(&p, 64, n * sizeof(fftw_complex)) != 0) return nullptr;
    return static_cast<fftw_complex*>(p);
}

extern "C" void fftw_free(void* p) { std::free(p); }

static bool is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

extern "C" fftw_plan fftw_plan_dft_1d(int n, fftw_complex* in, fftw_complex* out, int sign, unsigned)
{
    auto* p = new pcc_fftw_plan_s;
    p->n = n;
    p->sign = sign;
    p->in = in;
    p->out = out;
    const long double two_pi = 6.283185307179586476925286766559005768L;
    int half = n / 2 > 0 ? n / 2 : 1;
    p->twr.resize(half);
    p->twi.resize(half);
    for (int k = 0; k < half; ++k) {
        long double a = two_pi * (long double)k / (long double)n;
        p->twr[k] = (double)cosl(a);
        p->twi[k] = (double)(sign > 0 ? sinl(a) : -sinl(a));
    }
    if (is_pow2(n)) {
        int bits = 0;
        while ((1 << bits) < n) ++bits;
        p->rev.resize(n);
        for (int i = 0; i < n; ++i) {
            int r = 0;
            for (int b = 0; b < bits; ++b)
                if (i & (1 << b)) r |= 1 << (bits - 1 - b);
            p->rev[i] = r;
        }
    }
    p->scratch.resize(2 * (size_t)n);
    return p;
}

extern "C" void fftw_execute(const fftw_plan p)
{
    const int n = p->n;
    double* s = p->scratch.data();
    for (int i = 0; i < n; ++i) {
        s[2 * i] = p->in[i][0];
        s[2 * i + 1] = p->in[i][1];
    }
    if (!is_pow2(n)) {
        const long double two_pi = 6.283185307179586476925286766559005768L;
        for (int k = 0; k < n; ++k) {
            long double ar = 0, ai = 0;
            for (int j = 0; j < n; ++j) {
                long double a = two_pi * (long double)(((long long)j * k) % n) / n;
                long double c = cosl(a), sn = p->sign > 0 ? sinl(a) : -sinl(a);
                ar += s[2 * j] * c - s[2 * j + 1] * sn;
                ai += s[2 * j] * sn + s[2 * j + 1] * c;
            }
            p->out[k][0] = (double)ar;
            p->out[k][1] = (double)ai;
        }
        return;
    }
    for (int i = 0; i < n; ++i) {
        p->out[p->rev[i]][0] = s[2 * i];
        p->out[p->rev[i]][1] = s[2 * i + 1];
    }
    for (int len = 2; len <= n; len <<= 1) {
        const int h = len / 2;
        const int step = n / len;
        for (int base = 0; base < n; base += len) {
            for (int k = 0; k < h; ++k) {
                const double wr = p->twr[k * step], wi = p->twi[k * step];
                double* a = p->out[base + k];
                double* b = p->out[base + k + h];
                const double br = b[0] * wr - b[1] * wi;
                const double bi = b[0] * wi + b[1] * wr;
                b[0] = a[0] - br;
                b[1] = a[1] - bi;
                a[0] = a[0] + br;
                a[1] = a[1] + bi;
            }
        }
    }
}

extern "C" void fftw_destroy_plan(fftw_plan p) { delete p; }
