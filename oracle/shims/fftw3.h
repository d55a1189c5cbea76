/*
 * fftw3.h -- stand-in for the subset of the FFTW3 API that the reference
 * solver uses (SpectralTransformer.cpp:25-50 of tobjec/parallel-critical-collapse).
 *
 * TEST INFRASTRUCTURE ONLY.  libfftw3 is not installed in this image, so the
 * oracle recipe (oracle/build_ref.sh) compiles the reference sources against
 * this header and fftw_shim.cpp.  The transform is FFTW's unnormalised DFT
 *     out[k] = sum_j in[j] * exp(sign * 2*pi*i * j*k / n)
 * computed by an iterative radix-2 Cooley-Tukey (every Ntau in the reference
 * is a power of two); other lengths fall back to a direct O(n^2) sum.
 * Rounding therefore differs from a real FFTW run at the 1e-16 level.
 */
#pragma once
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef double fftw_complex[2];
typedef struct pcc_fftw_plan_s* fftw_plan;

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_MEASURE (0U)
#define FFTW_ESTIMATE (1U << 6)

fftw_complex* fftw_alloc_complex(size_t n);
void fftw_free(void* p);
fftw_plan fftw_plan_dft_1d(int n, fftw_complex* in, fftw_complex* out, int sign, unsigned flags);
void fftw_execute(const fftw_plan plan);
void fftw_destroy_plan(fftw_plan plan);

#ifdef __cplusplus
}
#endif
