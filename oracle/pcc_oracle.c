/*
 * pcc_oracle.c -- TEST INFRASTRUCTURE ONLY: the CPU oracle for the CUDA
 * Newton-shooting path.  See pcc_oracle.h for scope and conventions.
 *
 * Every function restates one reference routine of
 * tobjec/parallel-critical-collapse (file:line cited at each definition) in
 * the same order of operations, so that differences to the compiled reference
 * stay at the level of FFT round-off.  Complex numbers are interleaved double
 * pairs; complex division follows libgcc's __divdc3 (Smith's method), which is
 * what std::complex<double> division in the reference compiles to.
 */
#include "pcc_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define RE(a, i) ((a)[2 * (i)])
#define IM(a, i) ((a)[2 * (i) + 1])

static const double PI = 3.14159265358979323846;

/* ------------------------------------------------------------------------ */
/* complex helpers                                                           */
/* ------------------------------------------------------------------------ */
static void cdiv(double a, double b, double c, double d, double* x, double* y)
{
    /* (a+ib)/(c+id), libgcc __divdc3 ordering */
    double ratio, denom;
    if (fabs(c) < fabs(d)) {
        ratio = c / d;
        denom = (c * ratio) + d;
        if (fabs(ratio) > 2.2250738585072014e-308) {
            *x = ((a * ratio) + b) / denom;
            *y = ((b * ratio) - a) / denom;
        } else {
            *x = ((c * (a / d)) + b) / denom;
            *y = ((c * (b / d)) - a) / denom;
        }
    } else {
        ratio = d / c;
        denom = (d * ratio) + c;
        if (fabs(ratio) > 2.2250738585072014e-308) {
            *x = ((b * ratio) + a) / denom;
            *y = (b - (a * ratio)) / denom;
        } else {
            *x = (a + (d * (b / c))) / denom;
            *y = (b - (d * (a / c))) / denom;
        }
    }
}

static double* dalloc(size_t n) { return (double*)calloc(n ? n : 1, sizeof(double)); }

/* ------------------------------------------------------------------------ */
/* DFT: FFTW's unnormalised transform out[k] = sum_j in[j] e^{sign 2 pi i jk/n}
 * (the library behind SpectralTransformer.cpp:22-40).  Radix-2 decimation in
 * time with twiddles from long-double trig; n must be a power of two.        */
/* ------------------------------------------------------------------------ */
/* twiddle table cos/sin(2 pi k / n), k < n/2, cached for the last n used */
static int tw_n = 0;
static double* tw_c = NULL;
static double* tw_s = NULL;

static void twiddles(int n)
{
    if (tw_n == n) return;
    free(tw_c);
    free(tw_s);
    int h = n / 2 > 0 ? n / 2 : 1;
    tw_c = dalloc(h);
    tw_s = dalloc(h);
    const long double two_pi = 6.283185307179586476925286766559005768L;
    for (int k = 0; k < h; ++k) {
        long double ang = two_pi * (long double)k / (long double)n;
        tw_c[k] = (double)cosl(ang);
        tw_s[k] = (double)sinl(ang);
    }
    tw_n = n;
}

void orc_dft(int n, double* a, int sign)
{
    twiddles(n);
    int j = 0;
    for (int i = 1; i < n; ++i) {
        int bit = n >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) {
            double t = RE(a, i);
            RE(a, i) = RE(a, j);
            RE(a, j) = t;
            t = IM(a, i);
            IM(a, i) = IM(a, j);
            IM(a, j) = t;
        }
    }
    for (int len = 2; len <= n; len <<= 1) {
        int h = len / 2;
        int step = n / len;
        for (int k = 0; k < h; ++k) {
            double wr = tw_c[k * step];
            double wi = sign > 0 ? tw_s[k * step] : -tw_s[k * step];
            for (int base = 0; base < n; base += len) {
                int p = base + k, q = p + h;
                double br = RE(a, q) * wr - IM(a, q) * wi;
                double bi = RE(a, q) * wi + IM(a, q) * wr;
                RE(a, q) = RE(a, p) - br;
                IM(a, q) = IM(a, p) - bi;
                RE(a, p) = RE(a, p) + br;
                IM(a, p) = IM(a, p) + bi;
            }
        }
    }
}

/* SpectralTransformer::forwardFFT, real -> complex (SpectralTransformer.cpp:57-72):
 * the "forward" plan is FFTW_BACKWARD (e^{+i}), result scaled by 1/N.        */
void orc_forward_real(int n, const double* in, double* out)
{
    for (int i = 0; i < n; ++i) {
        RE(out, i) = in[i];
        IM(out, i) = 0.0;
    }
    orc_dft(n, out, +1);
    for (int i = 0; i < 2 * n; ++i) out[i] /= (double)n;
}

/* SpectralTransformer::forwardFFT, complex -> complex (:97-112) */
static void orc_forward_cplx(int n, const double* in, double* out)
{
    if (out != in) memcpy(out, in, sizeof(double) * 2 * n);
    orc_dft(n, out, +1);
    for (int i = 0; i < 2 * n; ++i) out[i] /= (double)n;
}

/* SpectralTransformer::backwardFFT, complex -> real (:77-92): FFTW_FORWARD
 * (e^{-i}), unscaled, real part kept.                                        */
void orc_backward_real(int n, const double* in, double* out)
{
    double* t = dalloc(2 * n);
    memcpy(t, in, sizeof(double) * 2 * n);
    orc_dft(n, t, -1);
    for (int i = 0; i < n; ++i) out[i] = RE(t, i);
    free(t);
}

/* SpectralTransformer::backwardFFT, complex -> complex (:117-132) */
static void orc_backward_cplx(int n, const double* in, double* out)
{
    if (out != in) memcpy(out, in, sizeof(double) * 2 * n);
    orc_dft(n, out, -1);
}

/* SpectralTransformer::differentiate (:140-158): out_k = -(i m k0) in_k with
 * m = k (k < N/2) or k - N, Nyquist set to zero.                             */
void orc_differentiate(int n, const double* in, double* out, double period)
{
    double k0c = 2 * PI / period;
    for (int k = 0; k < n; ++k) {
        if (k != n / 2) {
            int m = (k < n / 2) ? k : k - n;
            double s = m * k0c;
            /* -(0 + i s)(x + i y) = (s y, -s x) */
            double x = RE(in, k), y = IM(in, k);
            RE(out, k) = s * y;
            IM(out, k) = -(s * x);
        } else {
            RE(out, n / 2) = 0.0;
            IM(out, n / 2) = 0.0;
        }
    }
}

/* SpectralTransformer::lamIntegrate (:165-189): out_m = f_m / (lambda - i m k0)
 * with the DC, near-zero and Nyquist special cases.                          */
void orc_lam_integrate(int n, const double* fk, double* out, const double* lambda, double period)
{
    double k0c = 2 * PI / period;
    double lr = lambda[0], li = lambda[1];
    if (lr != 0.0 || li != 0.0)
        cdiv(RE(fk, 0), IM(fk, 0), lr, li, &RE(out, 0), &IM(out, 0));
    else
        RE(out, 0) = IM(out, 0) = 0.0;
    for (int k = 1; k < n; ++k) {
        if (k != n / 2) {
            int m = (k < n / 2) ? k : k - n;
            double dr = lr - 0.0, di = li - m * k0c;
            if (hypot(dr, di) < 1e-14)
                RE(out, k) = IM(out, k) = 0.0;
            else
                cdiv(RE(fk, k), IM(fk, k), dr, di, &RE(out, k), &IM(out, k));
        } else {
            /* lambda / (lambda^2 + (k0 n/2)^2) * f_{n/2} */
            double s = k0c * n / 2.0;
            double l2r = lr * lr - li * li, l2i = lr * li + li * lr;
            double qr, qi;
            cdiv(lr, li, l2r + s * s, l2i, &qr, &qi);
            double fr = RE(fk, n / 2), fi = IM(fk, n / 2);
            RE(out, n / 2) = qr * fr - qi * fi;
            IM(out, n / 2) = qr * fi + qi * fr;
        }
    }
}

/* SpectralTransformer::halveModes (:196-217) */
void orc_halve_modes(int n_in, const double* in, double* out)
{
    int no = n_in / 2;
    double* t = dalloc(2 * no);
    for (int k = 0; k < no / 2; ++k) {
        RE(t, k) = RE(in, k);
        IM(t, k) = IM(in, k);
    }
    RE(t, no / 2) = RE(in, no / 2) + RE(in, 3 * no / 2);
    IM(t, no / 2) = IM(in, no / 2) + IM(in, 3 * no / 2);
    for (int k = no / 2 + 1; k < no; ++k) {
        RE(t, k) = RE(in, no + k);
        IM(t, k) = IM(in, no + k);
    }
    memcpy(out, t, sizeof(double) * 2 * no);
    free(t);
}

/* SpectralTransformer::doubleModes (:224-252).  Restated with its exact store
 * order: the upper-half copy runs from k = N_in/2, so out[3 N_in/2] ends up
 * holding the full in[N_in/2] while out[N_in/2] holds half of it.            */
void orc_double_modes(int n_in, const double* in, double* out)
{
    int no = 2 * n_in;
    double* t = dalloc(2 * no);
    for (int k = 0; k < n_in / 2; ++k) {
        RE(t, k) = RE(in, k);
        IM(t, k) = IM(in, k);
    }
    RE(t, n_in / 2) = 0.5 * RE(in, n_in / 2);
    IM(t, n_in / 2) = 0.5 * IM(in, n_in / 2);
    RE(t, 3 * n_in / 2) = 0.5 * RE(in, n_in / 2);
    IM(t, 3 * n_in / 2) = 0.5 * IM(in, n_in / 2);
    for (int k = n_in / 2; k < n_in; ++k) {
        RE(t, n_in + k) = RE(in, k);
        IM(t, n_in + k) = IM(in, k);
    }
    for (int k = n_in / 2 + 1; k < 3 * n_in / 2; ++k) RE(t, k) = IM(t, k) = 0.0;
    memcpy(out, t, sizeof(double) * 2 * no);
    free(t);
}

/* SpectralTransformer::solveInhom (:264-292): X' + f X = g, periodic, by the
 * integrating factor e^{F}, F' = f.                                          */
void orc_solve_inhom(int n, const double* f, const double* g, double* x, double period)
{
    double* fh = dalloc(2 * n);
    double* Fh = dalloc(2 * n);
    double* Fr = dalloc(n);
    double* h = dalloc(n);
    double* hh = dalloc(2 * n);
    double* Hh = dalloc(2 * n);
    double zero[2] = {0.0, 0.0};
    orc_forward_real(n, f, fh);
    orc_lam_integrate(n, fh, Fh, zero, period);
    orc_backward_real(n, Fh, Fr);
    for (int i = 0; i < n; ++i) h[i] = -g[i] * exp(Fr[i]);
    orc_forward_real(n, h, hh);
    orc_lam_integrate(n, hh, Hh, fh, period);
    orc_backward_real(n, Hh, x);
    for (int i = 0; i < n; ++i) x[i] *= exp(-Fr[i]);
    free(fh);
    free(Fh);
    free(Fr);
    free(h);
    free(hh);
    free(Hh);
}

/* spectral derivative of a real series: forwardFFT, differentiate, backwardFFT */
static void tau_derivative(int n, const double* in, double* out, double period)
{
    double* a = dalloc(2 * n);
    double* b = dalloc(2 * n);
    orc_forward_real(n, in, a);
    orc_differentiate(n, a, b, period);
    orc_backward_real(n, b, out);
    free(a);
    free(b);
}

/* ------------------------------------------------------------------------ */
/* InitialConditionGenerator                                                 */
/* ------------------------------------------------------------------------ */

/* FieldsToStateVector (InitialConditionGenerator.cpp:766-778):
 * Y = halveModes(FFT(U + i(V+F))/N); y holds n/2 complex modes.             */
void orc_fields_to_state(int n, const double* u, const double* v, const double* f, double* y)
{
    double* z = dalloc(2 * n);
    for (int j = 0; j < n; ++j) {
        RE(z, j) = u[j];
        IM(z, j) = v[j] + f[j];
    }
    orc_forward_cplx(n, z, z);
    orc_halve_modes(n, z, y);
    free(z);
}

/* computeLeftExpansion (InitialConditionGenerator.cpp:37-239): 5th-order
 * Taylor series at x = XLeft from f_c and psi_c.                             */
void orc_left_expansion(int n, double d, double xl, const double* f0, const double* psi0, double delta,
                        double* y)
{
    double *df = dalloc(n), *d2f = dalloc(n), *d3f = dalloc(n);
    tau_derivative(n, f0, df, delta);
    tau_derivative(n, df, d2f, delta);
    tau_derivative(n, d2f, d3f, delta);

    double *c1 = dalloc(n), *c2 = dalloc(n), *u1 = dalloc(n);
    for (int j = 0; j < n; ++j) {
        c1[j] = 1.0;
        c2[j] = -(d - 1.0) * psi0[j] * f0[j];
    }
    orc_solve_inhom(n, c1, c2, u1, delta);

    double *du1 = dalloc(n), *d2u1 = dalloc(n), *d3u1 = dalloc(n), *d4u1 = dalloc(n);
    tau_derivative(n, u1, du1, delta);
    tau_derivative(n, du1, d2u1, delta);
    tau_derivative(n, d2u1, d3u1, delta);
    tau_derivative(n, d3u1, d4u1, delta);

    double *U = dalloc(n), *V = dalloc(n), *F = dalloc(n);
    for (int j = 0; j < n; ++j) {
        const double f = f0[j], psi = psi0[j];
        const double u1j = u1[j];
        const double du = du1[j], d2u = d2u1[j], d3u = d3u1[j], d4u = d4u1[j];
        const double dfj = df[j], d2fj = d2f[j], d3fj = d3f[j];

        const double v1 = u1j;
        const double f2 = ((d - 3.0) * pow(d - 2.0, 3) * f * pow(u1j, 2)) / (8.0 * (d - 1.0));
        const double u2 = -psi;
        const double v2 = psi;

        const double common3 = ((d - 3.0) * pow(d - 2.0, 3) * pow(f, 3) * pow(u1j, 3) + 4.0 * dfj * (u1j + du) -
                                4.0 * f * (2.0 * u1j + 3.0 * du + d2u));
        const double u3 = common3 / (8.0 * (1.0 - d) * pow(f, 3));
        const double v3 = u3;

        const double f4 =
            -((d - 3.0) * pow(d - 2.0, 3) *
              ((pow(d - 2.0, 3) * (5.0 - 6.0 * d + d * d) * pow(f, 3) * pow(u1j, 4)) +
               8.0 * (d - 1.0) * dfj * u1j * (du + u1j) -
               8.0 * f * (pow(du, 2) + ((d - 1.0) * d2u + (-1.0 + 3.0 * d) * du) * u1j + (-1.0 + 2.0 * d) * pow(u1j, 2)))) /
            (128.0 * pow(d - 1.0, 2) * (1.0 + d) * pow(f, 2));

        const double u4 = (-192.0 * (d - 1.0) * pow(dfj, 2) * du * pow(f, 2) + 192.0 * (d - 1.0) * d2u * dfj * pow(f, 3) +
                           64.0 * (d - 1.0) * d2fj * du * pow(f, 3) + 640.0 * (d - 1.0) * dfj * du * pow(f, 3) -
                           64.0 * (d - 1.0) * (6.0 * d2u + d3u) * pow(f, 4) - 704.0 * (d - 1.0) * du * pow(f, 4) -
                           192.0 * (d - 1.0) * pow(dfj, 2) * pow(f, 2) * u1j + 64.0 * (d - 1.0) * d2fj * pow(f, 3) * u1j +
                           448.0 * (d - 1.0) * dfj * pow(f, 3) * u1j - 384.0 * (d - 1.0) * pow(f, 4) * u1j +
                           32.0 * pow(d - 2.0, 3) * (3.0 - 7.0 * d + 2.0 * d * d) * pow(f, 6) * pow(u1j, 2) * (du + u1j)) /
                          (128.0 * pow(d - 1.0, 2) * (1.0 + d) * pow(f, 7));
        const double v4 = -u4;

        const double q = 3.0 - 13.0 * d + 4.0 * d * d;
        const double u5 =
            (-64.0 * (d - 1.0) * d2fj * d2u * pow(f, 2) - 16.0 * (d - 1.0) * (15.0 * d2fj + d3fj) * du * pow(f, 2) -
             32.0 * (d - 1.0) * dfj * (20.0 * d2u + 3.0 * d3u + 40.0 * du) * pow(f, 2) +
             560.0 * (d - 1.0) * d2u * pow(f, 3) + 160.0 * (d - 1.0) * d3u * pow(f, 3) +
             16.0 * (d - 1.0) * d4u * pow(f, 3) + 800.0 * (d - 1.0) * du * pow(f, 3) -
             16.0 * (d - 1.0) * (11.0 * d2fj + d3fj) * pow(f, 2) * u1j - 736.0 * (d - 1.0) * dfj * pow(f, 2) * u1j +
             384.0 * (d - 1.0) * pow(f, 3) * u1j - 8.0 * pow(d - 2.0, 3) * q * pow(du, 2) * pow(f, 5) * u1j +
             8.0 * pow(d - 2.0, 3) * q * dfj * du * pow(f, 4) * pow(u1j, 2) -
             8.0 * pow(d - 2.0, 3) * q * (d2u + 5.0 * du) * pow(f, 5) * pow(u1j, 2) +
             8.0 * pow(d - 2.0, 3) * q * dfj * pow(f, 4) * pow(u1j, 3) -
             24.0 * pow(d - 2.0, 3) * q * pow(f, 5) * pow(u1j, 3) +
             pow(d - 2.0, 6) * (3.0 + 29.0 * d - 19.0 * d * d + 3.0 * d * d * d) * pow(f, 7) * pow(u1j, 5) -
             240.0 * (d - 1.0) * pow(dfj, 3) * (du + u1j) +
             80.0 * (d - 1.0) * dfj * f * (2.0 * d2fj * du + dfj * (3.0 * d2u + 11.0 * du) + 2.0 * (d2fj + 4.0 * dfj) * u1j)) /
            (128.0 * pow(d - 1.0, 2) * (1.0 + d) * pow(f, 7));
        const double v5 = u5;

        U[j] = xl * u1j + pow(xl, 2) * u2 + pow(xl, 3) * u3 + pow(xl, 4) * u4 + pow(xl, 5) * u5;
        V[j] = xl * v1 + pow(xl, 2) * v2 + pow(xl, 3) * v3 + pow(xl, 4) * v4 + pow(xl, 5) * v5;
        F[j] = f + pow(xl, 2) * f2 + pow(xl, 4) * f4;
    }
    orc_fields_to_state(n, U, V, F, y);
    RE(y, 2) = delta;

    free(df); free(d2f); free(d3f); free(c1); free(c2); free(u1);
    free(du1); free(d2u1); free(d3u1); free(d4u1); free(U); free(V); free(F);
}

/* computeRightExpansion (InitialConditionGenerator.cpp:252-667, the serial
 * branch :460-619): 3rd-order series about the horizon x = 1 from U_p.       */
void orc_right_expansion(int n, double d, double xr, const double* u0, double delta, double* y)
{
    const double dx = xr - 1.0;
    const double p3 = pow(d - 2.0, 3);
    double *du0 = dalloc(n), *d2u0 = dalloc(n);
    {
        double* a = dalloc(2 * n);
        double* b = dalloc(2 * n);
        double* c = dalloc(2 * n);
        orc_forward_real(n, u0, a);
        orc_differentiate(n, a, b, delta);
        orc_backward_real(n, b, du0);
        orc_differentiate(n, b, c, delta);
        orc_backward_real(n, c, d2u0);
        free(a); free(b); free(c);
    }
    double *c1 = dalloc(n), *c2 = dalloc(n), *ia20 = dalloc(n), *v0 = dalloc(n);
    double *f1 = dalloc(n), *u1 = dalloc(n), *ia21 = dalloc(n), *v1 = dalloc(n);
    double *f2 = dalloc(n), *ia22 = dalloc(n), *u2 = dalloc(n), *du2 = dalloc(n), *v2 = dalloc(n);
    double *f3 = dalloc(n), *ia23 = dalloc(n), *u3 = dalloc(n), *v3 = dalloc(n);
    double *F = dalloc(n), *U = dalloc(n), *V = dalloc(n);

    for (int j = 0; j < n; ++j) {
        c1[j] = 3.0 - d - pow(d - 2.0, 3) * u0[j] * u0[j] / 4.0;
        c2[j] = d - 3.0;
    }
    orc_solve_inhom(n, c1, c2, ia20, delta);

    for (int j = 0; j < n; ++j) {
        c1[j] = (6.0 - 2.0 * d + (d - 2.0) * ia20[j]) / (2.0 * ia20[j]);
        c2[j] = (d - 2.0) * u0[j] / 2.0;
    }
    orc_solve_inhom(n, c1, c2, v0, delta);

    for (int j = 0; j < n; ++j) {
        f1[j] = 3.0 - d + (d - 3.0) / ia20[j];
        ia21[j] = -ia20[j] * (8.0 * (d - 3.0) + p3 * (u0[j] * u0[j] + v0[j] * v0[j])) / 8.0 + d - 3.0;
        u1[j] = ((d - 2.0 - 2.0 * (d - 3.0) / ia20[j]) * u0[j] + (d - 2.0) * v0[j]) / 4.0 - du0[j] / 2.0;
    }

    for (int j = 0; j < n; ++j) {
        c1[j] = (6.0 - 2.0 * d + d * ia20[j] - 2.0 * f1[j] * ia20[j]) / (2.0 * ia20[j]);
        c2[j] = (2.0 * (3.0 - d) * (f1[j] - 1.0) * ia20[j] * v0[j] + 2.0 * (d - 3.0) * ia21[j] * v0[j] +
                 (d - 2.0) * pow(ia20[j], 2) * ((f1[j] - 1.0) * u0[j] + u1[j] + (f1[j] - 1.0) * v0[j])) /
                (2.0 * pow(ia20[j], 2));
    }
    orc_solve_inhom(n, c1, c2, v1, delta);

    for (int j = 0; j < n; ++j)
        f2[j] = (d - 3.0) * ((f1[j] - 1.0) * (1.0 - ia20[j]) * ia20[j] - ia21[j]) / (2.0 * pow(ia20[j], 2));

    for (int j = 0; j < n; ++j)
        ia22[j] = (3.0 - d - (ia21[j] - ia20[j]) * (8.0 * (d - 3.0) + p3 * (pow(u0[j], 2) + pow(v0[j], 2))) / 8.0 -
                   p3 * ia20[j] * (u0[j] * u1[j] + v0[j] * v1[j]) / 4.0) /
                  2.0;

    for (int j = 0; j < n; ++j) {
        const double A = 4.0 * (3.0 - d) * (d - 6.0 + f1[j]) * ia20[j];
        const double B = (d - 2.0) * (d - 8.0 + 2.0 * f1[j]) * pow(ia20[j], 2);
        const double C = 4.0 * (d - 3.0) * (d - 3.0 + 2.0 * ia21[j]);
        const double D = -(d - 3.0) * p3 * ia20[j] * pow(u0[j], 3);
        const double E = (4.0 * (6.0 - 2.0 * d + (d - 2.0) * ia20[j]) * u1[j] +
                          (d - 2.0) * v0[j] * (6.0 - 2.0 * d + (d - 8.0 + 2.0 * f1[j]) * ia20[j]) -
                          8.0 * ia20[j] * v1[j] + 4.0 * d * ia20[j] * v1[j] - 12.0 * du0[j] + 4.0 * d * du0[j] +
                          8.0 * ia20[j] * du0[j] - 2.0 * d * ia20[j] * du0[j] + 4.0 * f1[j] * ia20[j] * du0[j] +
                          4.0 * ia20[j] * d2u0[j]) *
                         ia20[j];
        u2[j] = (A + B + C) * u0[j] + D + E;
        u2[j] /= 32.0 * pow(ia20[j], 2);
    }
    tau_derivative(n, u2, du2, delta);

    for (int j = 0; j < n; ++j) {
        c1[j] = 1.0 + d / 2.0 - 2.0 * f1[j] + (3.0 - d) / ia20[j];
        c2[j] = (2.0 * (3.0 - d) * pow(ia21[j], 2) * v0[j] +
                 2.0 * (d - 3.0) * pow(ia20[j], 2) * ((f1[j] - 1.0 - f2[j]) * v0[j] - (f1[j] - 1.0) * v1[j]) +
                 ((d - 2.0) * ((1.0 - f1[j] + f2[j]) * u0[j] + (f1[j] - 1.0) * u1[j] + u2[j] + (1.0 - f1[j] + f2[j]) * v0[j]) +
                  ((d - 2.0) * (f1[j] - 1.0) - 2.0 * f2[j]) * v1[j]) *
                     pow(ia20[j], 3) +
                 2.0 * (d - 3.0) * ia20[j] * (ia22[j] * v0[j] + ia21[j] * ((f1[j] - 1.0) * v0[j] + v1[j]))) /
                (2.0 * pow(ia20[j], 3));
    }
    orc_solve_inhom(n, c1, c2, v2, delta);

    for (int j = 0; j < n; ++j) {
        const double a0 = ia20[j], a1 = ia21[j], a2 = ia22[j];
        f3[j] = ((-3.0 + d) * ((1.0 - f1[j] + f2[j]) * pow(a0, 2) + (-1.0 + f1[j] - f2[j]) * pow(a0, 3) + pow(a1, 2) -
                               a0 * ((-1.0 + f1[j]) * a1 + a2))) /
                (3.0 * pow(a0, 3));
        ia23[j] = (-3.0 + d +
                   (-((a0 - a1 + a2) * (8.0 * (-3.0 + d) + p3 * (u0[j] * u0[j] + v0[j] * v0[j]))) +
                    2.0 * p3 * (a0 - a1) * (u0[j] * u1[j] + v0[j] * v1[j]) -
                    p3 * a0 * (pow(u1[j], 2) + 2.0 * u0[j] * u2[j] + pow(v1[j], 2) + 2.0 * v0[j] * v2[j])) /
                       8.0) /
                  3.0;
        u3[j] = -(16.0 * (-3.0 + d) * pow(a1, 2) * u0[j] +
                  4.0 * (-3.0 + d) * a0 * ((-3.0 + d + f1[j] * (-3.0 + d - 2.0 * a1) + 6.0 * a1 - 4.0 * a2) * u0[j] - 4.0 * a1 * u1[j]) -
                  (d - 3.0) * pow(a0, 2) *
                      (4.0 * (-10.0 + d + f1[j] * (-1.0 + d + f1[j]) - 2.0 * f2[j]) * u0[j] + p3 * (1.0 + f1[j]) * pow(u0[j], 3) +
                       2.0 * (-4.0 * (-3.0 + f1[j]) * u1[j] - 8.0 * u2[j] + (1.0 + f1[j]) * (-2.0 * du0[j] + (d - 2.0) * v0[j]))) +
                  pow(a0, 3) *
                      (8.0 * du0[j] - 2.0 * d * du0[j] + 12.0 * du0[j] * f1[j] - 2.0 * d * du0[j] * f1[j] +
                       4.0 * du0[j] * pow(f1[j], 2) + 4.0 * d2u0[j] * (1.0 + f1[j]) - 8.0 * du0[j] * f2[j] +
                       (d - 2.0) * (-16.0 + d + f1[j] * (2.0 + d + 2.0 * f1[j]) - 4.0 * f2[j]) * u0[j] -
                       4.0 * (d - 2.0) * (-3.0 + f1[j]) * u1[j] + 16.0 * u2[j] - 8.0 * d * u2[j] + 32.0 * v0[j] -
                       18.0 * d * v0[j] + pow(d, 2) * v0[j] - 4.0 * f1[j] * v0[j] + pow(d, 2) * f1[j] * v0[j] -
                       4.0 * pow(f1[j], 2) * v0[j] + 2.0 * d * pow(f1[j], 2) * v0[j] + 8.0 * f2[j] * v0[j] -
                       4.0 * d * f2[j] * v0[j] - 24.0 * v1[j] + 12.0 * d * v1[j] + 8.0 * f1[j] * v1[j] -
                       4.0 * d * f1[j] * v1[j] + 16.0 * v2[j] - 8.0 * d * v2[j] + 16.0 * du2[j])) /
                (96.0 * pow(a0, 3));
    }

    for (int j = 0; j < n; ++j) {
        const double a0 = ia20[j], a1 = ia21[j], a2 = ia22[j], a3 = ia23[j];
        c1[j] = 2.0 + d / 2.0 - 3.0 * f1[j] + (3.0 - d) / a0;
        c2[j] = ((d - 3.0) * pow(a1, 3) * v0[j]) / pow(a0, 4) -
                ((d - 3.0) * a1 * (2.0 * a2 * v0[j] + a1 * ((-1.0 + f1[j]) * v0[j] + v1[j]))) / pow(a0, 3) -
                ((d - 3.0) * ((-1.0 + f1[j] - f2[j] + f3[j]) * v0[j] + (1.0 - f1[j] + f2[j]) * v1[j] + (-1.0 + f1[j]) * v2[j])) / a0 +
                ((d - 2.0) * (-1.0 + f1[j] - f2[j] + f3[j]) * u0[j] - (d - 2.0) * (-1.0 + f1[j] - f2[j]) * u1[j] +
                 2.0 * u2[j] - d * u2[j] - 2.0 * f1[j] * u2[j] + d * f1[j] * u2[j] - 2.0 * u3[j] + d * u3[j] +
                 2.0 * v0[j] - d * v0[j] - 2.0 * f1[j] * v0[j] + d * f1[j] * v0[j] + 2.0 * f2[j] * v0[j] -
                 d * f2[j] * v0[j] - 2.0 * f3[j] * v0[j] + d * f3[j] * v0[j] - 2.0 * v1[j] + d * v1[j] +
                 2.0 * f1[j] * v1[j] - d * f1[j] * v1[j] - 2.0 * f2[j] * v1[j] + d * f2[j] * v1[j] -
                 2.0 * f3[j] * v1[j] + ((d - 2.0) * (-1.0 + f1[j]) - 4.0 * f2[j]) * v2[j]) /
                    2.0 +
                ((d - 3.0) * (a3 * v0[j] + a2 * ((-1.0 + f1[j]) * v0[j] + v1[j]) +
                              a1 * ((1.0 - f1[j] + f2[j]) * v0[j] + (-1.0 + f1[j]) * v1[j] + v2[j]))) /
                    pow(a0, 2);
    }
    orc_solve_inhom(n, c1, c2, v3, delta);

    for (int j = 0; j < n; ++j) {
        F[j] = 1.0 + dx * f1[j] + dx * dx * f2[j] + dx * dx * dx * f3[j];
        U[j] = u0[j] + dx * u1[j] + dx * dx * u2[j] + dx * dx * dx * u3[j];
        V[j] = v0[j] + dx * v1[j] + dx * dx * v2[j] + dx * dx * dx * v3[j];
    }
    orc_fields_to_state(n, U, V, F, y);
    RE(y, 2) = delta;

    free(du0); free(d2u0); free(c1); free(c2); free(ia20); free(v0); free(f1); free(u1); free(ia21);
    free(v1); free(f2); free(ia22); free(u2); free(du2); free(v2); free(f3); free(ia23); free(u3);
    free(v3); free(F); free(U); free(V);
}

/* packSpectralFields (InitialConditionGenerator.cpp:678-711) */
void orc_pack(int n, const double* odd1, const double* odd2, const double* even, double* z)
{
    const int nn = 3 * n / 4;
    double *a = dalloc(2 * n), *b = dalloc(2 * n), *c = dalloc(2 * n);
    orc_forward_real(n, odd1, a);
    orc_forward_real(n, odd2, b);
    orc_forward_real(n, even, c);
    orc_halve_modes(n, a, a);
    orc_halve_modes(n, b, b);
    orc_halve_modes(n, c, c);
    for (int j = 0; j < nn / 6; ++j) {
        z[2 * j] = RE(a, 2 * j + 1);
        z[2 * j + 1] = IM(a, 2 * j + 1);
        z[2 * j + nn / 3] = RE(b, 2 * j + 1);
        z[2 * j + 1 + nn / 3] = IM(b, 2 * j + 1);
        z[2 * j + 2 * nn / 3] = RE(c, 2 * j);
        z[2 * j + 1 + 2 * nn / 3] = IM(c, 2 * j);
    }
    z[2 * nn / 3 + 1] = RE(c, nn / 3);
    free(a);
    free(b);
    free(c);
}

/* unpackSpectralFields (InitialConditionGenerator.cpp:719-758) */
void orc_unpack(int n, const double* z, double* odd1, double* odd2, double* even)
{
    const int nn = 3 * n / 4, h = n / 2;
    double *a = dalloc(2 * n), *b = dalloc(2 * n), *c = dalloc(2 * n);
    for (int j = 0; j < nn / 6; ++j) {
        RE(a, 2 * j + 1) = z[2 * j];
        IM(a, 2 * j + 1) = z[2 * j + 1];
        RE(a, h - 2 * j - 1) = RE(a, 2 * j + 1);
        IM(a, h - 2 * j - 1) = -IM(a, 2 * j + 1);
        RE(b, 2 * j + 1) = z[2 * j + nn / 3];
        IM(b, 2 * j + 1) = z[2 * j + 1 + nn / 3];
        RE(b, h - 2 * j - 1) = RE(b, 2 * j + 1);
        IM(b, h - 2 * j - 1) = -IM(b, 2 * j + 1);
        RE(c, 2 * j) = z[2 * j + 2 * nn / 3];
        IM(c, 2 * j) = z[2 * j + 1 + 2 * nn / 3];
        if (j != 0) {
            RE(c, h - 2 * j) = RE(c, 2 * j);
            IM(c, h - 2 * j) = -IM(c, 2 * j);
        }
    }
    IM(c, 0) = 0.0;
    orc_double_modes(h, a, a);
    orc_double_modes(h, b, b);
    orc_double_modes(h, c, c);
    RE(c, nn / 3) = z[2 * nn / 3 + 1] / 2.0;
    IM(c, nn / 3) = 0.0;
    RE(c, nn) = z[2 * nn / 3 + 1] / 2.0;
    IM(c, nn) = 0.0;
    orc_backward_real(n, a, odd1);
    orc_backward_real(n, b, odd2);
    orc_backward_real(n, c, even);
    free(a);
    free(b);
    free(c);
}

/* doubleModes + the phase fix on mode 2 (InitialConditionGenerator.cpp:798-800):
 * Re c[2] := -Re c[N-2], which drops Delta from the spectrum.                */
static void expand_state(int n, const double* y, double* c)
{
    orc_double_modes(n / 2, y, c);
    RE(c, 2) = -RE(c, n - 2);
}

/* StateVectorToFields with derivatives and IA2 (InitialConditionGenerator.cpp:
 * 791-884, the non-hybrid branch :842-882).                                  */
void orc_state_to_fields(int n, double dim, const double* y, double x, double* u, double* v, double* f,
                         double* ia2, double* dudt, double* dvdt, double* dfdt)
{
    const double delta = RE(y, 2);
    double *c1 = dalloc(2 * n), *c2 = dalloc(2 * n);
    expand_state(n, y, c1);
    orc_differentiate(n, c1, c2, delta);
    orc_backward_cplx(n, c1, c1);
    for (int j = 0; j < n / 2; ++j) {
        u[j] = 0.5 * (RE(c1, j) - RE(c1, j + n / 2));
        v[j] = 0.5 * (IM(c1, j) - IM(c1, j + n / 2));
        f[j] = 0.5 * (IM(c1, j) + IM(c1, j + n / 2));
    }
    for (int j = 0; j < n / 2; ++j) {
        u[j + n / 2] = -u[j];
        v[j + n / 2] = -v[j];
        f[j + n / 2] = f[j];
    }
    orc_backward_cplx(n, c2, c2);
    for (int j = 0; j < n / 2; ++j) {
        dudt[j] = 0.5 * (RE(c2, j) - RE(c2, j + n / 2));
        dvdt[j] = 0.5 * (IM(c2, j) - IM(c2, j + n / 2));
        dfdt[j] = 0.5 * (IM(c2, j) + IM(c2, j + n / 2));
    }
    for (int j = 0; j < n / 2; ++j) {
        dudt[j + n / 2] = -dudt[j];
        dvdt[j + n / 2] = -dvdt[j];
        dfdt[j + n / 2] = dfdt[j];
    }
    double *k1 = dalloc(n), *k2 = dalloc(n);
    for (int j = 0; j < n; ++j) {
        k1[j] = -(((x + f[j]) * u[j] * u[j] + (x - f[j]) * v[j] * v[j]) * pow((dim - 2.0), 3) / (8.0 * x) + (dim - 3.0));
        k2[j] = (dim - 3.0);
    }
    orc_solve_inhom(n, k1, k2, ia2, delta);
    free(c1);
    free(c2);
    free(k1);
    free(k2);
}

/* StateVectorToFields without derivatives (InitialConditionGenerator.cpp:891-932) */
void orc_state_to_fields_light(int n, const double* y, double* u, double* v, double* f)
{
    double* c1 = dalloc(2 * n);
    expand_state(n, y, c1);
    orc_backward_cplx(n, c1, c1);
    for (int j = 0; j < n / 2; ++j) {
        u[j] = 0.5 * (RE(c1, j) - RE(c1, j + n / 2));
        v[j] = 0.5 * (IM(c1, j) - IM(c1, j + n / 2));
        f[j] = 0.5 * (IM(c1, j) + IM(c1, j + n / 2));
    }
    for (int j = 0; j < n / 2; ++j) {
        u[j + n / 2] = -u[j];
        v[j + n / 2] = -v[j];
        f[j + n / 2] = f[j];
    }
    free(c1);
}

/* ------------------------------------------------------------------------ */
/* ODEStepper                                                                */
/* ------------------------------------------------------------------------ */

/* ODEStepper::computeDerivatives (ODEStepper.cpp:92-136) */
void orc_rhs(int n, double dim, const double* yreal, double x, double* dyreal)
{
    double *U = dalloc(n), *V = dalloc(n), *F = dalloc(n), *A = dalloc(n);
    double *dU = dalloc(n), *dV = dalloc(n), *dF = dalloc(n);
    double *ux = dalloc(n), *vx = dalloc(n), *fx = dalloc(n);
    orc_state_to_fields(n, dim, yreal, x, U, V, F, A, dU, dV, dF);
    for (int j = 0; j < n; ++j) {
        ux[j] = (F[j] * ((dim - 2.0) * V[j] - (2.0 * (dim - 3.0) / A[j] - (dim - 2.0)) * U[j]) - 2.0 * x * dU[j]) /
                (2.0 * x * (F[j] + x));
        vx[j] = (F[j] * ((dim - 2.0) * U[j] - (2.0 * (dim - 3.0) / A[j] - (dim - 2.0)) * V[j]) + 2.0 * x * dV[j]) /
                (2.0 * x * (F[j] - x));
        fx[j] = (dim - 3.0) * F[j] * (1.0 - A[j]) / (A[j] * x);
    }
    orc_fields_to_state(n, ux, vx, fx, dyreal);
    RE(dyreal, 2) = 0.0;
    free(U); free(V); free(F); free(A); free(dU); free(dV); free(dF); free(ux); free(vx); free(fx);
}

/* Gauss-Legendre tableaux (ODEStepper.cpp:27-79) */
static int tableau(int scheme, double a[3][3], double b[3], double c[3])
{
    memset(a, 0, sizeof(double) * 9);
    if (scheme == 1) {
        a[0][0] = 0.5;
        b[0] = 1.0;
        c[0] = 0.5;
        return 1;
    }
    if (scheme == 3) {
        a[0][0] = 5.0 / 36.0;
        a[0][1] = 2.0 / 9.0 - 1.0 / sqrt(15.0);
        a[0][2] = 5.0 / 36.0 - 0.5 / sqrt(15.0);
        a[1][0] = 5.0 / 36.0 + sqrt(15.0) / 24.0;
        a[1][1] = 2.0 / 9.0;
        a[1][2] = 5.0 / 36.0 - sqrt(15.0) / 24.0;
        a[2][0] = 5.0 / 36.0 + 0.5 / sqrt(15.0);
        a[2][1] = 2.0 / 9.0 + 1.0 / sqrt(15.0);
        a[2][2] = 5.0 / 36.0;
        b[0] = b[2] = 5.0 / 18.0;
        b[1] = 4.0 / 9.0;
        c[0] = 0.5 - sqrt(15.0) / 10.0;
        c[1] = 0.5;
        c[2] = 0.5 + sqrt(15.0) / 10.0;
        return 3;
    }
    a[0][0] = 0.25;
    a[0][1] = 0.25 - 0.5 / sqrt(3.0);
    a[1][0] = 0.25 + 0.5 / sqrt(3.0);
    a[1][1] = 0.25;
    b[0] = b[1] = 0.5;
    c[0] = 0.5 - 0.5 / sqrt(3.0);
    c[1] = 0.5 + 0.5 / sqrt(3.0);
    return 2;
}

/* ODEStepper::stepIRK (ODEStepper.cpp:163-292): fixed-point iteration on the
 * stage values, RMS stage change against a tolerance relaxed after maxIts/2,
 * then y += dx sum_i b_i f_i with the RHS of the last iteration.             */
int orc_irk_step(int n, double dim, int scheme, double precision, int max_its, const double* yin, double xin,
                 double xout, double* yout, int* its_out)
{
    double a[3][3], b[3], c[3];
    const int s = tableau(scheme, a, b, c);
    const double dx = xout - xin;
    double xs[3];
    double* y = dalloc(n);
    double* f = dalloc((size_t)s * n);
    double* yk1 = dalloc((size_t)s * n);
    double* yk2 = dalloc((size_t)s * n);
    int its_reached = 0, converged = 0;
    memcpy(y, yin, sizeof(double) * n);
    for (int i = 0; i < s; ++i) xs[i] = xin + dx * c[i];
    for (int i = 0; i < s; ++i) memcpy(yk2 + (size_t)i * n, y, sizeof(double) * n);
    for (int its = 0; its < max_its; ++its) {
        ++its_reached;
        memcpy(yk1, yk2, sizeof(double) * s * n);
        double norm2 = 0.0;
        for (int i = 0; i < s; ++i) orc_rhs(n, dim, yk2 + (size_t)i * n, xs[i], f + (size_t)i * n);
        for (int i = 0; i < s; ++i)
            for (int j = 0; j < n; ++j) {
                double tmp = y[j];
                for (int k = 0; k < s; ++k) tmp += dx * a[i][k] * f[(size_t)k * n + j];
                yk2[(size_t)i * n + j] = tmp;
            }
        for (int i = 0; i < s; ++i)
            for (int j = 0; j < n; ++j) {
                double df = yk1[(size_t)i * n + j] - yk2[(size_t)i * n + j];
                norm2 += df * df;
            }
        norm2 = sqrt(norm2 / (n * s));
        double p10 = precision;
        if (its > max_its / 2) p10 = precision * 10.0 * (2.0 * (double)its / (double)max_its - 0.5);
        if (norm2 < p10) {
            converged = 1;
            break;
        }
    }
    for (int i = 0; i < s; ++i)
        for (int j = 0; j < n; ++j) y[j] += dx * b[i] * f[(size_t)i * n + j];
    memcpy(yout, y, sizeof(double) * n);
    if (its_out) *its_out = its_reached;
    free(y);
    free(f);
    free(yk1);
    free(yk2);
    return converged;
}

/* ------------------------------------------------------------------------ */
/* ShootingSolver                                                            */
/* ------------------------------------------------------------------------ */

/* integrateToMatchPoint (ShootingSolver.cpp:53-145).  Returns ORC_OK, or
 * ORC_IRK_NO_CONVERGENCE with *fail_index = the grid index the failing step
 * started from (the reference prints it and exits).                         */
int orc_sweep(const orc_cfg* c, const double* grid, int start, int end, int forward, const double* yinit,
              double* yfinal, int* fail_index, long long* rhs_evals)
{
    const int n = c->ntau;
    const int s = c->scheme == 1 ? 1 : (c->scheme == 3 ? 3 : 2);
    double* y1 = dalloc(n);
    double* y2 = dalloc(n);
    memcpy(y1, yinit, sizeof(double) * n);
    int status = ORC_OK;
    if (forward) {
        for (int i = start; i < end; ++i) {
            int its = 0;
            int ok = orc_irk_step(n, c->dim, c->scheme, c->prec_irk, c->max_irk, y1, grid[i], grid[i + 1], y2, &its);
            if (rhs_evals) *rhs_evals += (long long)its * s;
            if (!ok) {
                status = ORC_IRK_NO_CONVERGENCE;
                if (fail_index) *fail_index = i;
                break;
            }
            memcpy(y1, y2, sizeof(double) * n);
        }
    } else {
        for (int i = start; i > end; --i) {
            int its = 0;
            int ok = orc_irk_step(n, c->dim, c->scheme, c->prec_irk, c->max_irk, y1, grid[i], grid[i - 1], y2, &its);
            if (rhs_evals) *rhs_evals += (long long)its * s;
            if (!ok) {
                status = ORC_IRK_NO_CONVERGENCE;
                if (fail_index) *fail_index = i;
                break;
            }
            memcpy(y1, y2, sizeof(double) * n);
        }
    }
    memcpy(yfinal, y1, sizeof(double) * n);
    free(y1);
    free(y2);
    return status;
}

/* computeMismatch (ShootingSolver.cpp:154-182) */
int orc_mismatch(int n, const double* yl, const double* yr, double precision, double* out)
{
    for (int i = 0; i < n; ++i) out[i] = yr[i] - yl[i];
    int status = (RE(out, 2) > precision) ? ORC_DELTA_MISMATCH : ORC_OK;
    RE(out, 2) = RE(yl, 2);
    return status;
}

/* ------------------------------------------------------------------------ */
/* NewtonSolver                                                              */
/* ------------------------------------------------------------------------ */

/* generateGrid (NewtonSolver.cpp:477-519): uniform in z = log x - log(1-x) */
void orc_grid(const orc_cfg* c, double* g)
{
    const int il = 0, im = c->nl, ir = c->nl + c->nr;
    g[il] = c->xl;
    g[im] = c->xm;
    g[ir] = c->xr;
    double zl = log(c->xl) - log(1.0 - c->xl);
    double zm = log(c->xm) - log(1.0 - c->xm);
    double zr = log(c->xr) - log(1.0 - c->xr);
    double dzl = (zm - zl) / (double)c->nl;
    double dzr = (zr - zm) / (double)c->nr;
    for (int j = il + 1; j < im; ++j) {
        double e = zl + (double)(j - il) * dzl;
        g[j] = exp(e) / (1.0 + exp(e));
    }
    for (int j = im + 1; j < ir; ++j) {
        double e = zm + (double)(j - im) * dzr;
        g[j] = exp(e) / (1.0 + exp(e));
    }
}

/* NewtonSolver::shoot (NewtonSolver.cpp:403-423) with initializeInput (:428-432) */
int orc_shoot(const orc_cfg* c, const double* grid, const double* in0, double* out0, long long* rhs_evals)
{
    const int n = c->ntau, nn = 3 * n / 4;
    double* in = dalloc(nn);
    memcpy(in, in0, sizeof(double) * nn);
    const double delta = in[2 * nn / 3 + 2];
    in[2 * nn / 3 + 2] = 0.0;
    double *up = dalloc(n), *psic = dalloc(n), *fc = dalloc(n);
    orc_unpack(n, in, up, psic, fc);
    double *yl = dalloc(n), *yr = dalloc(n), *yl2 = dalloc(n), *yr2 = dalloc(n), *mm = dalloc(n);
    orc_left_expansion(n, c->dim, c->xl, fc, psic, delta, yl);
    orc_right_expansion(n, c->dim, c->xr, up, delta, yr);
    int fail = -1;
    int st = orc_sweep(c, grid, 0, c->nl, 1, yl, yl2, &fail, rhs_evals);
    if (st == ORC_OK) st = orc_sweep(c, grid, c->nl + c->nr, c->nl, 0, yr, yr2, &fail, rhs_evals);
    if (st == ORC_OK) st = orc_mismatch(n, yl2, yr2, c->prec_irk, mm);
    double *u = dalloc(n), *v = dalloc(n), *f = dalloc(n);
    orc_state_to_fields_light(n, mm, u, v, f);
    orc_pack(n, u, v, f, out0);
    free(in); free(up); free(psic); free(fc); free(yl); free(yr); free(yl2); free(yr2); free(mm);
    free(u); free(v); free(f);
    return st;
}

/* assembleJacobian, serial branch (NewtonSolver.cpp:667-699), columns [c0,c1):
 * cols[(col-c0)*Nnewton + row] = (F(u + eps e_col)_row - F(u)_row) / eps.   */
int orc_jacobian_columns(const orc_cfg* c, const double* grid, const double* in0, const double* out0, int c0,
                         int c1, double* cols, long long* rhs_evals)
{
    const int nn = 3 * c->ntau / 4;
    double* pin = dalloc(nn);
    double* pout = dalloc(nn);
    int status = ORC_OK;
    for (int col = c0; col < c1; ++col) {
        memcpy(pin, in0, sizeof(double) * nn);
        pin[col] += c->eps_newton;
        int st = orc_shoot(c, grid, pin, pout, rhs_evals);
        if (st != ORC_OK && status == ORC_OK) status = st;
        for (int j = 0; j < nn; ++j) cols[(size_t)(col - c0) * nn + j] = (pout[j] - out0[j]) / c->eps_newton;
    }
    free(pin);
    free(pout);
    return status;
}

/* LAPACK dgesv semantics for solveLinearSystem (NewtonSolver.cpp:739-757):
 * LU with partial pivoting (first maximal |a| in the column, as idamax),
 * then forward and back substitution.  a is row-major and overwritten.     */
int orc_dgesv(int n, double* a, double* b)
{
    for (int k = 0; k < n; ++k) {
        int p = k;
        double best = fabs(a[(size_t)k * n + k]);
        for (int i = k + 1; i < n; ++i) {
            double v = fabs(a[(size_t)i * n + k]);
            if (v > best) {
                best = v;
                p = i;
            }
        }
        if (best == 0.0) return ORC_SINGULAR;
        if (p != k) {
            for (int j = 0; j < n; ++j) {
                double t = a[(size_t)k * n + j];
                a[(size_t)k * n + j] = a[(size_t)p * n + j];
                a[(size_t)p * n + j] = t;
            }
            double t = b[k];
            b[k] = b[p];
            b[p] = t;
        }
        const double piv = a[(size_t)k * n + k];
        for (int i = k + 1; i < n; ++i) {
            double l = a[(size_t)i * n + k] / piv;
            a[(size_t)i * n + k] = l;
            for (int j = k + 1; j < n; ++j) a[(size_t)i * n + j] -= l * a[(size_t)k * n + j];
            b[i] -= l * b[k];
        }
    }
    for (int i = n - 1; i >= 0; --i) {
        double s = b[i];
        for (int j = i + 1; j < n; ++j) s -= a[(size_t)i * n + j] * b[j];
        b[i] = s / a[(size_t)i * n + i];
    }
    return ORC_OK;
}

/* computeL2Norm (NewtonSolver.cpp:763-768): sqrt(mean(v^2)) */
double orc_rms(int n, const double* v)
{
    double s = 0.0;
    for (int i = 0; i < n; ++i) s += v[i] * v[i];
    return sqrt(s / (double)n);
}
