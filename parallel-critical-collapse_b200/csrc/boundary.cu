// boundary.cu -- boundary-data (prologue) and mismatch/pack/difference
// (epilogue) kernels of a Jacobian build.  See boundary.cuh.
#include "boundary.cuh"
#include "pcc_internal.h"

namespace pcc {

enum {
    A_Z = 0,
    A_UP,
    A_PSIC,
    A_FC,
    A_FR,
    A_W  // first free work array
};

// InitialConditionGenerator::unpackSpectralFields (InitialConditionGenerator.cpp:
// 719-758) for one of the three packed fields: which = 0 (Odd1 = U_p),
// 1 (Odd2 = psi_c), 2 (Even = f_c).  z has the Delta slot already zeroed.
__device__ void unpack_field(const Blk& B, const double* z, int nn, int which, double* out)
{
    const int n = B.n, h = n / 2;
    double2* half = B.sb;  // n/2 complex
    for (int k = threadIdx.x; k < h; k += blockDim.x) half[k] = make_double2(0.0, 0.0);
    Blk::sync();
    if (threadIdx.x == 0) {
        const int off = which * nn / 3;
        for (int j = 0; j < nn / 6; ++j) {
            const double re = z[2 * j + off], im = z[2 * j + 1 + off];
            if (which < 2) {
                half[2 * j + 1] = make_double2(re, im);
                half[h - 2 * j - 1] = make_double2(re, -im);
            } else {
                half[2 * j] = make_double2(re, im);
                if (j != 0) half[h - 2 * j] = make_double2(re, -im);
            }
        }
        if (which == 2) half[0].y = 0.0;
    }
    Blk::sync();
    for (int k = threadIdx.x; k < n; k += blockDim.x) B.sa[k] = double_modes_at(half, h, k);
    Blk::sync();
    if (which == 2 && threadIdx.x == 0) {
        const double c = z[2 * nn / 3 + 1] / 2.0;
        B.sa[nn / 3] = make_double2(c, 0.0);
        B.sa[nn] = make_double2(c, 0.0);
    }
    Blk::sync();
    B.backward();
    B.store_real(out);
}

// InitialConditionGenerator::computeLeftExpansion (InitialConditionGenerator.cpp:37-239)
__device__ void left_expansion(const Blk& B, double d, double xl, const double* f0, const double* psi0,
                               double delta, double* y)
{
    const int n = B.n;
    double* df = B.arr(A_W + 0);
    double* d2f = B.arr(A_W + 1);
    double* d3f = B.arr(A_W + 2);
    double* c1 = B.arr(A_W + 3);
    double* c2 = B.arr(A_W + 4);
    double* u1 = B.arr(A_W + 5);
    double* du1 = B.arr(A_W + 6);
    double* d2u1 = B.arr(A_W + 7);
    double* d3u1 = B.arr(A_W + 8);
    double* d4u1 = B.arr(A_W + 9);
    double* U = B.arr(A_W + 10);
    double* V = B.arr(A_W + 11);
    double* F = B.arr(A_W + 12);

    B.tau_derivative(f0, df, delta);
    B.tau_derivative(df, d2f, delta);
    B.tau_derivative(d2f, d3f, delta);
    for (int j = threadIdx.x; j < n; j += blockDim.x) {
        c1[j] = 1.0;
        c2[j] = -(d - 1.0) * psi0[j] * f0[j];
    }
    Blk::sync();
    B.solve_inhom(c1, c2, u1, delta, B.arr(A_FR));
    B.tau_derivative(u1, du1, delta);
    B.tau_derivative(du1, d2u1, delta);
    B.tau_derivative(d2u1, d3u1, delta);
    B.tau_derivative(d3u1, d4u1, delta);

    for (int j = threadIdx.x; j < n; j += blockDim.x) {
        const double f = f0[j], psi = psi0[j];
        const double u1j = u1[j];
        const double du = du1[j], d2u = d2u1[j], d3u = d3u1[j], d4u = d4u1[j];
        const double dfj = df[j], d2fj = d2f[j], d3fj = d3f[j];
        const double p3 = pow(d - 2.0, 3);

        const double v1 = u1j;
        const double f2 = ((d - 3.0) * p3 * f * pow(u1j, 2)) / (8.0 * (d - 1.0));
        const double u2 = -psi;
        const double v2 = psi;
        const double common3 =
            ((d - 3.0) * p3 * pow(f, 3) * pow(u1j, 3) + 4.0 * dfj * (u1j + du) - 4.0 * f * (2.0 * u1j + 3.0 * du + d2u));
        const double u3 = common3 / (8.0 * (1.0 - d) * pow(f, 3));
        const double v3 = u3;
        const double f4 =
            -((d - 3.0) * p3 *
              ((p3 * (5.0 - 6.0 * d + d * d) * pow(f, 3) * pow(u1j, 4)) + 8.0 * (d - 1.0) * dfj * u1j * (du + u1j) -
               8.0 * f * (pow(du, 2) + ((d - 1.0) * d2u + (-1.0 + 3.0 * d) * du) * u1j + (-1.0 + 2.0 * d) * pow(u1j, 2)))) /
            (128.0 * pow(d - 1.0, 2) * (1.0 + d) * pow(f, 2));
        const double u4 =
            (-192.0 * (d - 1.0) * pow(dfj, 2) * du * pow(f, 2) + 192.0 * (d - 1.0) * d2u * dfj * pow(f, 3) +
             64.0 * (d - 1.0) * d2fj * du * pow(f, 3) + 640.0 * (d - 1.0) * dfj * du * pow(f, 3) -
             64.0 * (d - 1.0) * (6.0 * d2u + d3u) * pow(f, 4) - 704.0 * (d - 1.0) * du * pow(f, 4) -
             192.0 * (d - 1.0) * pow(dfj, 2) * pow(f, 2) * u1j + 64.0 * (d - 1.0) * d2fj * pow(f, 3) * u1j +
             448.0 * (d - 1.0) * dfj * pow(f, 3) * u1j - 384.0 * (d - 1.0) * pow(f, 4) * u1j +
             32.0 * p3 * (3.0 - 7.0 * d + 2.0 * d * d) * pow(f, 6) * pow(u1j, 2) * (du + u1j)) /
            (128.0 * pow(d - 1.0, 2) * (1.0 + d) * pow(f, 7));
        const double v4 = -u4;
        const double qd = 3.0 - 13.0 * d + 4.0 * d * d;
        const double u5 =
            (-64.0 * (d - 1.0) * d2fj * d2u * pow(f, 2) - 16.0 * (d - 1.0) * (15.0 * d2fj + d3fj) * du * pow(f, 2) -
             32.0 * (d - 1.0) * dfj * (20.0 * d2u + 3.0 * d3u + 40.0 * du) * pow(f, 2) +
             560.0 * (d - 1.0) * d2u * pow(f, 3) + 160.0 * (d - 1.0) * d3u * pow(f, 3) +
             16.0 * (d - 1.0) * d4u * pow(f, 3) + 800.0 * (d - 1.0) * du * pow(f, 3) -
             16.0 * (d - 1.0) * (11.0 * d2fj + d3fj) * pow(f, 2) * u1j - 736.0 * (d - 1.0) * dfj * pow(f, 2) * u1j +
             384.0 * (d - 1.0) * pow(f, 3) * u1j - 8.0 * p3 * qd * pow(du, 2) * pow(f, 5) * u1j +
             8.0 * p3 * qd * dfj * du * pow(f, 4) * pow(u1j, 2) - 8.0 * p3 * qd * (d2u + 5.0 * du) * pow(f, 5) * pow(u1j, 2) +
             8.0 * p3 * qd * dfj * pow(f, 4) * pow(u1j, 3) - 24.0 * p3 * qd * pow(f, 5) * pow(u1j, 3) +
             pow(d - 2.0, 6) * (3.0 + 29.0 * d - 19.0 * d * d + 3.0 * d * d * d) * pow(f, 7) * pow(u1j, 5) -
             240.0 * (d - 1.0) * pow(dfj, 3) * (du + u1j) +
             80.0 * (d - 1.0) * dfj * f * (2.0 * d2fj * du + dfj * (3.0 * d2u + 11.0 * du) + 2.0 * (d2fj + 4.0 * dfj) * u1j)) /
            (128.0 * pow(d - 1.0, 2) * (1.0 + d) * pow(f, 7));
        const double v5 = u5;
        U[j] = xl * u1j + pow(xl, 2) * u2 + pow(xl, 3) * u3 + pow(xl, 4) * u4 + pow(xl, 5) * u5;
        V[j] = xl * v1 + pow(xl, 2) * v2 + pow(xl, 3) * v3 + pow(xl, 4) * v4 + pow(xl, 5) * v5;
        F[j] = f + pow(xl, 2) * f2 + pow(xl, 4) * f4;
    }
    Blk::sync();
    B.fields_to_state(U, V, F, y);
    if (threadIdx.x == 0) y[4] = delta;  // Re Y[2] = Delta
    Blk::sync();
}

// InitialConditionGenerator::computeRightExpansion (InitialConditionGenerator.cpp:252-667,
// serial branch :460-619)
__device__ void right_expansion(const Blk& B, double d, double xr, const double* u0, double delta, double* y)
{
    const int n = B.n;
    const double dx = xr - 1.0;
    const double p3 = pow(d - 2.0, 3);
    double* du0 = B.arr(A_W + 0);
    double* d2u0 = B.arr(A_W + 1);
    double* c1 = B.arr(A_W + 2);
    double* c2 = B.arr(A_W + 3);
    double* ia20 = B.arr(A_W + 4);
    double* v0 = B.arr(A_W + 5);
    double* f1 = B.arr(A_W + 6);
    double* u1 = B.arr(A_W + 7);
    double* ia21 = B.arr(A_W + 8);
    double* v1 = B.arr(A_W + 9);
    double* f2 = B.arr(A_W + 10);
    double* ia22 = B.arr(A_W + 11);
    double* u2 = B.arr(A_W + 12);
    double* du2 = B.arr(A_W + 13);
    double* v2 = B.arr(A_W + 14);
    double* f3 = B.arr(A_W + 15);
    double* ia23 = B.arr(A_W + 16);
    double* u3 = B.arr(A_W + 17);
    double* v3 = B.arr(A_W + 18);
    double* F = B.arr(A_W + 19);
    double* U = B.arr(A_W + 20);
    double* V = B.arr(A_W + 21);
    double* fr = B.arr(A_FR);

    // du0 = IFFT(D FFT u0), d2u0 = IFFT(D D FFT u0) (:266-271); the second
    // spectrum is recomputed rather than kept (sb is the FFT's partner buffer)
    B.tau_derivative(u0, du0, delta);
    B.load_real(u0);
    B.forward();
    B.differentiate(delta);
    B.differentiate(delta);
    B.backward();
    B.store_real(d2u0);

    for (int j = threadIdx.x; j < n; j += blockDim.x) {
        c1[j] = 3.0 - d - p3 * u0[j] * u0[j] / 4.0;
        c2[j] = d - 3.0;
    }
    Blk::sync();
    B.solve_inhom(c1, c2, ia20, delta, fr);

    for (int j = threadIdx.x; j < n; j += blockDim.x) {
        c1[j] = (6.0 - 2.0 * d + (d - 2.0) * ia20[j]) / (2.0 * ia20[j]);
        c2[j] = (d - 2.0) * u0[j] / 2.0;
    }
    Blk::sync();
    B.solve_inhom(c1, c2, v0, delta, fr);

    for (int j = threadIdx.x; j < n; j += blockDim.x) {
        f1[j] = 3.0 - d + (d - 3.0) / ia20[j];
        ia21[j] = -ia20[j] * (8.0 * (d - 3.0) + p3 * (u0[j] * u0[j] + v0[j] * v0[j])) / 8.0 + d - 3.0;
        u1[j] = ((d - 2.0 - 2.0 * (d - 3.0) / ia20[j]) * u0[j] + (d - 2.0) * v0[j]) / 4.0 - du0[j] / 2.0;
    }
    Blk::sync();
    for (int j = threadIdx.x; j < n; j += blockDim.x) {
        c1[j] = (6.0 - 2.0 * d + d * ia20[j] - 2.0 * f1[j] * ia20[j]) / (2.0 * ia20[j]);
        c2[j] = (2.0 * (3.0 - d) * (f1[j] - 1.0) * ia20[j] * v0[j] + 2.0 * (d - 3.0) * ia21[j] * v0[j] +
                 (d - 2.0) * pow(ia20[j], 2) * ((f1[j] - 1.0) * u0[j] + u1[j] + (f1[j] - 1.0) * v0[j])) /
                (2.0 * pow(ia20[j], 2));
    }
    Blk::sync();
    B.solve_inhom(c1, c2, v1, delta, fr);

    for (int j = threadIdx.x; j < n; j += blockDim.x) {
        f2[j] = (d - 3.0) * ((f1[j] - 1.0) * (1.0 - ia20[j]) * ia20[j] - ia21[j]) / (2.0 * pow(ia20[j], 2));
        ia22[j] = (3.0 - d - (ia21[j] - ia20[j]) * (8.0 * (d - 3.0) + p3 * (pow(u0[j], 2) + pow(v0[j], 2))) / 8.0 -
                   p3 * ia20[j] * (u0[j] * u1[j] + v0[j] * v1[j]) / 4.0) /
                  2.0;
    }
    Blk::sync();
    for (int j = threadIdx.x; j < n; j += blockDim.x) {
        const double a0 = ia20[j];
        const double A = 4.0 * (3.0 - d) * (d - 6.0 + f1[j]) * a0;
        const double Bq = (d - 2.0) * (d - 8.0 + 2.0 * f1[j]) * pow(a0, 2);
        const double C = 4.0 * (d - 3.0) * (d - 3.0 + 2.0 * ia21[j]);
        const double D = -(d - 3.0) * p3 * a0 * pow(u0[j], 3);
        const double E = (4.0 * (6.0 - 2.0 * d + (d - 2.0) * a0) * u1[j] +
                          (d - 2.0) * v0[j] * (6.0 - 2.0 * d + (d - 8.0 + 2.0 * f1[j]) * a0) - 8.0 * a0 * v1[j] +
                          4.0 * d * a0 * v1[j] - 12.0 * du0[j] + 4.0 * d * du0[j] + 8.0 * a0 * du0[j] -
                          2.0 * d * a0 * du0[j] + 4.0 * f1[j] * a0 * du0[j] + 4.0 * a0 * d2u0[j]) *
                         a0;
        double u2j = (A + Bq + C) * u0[j] + D + E;
        u2j /= 32.0 * pow(a0, 2);
        u2[j] = u2j;
    }
    Blk::sync();
    B.tau_derivative(u2, du2, delta);

    for (int j = threadIdx.x; j < n; j += blockDim.x) {
        const double a0 = ia20[j], a1 = ia21[j], a2 = ia22[j];
        c1[j] = 1.0 + d / 2.0 - 2.0 * f1[j] + (3.0 - d) / a0;
        c2[j] = (2.0 * (3.0 - d) * pow(a1, 2) * v0[j] +
                 2.0 * (d - 3.0) * pow(a0, 2) * ((f1[j] - 1.0 - f2[j]) * v0[j] - (f1[j] - 1.0) * v1[j]) +
                 ((d - 2.0) * ((1.0 - f1[j] + f2[j]) * u0[j] + (f1[j] - 1.0) * u1[j] + u2[j] + (1.0 - f1[j] + f2[j]) * v0[j]) +
                  ((d - 2.0) * (f1[j] - 1.0) - 2.0 * f2[j]) * v1[j]) *
                     pow(a0, 3) +
                 2.0 * (d - 3.0) * a0 * (a2 * v0[j] + a1 * ((f1[j] - 1.0) * v0[j] + v1[j]))) /
                (2.0 * pow(a0, 3));
    }
    Blk::sync();
    B.solve_inhom(c1, c2, v2, delta, fr);

    for (int j = threadIdx.x; j < n; j += blockDim.x) {
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
    Blk::sync();
    for (int j = threadIdx.x; j < n; j += blockDim.x) {
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
    Blk::sync();
    B.solve_inhom(c1, c2, v3, delta, fr);

    for (int j = threadIdx.x; j < n; j += blockDim.x) {
        F[j] = 1.0 + dx * f1[j] + dx * dx * f2[j] + dx * dx * dx * f3[j];
        U[j] = u0[j] + dx * u1[j] + dx * dx * u2[j] + dx * dx * dx * u3[j];
        V[j] = v0[j] + dx * v1[j] + dx * dx * v2[j] + dx * dx * dx * v3[j];
    }
    Blk::sync();
    B.fields_to_state(U, V, F, y);
    if (threadIdx.x == 0) y[4] = delta;
    Blk::sync();
}

// packSpectralFields (InitialConditionGenerator.cpp:678-711) of one field into z
__device__ void pack_field(const Blk& B, const double* x, int nn, int which, double* z)
{
    const int n = B.n;
    B.load_real(x);
    B.forward();
    // halveModes: half[k] = sa[k] (k < n/4), sa[n/4] + sa[3n/4] (k = n/4), sa[n/2+k] above
    if (threadIdx.x == 0) {
        const int off = which * nn / 3;
        for (int j = 0; j < nn / 6; ++j) {
            const int k = which < 2 ? 2 * j + 1 : 2 * j;  // both below n/4
            z[2 * j + off] = B.sa[k].x;
            z[2 * j + 1 + off] = B.sa[k].y;
        }
        if (which == 2) z[2 * nn / 3 + 1] = B.sa[n / 4].x + B.sa[3 * n / 4].x;
    }
    Blk::sync();
}

__global__ void __launch_bounds__(256) prologue_kernel(BoundaryParams P)
{
    extern __shared__ double2 sh[];
    Blk B;
    B.n = P.ntau;
    B.tw = P.tw;
    B.sa = sh;
    B.sb = sh + P.ntau;
    B.scr = P.scratch + (size_t)blockIdx.x * kBoundaryArrays * P.ntau;
    __shared__ int item_s;
    for (;;) {
        if (threadIdx.x == 0) item_s = atomicAdd(P.work_counter, 1);
        __syncthreads();
        const int item = item_s;
        __syncthreads();
        if (item >= P.n_items) break;
        const int slot = P.sweeps ? P.sweeps[item] : item;
        const int col = P.sweeps ? slot >> 1 : P.c0 + item / 2, side = slot & 1;
        double* z = B.arr(A_Z);
        for (int k = threadIdx.x; k < P.nn; k += blockDim.x) {
            double v = P.in0[k];
            if (k == col) v += P.eps;
            z[k] = v;
        }
        __syncthreads();
        const double delta = z[2 * P.nn / 3 + 2];
        __syncthreads();
        if (threadIdx.x == 0) z[2 * P.nn / 3 + 2] = 0.0;
        __syncthreads();
        double* y = P.yinit + (size_t)slot * P.ntau;
        if (side == 0) {
            unpack_field(B, z, P.nn, 1, B.arr(A_PSIC));
            unpack_field(B, z, P.nn, 2, B.arr(A_FC));
            left_expansion(B, P.dim, P.xl, B.arr(A_FC), B.arr(A_PSIC), delta, y);
        } else {
            unpack_field(B, z, P.nn, 0, B.arr(A_UP));
            right_expansion(B, P.dim, P.xr, B.arr(A_UP), delta, y);
        }
    }
}

__global__ void __launch_bounds__(256) epilogue_kernel(BoundaryParams P)
{
    extern __shared__ double2 sh[];
    Blk B;
    B.n = P.ntau;
    B.tw = P.tw;
    B.sa = sh;
    B.sb = sh + P.ntau;
    B.scr = P.scratch + (size_t)blockIdx.x * kBoundaryArrays * P.ntau;
    __shared__ int item_s;
    const int n = P.ntau, h = n / 2;
    for (;;) {
        if (threadIdx.x == 0) item_s = atomicAdd(P.work_counter, 1);
        __syncthreads();
        const int item = item_s;
        __syncthreads();
        if (item >= P.n_items) break;
        int lcol = item, rcol = item;
        if (P.abs_slots) {
            const int col = P.c0 + item;
            lcol = P.reuse && !column_moves_left(col, P.nn) ? P.nn : col;
            rcol = P.reuse && !column_moves_right(col, P.nn) ? P.nn : col;
        }
        const double* yl = P.yfinal + (size_t)(2 * lcol) * n;
        const double* yr = P.yfinal + (size_t)(2 * rcol + 1) * n;
        // computeMismatch: yR - yL, Delta guard, Re[2] := Re yL[2]
        double2* mm = B.sb;
        for (int k = threadIdx.x; k < h; k += blockDim.x)
            mm[k] = make_double2(yr[2 * k] - yl[2 * k], yr[2 * k + 1] - yl[2 * k + 1]);
        __syncthreads();
        if (threadIdx.x == 0) {
            P.status[item] = (mm[2].x > P.prec) ? 1 : 0;
            mm[2].x = yl[4];
        }
        __syncthreads();
        // StateVectorToFields, light variant (InitialConditionGenerator.cpp:891-932)
        for (int k = threadIdx.x; k < n; k += blockDim.x) B.sa[k] = double_modes_at(mm, h, k);
        __syncthreads();
        if (threadIdx.x == 0) B.sa[2].x = -B.sa[n - 2].x;
        __syncthreads();
        B.backward();
        double* U = B.arr(A_W + 0);
        double* V = B.arr(A_W + 1);
        double* F = B.arr(A_W + 2);
        for (int j = threadIdx.x; j < h; j += blockDim.x) {
            const double2 a = B.sa[j], b = B.sa[j + h];
            const double u = 0.5 * (a.x - b.x), v = 0.5 * (a.y - b.y), f = 0.5 * (a.y + b.y);
            U[j] = u;
            V[j] = v;
            F[j] = f;
            U[j + h] = -u;
            V[j + h] = -v;
            F[j + h] = f;
        }
        __syncthreads();
        double* z = P.outc + (size_t)item * P.nn;
        pack_field(B, U, P.nn, 0, z);
        pack_field(B, V, P.nn, 1, z);
        pack_field(B, F, P.nn, 2, z);
    }
}

// J[row][c0 + i] = (outc[i][row] - out0[row]) / eps  (NewtonSolver.cpp:642-645)
__global__ void fd_kernel(const double* __restrict__ outc, const double* __restrict__ out0, double* J, int nn,
                          int c0, int ncols, double eps)
{
    __shared__ double tile[32][33];
    const int ci0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
    for (int i = threadIdx.y; i < 32; i += blockDim.y) {
        const int ci = ci0 + i, r = r0 + threadIdx.x;
        if (ci < ncols && r < nn) tile[i][threadIdx.x] = (outc[(size_t)ci * nn + r] - out0[r]) / eps;
    }
    __syncthreads();
    for (int i = threadIdx.y; i < 32; i += blockDim.y) {
        const int r = r0 + i, ci = ci0 + threadIdx.x;
        if (ci < ncols && r < nn) J[(size_t)r * nn + c0 + ci] = tile[threadIdx.x][i];
    }
}

// pack (dir = 0: fields -> z) or unpack (dir = 1: z -> fields), one CTA
__global__ void __launch_bounds__(256) pack_kernel(int ntau, const double* __restrict__ tw, double* scratch,
                                                   double* up, double* psic, double* fc, double* z, int dir)
{
    extern __shared__ double2 sh[];
    Blk B;
    B.n = ntau;
    B.tw = reinterpret_cast<const double2*>(tw);
    B.sa = sh;
    B.sb = sh + ntau;
    B.scr = scratch;
    const int nn = 3 * ntau / 4;
    if (dir == 0) {
        pack_field(B, up, nn, 0, z);
        pack_field(B, psic, nn, 1, z);
        pack_field(B, fc, nn, 2, z);
    } else {
        unpack_field(B, z, nn, 0, up);
        unpack_field(B, z, nn, 1, psic);
        unpack_field(B, z, nn, 2, fc);
    }
}

// expansions from fields (item 0: left from fc/psic, item 1: right from up)
__global__ void __launch_bounds__(256) expansion_kernel(int ntau, double dim, double delta, double xl, double xr,
                                                        const double2* __restrict__ tw, double* scratch,
                                                        const double* fc, const double* psic, const double* up,
                                                        double* yl, double* yr)
{
    extern __shared__ double2 sh[];
    Blk B;
    B.n = ntau;
    B.tw = tw;
    B.sa = sh;
    B.sb = sh + ntau;
    B.scr = scratch + (size_t)blockIdx.x * kBoundaryArrays * ntau;
    if (blockIdx.x == 0 && yl) left_expansion(B, dim, xl, fc, psic, delta, yl);
    if (blockIdx.x == 1 && yr) right_expansion(B, dim, xr, up, delta, yr);
}

cudaError_t launch_expansions(int ntau, double dim, double delta, double xl, double xr, const double2* tw,
                              double* scratch, const double* fc, const double* psic, const double* up, double* yl,
                              double* yr, cudaStream_t st)
{
    const size_t smem = 2 * (size_t)ntau * sizeof(double2);
    cudaError_t e = cudaFuncSetAttribute(expansion_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    expansion_kernel<<<2, 256, smem, st>>>(ntau, dim, delta, xl, xr, tw, scratch, fc, psic, up, yl, yr);
    return cudaGetLastError();
}

// batched unscaled DFT, one CTA per series
__global__ void __launch_bounds__(256) dft_kernel(int n, int sign, const double2* __restrict__ tw,
                                                  const double2* in, double2* out)
{
    extern __shared__ double2 sh[];
    Blk B;
    B.n = n;
    B.tw = tw;
    B.sa = sh;
    B.sb = sh + n;
    B.scr = nullptr;
    const double2* x = in + (size_t)blockIdx.x * n;
    for (int j = threadIdx.x; j < n; j += blockDim.x) B.sa[j] = x[j];
    __syncthreads();
    B.fft(sign);
    double2* y = out + (size_t)blockIdx.x * n;
    for (int j = threadIdx.x; j < n; j += blockDim.x) y[j] = B.sa[j];
}

// The Debug field export of ShootingSolver::integrateToMatchPoint
// (ShootingSolver.cpp:85-97, 128-138): a state snapshot at x ->
// InitialConditionGenerator::StateVectorToFields (InitialConditionGenerator.cpp:
// 791-884: doubleModes, the phase fix, the inverse transform and the split,
// the IA2 constraint solve) -> A = sqrt(1/IA2), U, V, f.  One CTA per snapshot.
__global__ void __launch_bounds__(256) debug_fields_kernel(int ntau, double dim, double dm2c, int count,
                                                          const double* __restrict__ states,
                                                          const double* __restrict__ xs, double* fields,
                                                          double* scratch, const double2* __restrict__ tw)
{
    extern __shared__ double2 sh[];
    Blk B;
    B.n = ntau;
    B.tw = tw;
    B.sa = sh;
    B.sb = sh + ntau;
    B.scr = scratch + (size_t)blockIdx.x * kBoundaryArrays * ntau;
    const int h = ntau / 2;
    for (int k = blockIdx.x; k < count; k += gridDim.x) {
        const double2* y = reinterpret_cast<const double2*>(states + (size_t)k * ntau);
        const double delta = y[2].x;
        const double x = xs[k];
        for (int j = threadIdx.x; j < ntau; j += blockDim.x) B.sa[j] = double_modes_at(y, h, j);
        B.sync();
        if (threadIdx.x == 0) B.sa[2].x = -B.sa[ntau - 2].x;  // Re c[2] = -Re c[N-2]
        B.sync();
        B.backward();
        double *U = B.arr(0), *V = B.arr(1), *F = B.arr(2), *k1 = B.arr(3), *k2 = B.arr(4), *ia2 = B.arr(5);
        for (int j = threadIdx.x; j < h; j += blockDim.x) {
            const double2 a = B.sa[j], b = B.sa[j + h];
            const double u = 0.5 * (a.x - b.x), v = 0.5 * (a.y - b.y), f = 0.5 * (a.y + b.y);
            U[j] = u;
            V[j] = v;
            F[j] = f;
            U[j + h] = -u;
            V[j + h] = -v;
            F[j + h] = f;
        }
        B.sync();
        for (int j = threadIdx.x; j < ntau; j += blockDim.x) {
            k1[j] = -(((x + F[j]) * U[j] * U[j] + (x - F[j]) * V[j] * V[j]) * dm2c / (8.0 * x) + (dim - 3.0));
            k2[j] = dim - 3.0;
        }
        B.sync();
        B.solve_inhom(k1, k2, ia2, delta, B.arr(6));
        double* o = fields + (size_t)k * 4 * ntau;
        for (int j = threadIdx.x; j < ntau; j += blockDim.x) {
            o[j] = sqrt(1.0 / ia2[j]);
            o[ntau + j] = U[j];
            o[2 * ntau + j] = V[j];
            o[3 * ntau + j] = F[j];
        }
        B.sync();
    }
}

cudaError_t launch_debug_fields(int ntau, double dim, double dm2c, int count, const double* states, const double* xs,
                                double* fields, double* scratch, int ctas, const double2* tw, cudaStream_t st)
{
    const size_t smem = 2 * (size_t)ntau * sizeof(double2);
    cudaError_t e = cudaFuncSetAttribute(debug_fields_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    debug_fields_kernel<<<ctas < count ? ctas : count, 256, smem, st>>>(ntau, dim, dm2c, count, states, xs, fields,
                                                                        scratch, tw);
    return cudaGetLastError();
}

cudaError_t launch_dft(int n, int count, int sign, const double2* tw, const double2* in, double2* out,
                       cudaStream_t st)
{
    const size_t smem = 2 * (size_t)n * sizeof(double2);
    cudaError_t e = cudaFuncSetAttribute(dft_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    dft_kernel<<<count, 256, smem, st>>>(n, sign, tw, in, out);
    return cudaGetLastError();
}

cudaError_t launch_pack(int ntau, const double2* tw, double* scratch, double* up, double* psic, double* fc, double* z,
                        int dir, cudaStream_t st)
{
    const size_t smem = 2 * (size_t)ntau * sizeof(double2);
    cudaError_t e = cudaFuncSetAttribute(pack_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    pack_kernel<<<1, 256, smem, st>>>(ntau, reinterpret_cast<const double*>(tw), scratch, up, psic, fc, z, dir);
    return cudaGetLastError();
}

// ------------------------------------------------------------ host launchers
cudaError_t launch_prologue(const BoundaryParams& P, int ctas, cudaStream_t st)
{
    const size_t smem = 2 * (size_t)P.ntau * sizeof(double2);
    cudaError_t e = cudaFuncSetAttribute(prologue_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    prologue_kernel<<<ctas, 256, smem, st>>>(P);
    return cudaGetLastError();
}

cudaError_t launch_epilogue(const BoundaryParams& P, int ctas, cudaStream_t st)
{
    const size_t smem = 2 * (size_t)P.ntau * sizeof(double2);
    cudaError_t e = cudaFuncSetAttribute(epilogue_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    epilogue_kernel<<<ctas, 256, smem, st>>>(P);
    return cudaGetLastError();
}

// Finite differences of columns in column-major order (no transpose):
// cols[i nn + row] = (outc[i nn + row] - out0[row]) / eps, i < ncols.
__global__ void fd_cols_kernel(const double* __restrict__ outc, const double* __restrict__ out0, double* cols,
                               int nn, int ncols, double eps)
{
    const size_t total = (size_t)ncols * nn;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x)
        cols[i] = (outc[i] - out0[i % nn]) / eps;
}

cudaError_t launch_fd_cols(const double* outc, const double* out0, double* cols, int nn, int ncols, double eps,
                           cudaStream_t st)
{
    const size_t total = (size_t)ncols * nn;
    const int blocks = (int)((total + 255) / 256 < 4096 ? (total + 255) / 256 : 4096);
    fd_cols_kernel<<<blocks < 1 ? 1 : blocks, 256, 0, st>>>(outc, out0, cols, nn, ncols, eps);
    return cudaGetLastError();
}

cudaError_t launch_fd(const double* outc, const double* out0, double* J, int nn, int c0, int ncols, double eps,
                      cudaStream_t st)
{
    dim3 grid((ncols + 31) / 32, (nn + 31) / 32), block(32, 8);
    fd_kernel<<<grid, block, 0, st>>>(outc, out0, J, nn, c0, ncols, eps);
    return cudaGetLastError();
}

}  // namespace pcc
