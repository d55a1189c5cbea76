/*
 * lapacke.h -- declarations of the two LAPACKE routines the reference calls
 * (NewtonSolver.cpp:749 LAPACKE_dgesv, common.cpp:187 LAPACKE_dgels).
 *
 * TEST INFRASTRUCTURE ONLY.  No LAPACKE header is installed in this image;
 * the oracle recipe links the reference against the LP64 OpenBLAS 0.3.15
 * shipped in the opencv-python-headless wheel, which exports both symbols.
 */
#pragma once

#ifdef __cplusplus
extern "C" {
#endif

typedef int lapack_int;

#define LAPACK_ROW_MAJOR 101
#define LAPACK_COL_MAJOR 102

lapack_int LAPACKE_dgesv(int matrix_layout, lapack_int n, lapack_int nrhs, double* a, lapack_int lda,
                         lapack_int* ipiv, double* b, lapack_int ldb);
lapack_int LAPACKE_dgels(int matrix_layout, char trans, lapack_int m, lapack_int n, lapack_int nrhs,
                         double* a, lapack_int lda, double* b, lapack_int ldb);

#ifdef __cplusplus
}
#endif
