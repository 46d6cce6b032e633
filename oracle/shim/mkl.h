/* Minimal stand-in for <mkl.h> so the reference's array.cpp compiles without
 * MKL.  Only the dense array::Matrix methods call LAPACKE (array.cpp:344, 556,
 * 605, 670, 674); the sparse and block solver path never does.  The stubs in
 * lapacke_stub.cpp abort if anything reaches them.
 *
 * Test infrastructure only: part of the oracle build, never of the product. */
#pragma once
#include <stddef.h>

typedef int lapack_int;
#define LAPACK_ROW_MAJOR 101
#define LAPACK_COL_MAJOR 102

#ifdef __cplusplus
extern "C" {
#endif
lapack_int LAPACKE_dpotrf(int layout, char uplo, lapack_int n, double* a, lapack_int lda);
lapack_int LAPACKE_dpotri(int layout, char uplo, lapack_int n, double* a, lapack_int lda);
lapack_int LAPACKE_dgetrf(int layout, lapack_int m, lapack_int n, double* a, lapack_int lda,
                          lapack_int* ipiv);
#ifdef __cplusplus
}
#endif
