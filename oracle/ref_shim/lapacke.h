/* Test-infrastructure shim (see cblas.h beside it): standard LAPACKE prototypes for the routines
 * the reference's LinearAlgebra.cpp calls, mapped onto scipy's prefixed OpenBLAS exports.
 * LP64: lapack_int is a 32-bit int, matching the bundled library. */
#ifndef RR_ORACLE_SHIM_LAPACKE_H
#define RR_ORACLE_SHIM_LAPACKE_H

#ifndef lapack_complex_double
#define lapack_complex_double double _Complex
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef int lapack_int;
#define LAPACK_ROW_MAJOR 101
#define LAPACK_COL_MAJOR 102

lapack_int scipy_LAPACKE_dsyev(int layout, char jobz, char uplo, lapack_int n, double* a, lapack_int lda, double* w);
lapack_int scipy_LAPACKE_zheev(int layout, char jobz, char uplo, lapack_int n, lapack_complex_double* a,
                               lapack_int lda, double* w);
lapack_int scipy_LAPACKE_dgetrf(int layout, lapack_int m, lapack_int n, double* a, lapack_int lda,
                                lapack_int* ipiv);
lapack_int scipy_LAPACKE_dgetri(int layout, lapack_int n, double* a, lapack_int lda, const lapack_int* ipiv);
lapack_int scipy_LAPACKE_zgetrf(int layout, lapack_int m, lapack_int n, lapack_complex_double* a, lapack_int lda,
                                lapack_int* ipiv);
lapack_int scipy_LAPACKE_zgetri(int layout, lapack_int n, lapack_complex_double* a, lapack_int lda,
                                const lapack_int* ipiv);

#define LAPACKE_dsyev scipy_LAPACKE_dsyev
#define LAPACKE_zheev scipy_LAPACKE_zheev
#define LAPACKE_dgetrf scipy_LAPACKE_dgetrf
#define LAPACKE_dgetri scipy_LAPACKE_dgetri
#define LAPACKE_zgetrf scipy_LAPACKE_zgetrf
#define LAPACKE_zgetri scipy_LAPACKE_zgetri

#ifdef __cplusplus
}
#endif

#endif
