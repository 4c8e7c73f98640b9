/* Test-infrastructure shim: lets the reference's own RI sources compile unmodified and link
 * against the OpenBLAS copy that ships inside scipy (its exported symbols carry a `scipy_`
 * prefix).  Only the standard CBLAS prototypes the reference calls are declared here; the
 * `cblas_*` names are mapped onto the prefixed exports by macro.  Nothing in this header is
 * product code: it exists only so oracle/Makefile can build oracle/_ref/librrref.so. */
#ifndef RR_ORACLE_SHIM_CBLAS_H
#define RR_ORACLE_SHIM_CBLAS_H

#ifdef __cplusplus
extern "C" {
#endif

enum CBLAS_ORDER { CblasRowMajor = 101, CblasColMajor = 102 };
enum CBLAS_TRANSPOSE { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 };
typedef enum CBLAS_ORDER CBLAS_LAYOUT;

void scipy_cblas_dgemm(enum CBLAS_ORDER order, enum CBLAS_TRANSPOSE ta, enum CBLAS_TRANSPOSE tb, int m, int n,
                       int k, double alpha, const double* a, int lda, const double* b, int ldb, double beta,
                       double* c, int ldc);
void scipy_cblas_zgemm(enum CBLAS_ORDER order, enum CBLAS_TRANSPOSE ta, enum CBLAS_TRANSPOSE tb, int m, int n,
                       int k, const void* alpha, const void* a, int lda, const void* b, int ldb, const void* beta,
                       void* c, int ldc);
void scipy_cblas_dgemv(enum CBLAS_ORDER order, enum CBLAS_TRANSPOSE ta, int m, int n, double alpha,
                       const double* a, int lda, const double* x, int incx, double beta, double* y, int incy);
void scipy_cblas_zgemv(enum CBLAS_ORDER order, enum CBLAS_TRANSPOSE ta, int m, int n, const void* alpha,
                       const void* a, int lda, const void* x, int incx, const void* beta, void* y, int incy);
double scipy_cblas_ddot(int n, const double* x, int incx, const double* y, int incy);
void scipy_cblas_daxpy(int n, double alpha, const double* x, int incx, double* y, int incy);
void scipy_cblas_dscal(int n, double alpha, double* x, int incx);
void scipy_cblas_zaxpy(int n, const void* alpha, const void* x, int incx, void* y, int incy);
void scipy_cblas_zdotc_sub(int n, const void* x, int incx, const void* y, int incy, void* dotc);
void scipy_cblas_zscal(int n, const void* alpha, void* x, int incx);
void scipy_openblas_set_num_threads(int n);

#define cblas_dgemm scipy_cblas_dgemm
#define cblas_zgemm scipy_cblas_zgemm
#define cblas_dgemv scipy_cblas_dgemv
#define cblas_zgemv scipy_cblas_zgemv
#define cblas_ddot scipy_cblas_ddot
#define cblas_daxpy scipy_cblas_daxpy
#define cblas_dscal scipy_cblas_dscal
#define cblas_zaxpy scipy_cblas_zaxpy
#define cblas_zdotc_sub scipy_cblas_zdotc_sub
#define cblas_zscal scipy_cblas_zscal

#ifdef __cplusplus
}
#endif

#endif
