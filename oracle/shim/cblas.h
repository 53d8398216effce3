/* Test infrastructure (oracle build only): the CBLAS declarations that
 * GPRat's CPU BLAS adapter calls, bound to the scipy-bundled OpenBLAS
 * (LP64, symbols carry a "scipy_" prefix).  Enum values follow the CBLAS
 * standard, which the reference's adapter relies on. */
#ifndef GPRAT_ORACLE_SHIM_CBLAS_H
#define GPRAT_ORACLE_SHIM_CBLAS_H
#ifdef __cplusplus
extern "C" {
#endif

typedef enum CBLAS_ORDER { CblasRowMajor = 101, CblasColMajor = 102 } CBLAS_ORDER;
typedef enum CBLAS_TRANSPOSE { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 } CBLAS_TRANSPOSE;
typedef enum CBLAS_UPLO { CblasUpper = 121, CblasLower = 122 } CBLAS_UPLO;
typedef enum CBLAS_DIAG { CblasNonUnit = 131, CblasUnit = 132 } CBLAS_DIAG;
typedef enum CBLAS_SIDE { CblasLeft = 141, CblasRight = 142 } CBLAS_SIDE;

void scipy_cblas_dgemm(CBLAS_ORDER, CBLAS_TRANSPOSE, CBLAS_TRANSPOSE, int, int, int, double, const double *, int,
                       const double *, int, double, double *, int);
void scipy_cblas_dtrsm(CBLAS_ORDER, CBLAS_SIDE, CBLAS_UPLO, CBLAS_TRANSPOSE, CBLAS_DIAG, int, int, double,
                       const double *, int, double *, int);
void scipy_cblas_dsyrk(CBLAS_ORDER, CBLAS_UPLO, CBLAS_TRANSPOSE, int, int, double, const double *, int, double,
                       double *, int);
void scipy_cblas_dtrsv(CBLAS_ORDER, CBLAS_UPLO, CBLAS_TRANSPOSE, CBLAS_DIAG, int, const double *, int, double *,
                       int);
void scipy_cblas_dgemv(CBLAS_ORDER, CBLAS_TRANSPOSE, int, int, double, const double *, int, const double *, int,
                       double, double *, int);
double scipy_cblas_ddot(int, const double *, int, const double *, int);
void scipy_cblas_daxpy(int, double, const double *, int, double *, int);
void scipy_openblas_set_num_threads(int);

#define cblas_dgemm scipy_cblas_dgemm
#define cblas_dtrsm scipy_cblas_dtrsm
#define cblas_dsyrk scipy_cblas_dsyrk
#define cblas_dtrsv scipy_cblas_dtrsv
#define cblas_dgemv scipy_cblas_dgemv
#define cblas_ddot scipy_cblas_ddot
#define cblas_daxpy scipy_cblas_daxpy

#ifdef __cplusplus
}
#endif
#endif
