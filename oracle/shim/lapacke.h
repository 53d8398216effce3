/* Test infrastructure (oracle build only): LAPACKE_dpotrf2 bound to the
 * scipy-bundled OpenBLAS (symbol prefix "scipy_"). */
#ifndef GPRAT_ORACLE_SHIM_LAPACKE_H
#define GPRAT_ORACLE_SHIM_LAPACKE_H
#ifdef __cplusplus
extern "C" {
#endif
#define LAPACK_ROW_MAJOR 101
#define LAPACK_COL_MAJOR 102
int scipy_LAPACKE_dpotrf2(int matrix_layout, char uplo, int n, double *a, int lda);
#define LAPACKE_dpotrf2 scipy_LAPACKE_dpotrf2
#ifdef __cplusplus
}
#endif
#endif
