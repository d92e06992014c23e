/* Serial stand-in for lapacke.h: dgesv only, by partial-pivot LU (TEST INFRASTRUCTURE). */
#ifndef MP_SHIM_LAPACKE_H
#define MP_SHIM_LAPACKE_H
typedef int lapack_int;
#define LAPACK_ROW_MAJOR 101
#define LAPACK_COL_MAJOR 102
lapack_int LAPACKE_dgesv(int layout, lapack_int n, lapack_int nrhs, double* a, lapack_int lda,
                         lapack_int* ipiv, double* b, lapack_int ldb);
#endif
