/* Prototypes of the four LAPACKE routines the reference's hot path calls
 * (precond/FSAI/LU_main.cpp:41-43, precond/CPR.hpp:364, precond/Jacobi/Jacobi.tpp:64-65).
 * The oracle library links them from the OpenBLAS shared object shipped in the
 * image; no LAPACK source is part of this repository.  Test infrastructure only. */
#ifndef ORACLE_SHIM_LAPACKE_H
#define ORACLE_SHIM_LAPACKE_H
#define LAPACK_ROW_MAJOR 101
#define LAPACK_COL_MAJOR 102
typedef int lapack_int;
extern "C" {
lapack_int LAPACKE_dgetrf(int layout, lapack_int m, lapack_int n, double* a, lapack_int lda, lapack_int* ipiv);
lapack_int LAPACKE_dgetrs(int layout, char trans, lapack_int n, lapack_int nrhs, const double* a, lapack_int lda,
                          const lapack_int* ipiv, double* b, lapack_int ldb);
lapack_int LAPACKE_dgesv(int layout, lapack_int n, lapack_int nrhs, double* a, lapack_int lda, lapack_int* ipiv,
                         double* b, lapack_int ldb);
lapack_int LAPACKE_dgetri(int layout, lapack_int n, double* a, lapack_int lda, const lapack_int* ipiv);
}
#endif
