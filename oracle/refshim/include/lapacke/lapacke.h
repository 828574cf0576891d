// Stand-in for the four LAPACKE drivers the reference's src/Math/Matrix.cpp calls (row-major
// only): LU with partial pivoting (dgetrf), inverse from it (dgetri), a linear solve (dgesv)
// and a least-squares solve of a full-rank overdetermined system by Householder QR (dgels).
// Textbook algorithms (Golub & Van Loan), written here: their rounding differs from a tuned
// LAPACK's in the last bits.  Test infrastructure only.
#ifndef CAFFE_REFSHIM_LAPACKE_H
#define CAFFE_REFSHIM_LAPACKE_H

typedef int lapack_int;
#define LAPACK_ROW_MAJOR 101
#define LAPACK_COL_MAJOR 102

#ifdef __cplusplus
extern "C" {
#endif

lapack_int LAPACKE_dgetrf(int layout, lapack_int m, lapack_int n, double* a, lapack_int lda, lapack_int* ipiv);
lapack_int LAPACKE_dgetri(int layout, lapack_int n, double* a, lapack_int lda, const lapack_int* ipiv);
lapack_int LAPACKE_dgesv(int layout, lapack_int n, lapack_int nrhs, double* a, lapack_int lda, lapack_int* ipiv, double* b,
                         lapack_int ldb);
lapack_int LAPACKE_dgels(int layout, char trans, lapack_int m, lapack_int n, lapack_int nrhs, double* a, lapack_int lda,
                         double* b, lapack_int ldb);

#ifdef __cplusplus
}
#endif

#endif
