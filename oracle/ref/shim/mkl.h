/* mkl.h -- MKL names used by the reference, mapped to the scipy OpenBLAS
 * (scipy_-prefixed LP64 symbols).  Test infrastructure only. */
#ifndef GTF_REF_MKL_H
#define GTF_REF_MKL_H
#include <stddef.h>
typedef enum { CblasRowMajor = 101, CblasColMajor = 102 } CBLAS_LAYOUT;
typedef enum { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 } CBLAS_TRANSPOSE;
#define LAPACK_ROW_MAJOR 101
#define LAPACK_COL_MAJOR 102
void *mkl_malloc(size_t size, int align);
void mkl_free(void *p);
void cblas_dgemm(CBLAS_LAYOUT layout, CBLAS_TRANSPOSE ta, CBLAS_TRANSPOSE tb,
                 int m, int n, int k, double alpha, const double *a, int lda,
                 const double *b, int ldb, double beta, double *c, int ldc);
int LAPACKE_dgetrf(int layout, int m, int n, double *a, int lda, int *ipiv);
int LAPACKE_dgetri(int layout, int n, double *a, int lda, const int *ipiv);
#endif
