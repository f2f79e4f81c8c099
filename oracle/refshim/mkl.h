/*
 * Minimal stand-in for the Intel MKL header that the reference sources include.
 *
 * Test infrastructure only (see magma.h in this folder).  Declares the two MKL
 * routines the reference calls in pinv() (src/amica.cu:41,81,107); their
 * implementations live in refshim.cu.
 */
#ifndef AMICA_REFSHIM_MKL_H
#define AMICA_REFSHIM_MKL_H

#define LAPACK_ROW_MAJOR 101
#define LAPACK_COL_MAJOR 102
#define LAPACK_WORK_MEMORY_ERROR -1010
#define LAPACK_TRANSPOSE_MEMORY_ERROR -1011

typedef enum { CblasRowMajor = 101, CblasColMajor = 102 } CBLAS_LAYOUT;
typedef enum { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 } CBLAS_TRANSPOSE;

#ifdef __cplusplus
extern "C" {
#endif

int LAPACKE_dgesvd(int matrix_layout, char jobu, char jobvt, int m, int n,
                   double *a, int lda, double *s, double *u, int ldu,
                   double *vt, int ldvt, double *superb);

void cblas_dgemm(CBLAS_LAYOUT layout, CBLAS_TRANSPOSE transa,
                 CBLAS_TRANSPOSE transb, int m, int n, int k, double alpha,
                 const double *a, int lda, const double *b, int ldb,
                 double beta, double *c, int ldc);

#ifdef __cplusplus
}
#endif

#endif
