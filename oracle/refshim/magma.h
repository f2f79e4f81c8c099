/*
 * Minimal stand-in for the MAGMA 1.2 header that the reference sources include.
 *
 * Test infrastructure only: it lets the reference's own CUDA sources
 * (src/amica.cu, src/preprocess.cu, src/error.cu) compile and link for
 * sm_100a so that their outputs can pin the FP64 oracle.  Nothing in the
 * product includes or links this file.
 *
 * Only the five MAGMA entry points the reference calls are declared
 * (src/amica.cu:630,881; src/preprocess.cu:174,220,247; src/error.cu:90).
 * Their implementations live in refshim.cu and are written on cuSOLVER.
 */
#ifndef AMICA_REFSHIM_MAGMA_H
#define AMICA_REFSHIM_MAGMA_H

#include <cuda_runtime.h>

typedef int magma_int_t;
typedef int magma_err_t;
typedef char magma_vec_t;
typedef char magma_uplo_t;

#define MagmaVec   'V'
#define MagmaNoVec 'N'
#define MagmaUpper 'U'
#define MagmaLower 'L'
#define MAGMA_SUCCESS 0

#ifdef __cplusplus
extern "C" {
#endif

magma_err_t magma_init(void);
const char *magma_strerror(magma_err_t error);

/* LU factorisation with partial pivoting of a device matrix (column-major).
 * ipiv is a HOST array, 1-based, as in MAGMA. */
magma_int_t magma_dgetrf_gpu(magma_int_t m, magma_int_t n, double *dA,
                             magma_int_t ldda, magma_int_t *ipiv,
                             magma_int_t *info);

/* Symmetric eigendecomposition of a device matrix; eigenvalues (ascending)
 * go to the HOST array w, eigenvectors overwrite dA (columns). */
magma_int_t magma_dsyevd_gpu(magma_vec_t jobz, magma_uplo_t uplo,
                             magma_int_t n, double *dA, magma_int_t ldda,
                             double *w, double *wA, magma_int_t ldwa,
                             double *work, magma_int_t lwork,
                             magma_int_t *iwork, magma_int_t liwork,
                             magma_int_t *info);

/* Solve dA * X = dB in place (dB <- X); ipiv is a HOST array. */
magma_int_t magma_dgesv_gpu(magma_int_t n, magma_int_t nrhs, double *dA,
                            magma_int_t ldda, magma_int_t *ipiv, double *dB,
                            magma_int_t lddb, magma_int_t *info);

#ifdef __cplusplus
}
#endif

#endif
