/*
 * Implementations of the seven MAGMA / MKL symbols the reference links against
 * (magma_init, magma_strerror, magma_dgetrf_gpu, magma_dsyevd_gpu,
 * magma_dgesv_gpu, LAPACKE_dgesvd, cblas_dgemm), written on cuSOLVER and plain
 * host loops.
 *
 * Test infrastructure only.  This file is linked with the reference's own
 * sources (compiled in place from the reference tree by oracle/Makefile) to
 * produce oracle/_ref/cudaamica_ref, whose outputs pin the FP64 oracle.  The
 * product never links it.
 *
 * Semantics follow the MAGMA 1.2 / LAPACK conventions the reference relies on:
 * column-major matrices, 1-based pivots returned in HOST arrays, eigenvalues
 * in ascending order with eigenvectors overwriting the input, and every call
 * synchronous on return.
 */
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cuda_runtime.h>
#include <cusolverDn.h>
#include "magma.h"
#include "mkl.h"

static cusolverDnHandle_t g_solver = nullptr;

static void shim_fail(const char *what, int code) {
    fprintf(stderr, "refshim: %s failed (%d)\n", what, code);
    exit(1);
}
#define SHIM_CUDA(x) do { cudaError_t e_ = (x); if (e_ != cudaSuccess) shim_fail(#x, (int)e_); } while (0)
#define SHIM_SOLVER(x) do { cusolverStatus_t s_ = (x); if (s_ != CUSOLVER_STATUS_SUCCESS) shim_fail(#x, (int)s_); } while (0)

static cusolverDnHandle_t solver() {
    if (!g_solver) SHIM_SOLVER(cusolverDnCreate(&g_solver));
    return g_solver;
}

extern "C" magma_err_t magma_init(void) {
    solver();
    return MAGMA_SUCCESS;
}

extern "C" const char *magma_strerror(magma_err_t error) {
    return error == 0 ? "MAGMA_SUCCESS" : "refshim: MAGMA-equivalent call failed";
}

extern "C" magma_int_t magma_dgetrf_gpu(magma_int_t m, magma_int_t n, double *dA,
                                        magma_int_t ldda, magma_int_t *ipiv,
                                        magma_int_t *info) {
    SHIM_CUDA(cudaDeviceSynchronize());
    int lwork = 0;
    SHIM_SOLVER(cusolverDnDgetrf_bufferSize(solver(), m, n, dA, ldda, &lwork));
    double *work = nullptr;
    int *dipiv = nullptr, *dinfo = nullptr;
    SHIM_CUDA(cudaMalloc(&work, sizeof(double) * (lwork > 0 ? lwork : 1)));
    SHIM_CUDA(cudaMalloc(&dipiv, sizeof(int) * (m < n ? m : n)));
    SHIM_CUDA(cudaMalloc(&dinfo, sizeof(int)));
    SHIM_SOLVER(cusolverDnDgetrf(solver(), m, n, dA, ldda, work, dipiv, dinfo));
    SHIM_CUDA(cudaDeviceSynchronize());
    SHIM_CUDA(cudaMemcpy(ipiv, dipiv, sizeof(int) * (m < n ? m : n), cudaMemcpyDeviceToHost));
    SHIM_CUDA(cudaMemcpy(info, dinfo, sizeof(int), cudaMemcpyDeviceToHost));
    cudaFree(work); cudaFree(dipiv); cudaFree(dinfo);
    return MAGMA_SUCCESS;
}

extern "C" magma_int_t magma_dsyevd_gpu(magma_vec_t jobz, magma_uplo_t uplo,
                                        magma_int_t n, double *dA, magma_int_t ldda,
                                        double *w, double *, magma_int_t,
                                        double *, magma_int_t, magma_int_t *,
                                        magma_int_t, magma_int_t *info) {
    SHIM_CUDA(cudaDeviceSynchronize());
    cusolverEigMode_t mode = (jobz == MagmaVec) ? CUSOLVER_EIG_MODE_VECTOR : CUSOLVER_EIG_MODE_NOVECTOR;
    cublasFillMode_t fill = (uplo == MagmaUpper) ? CUBLAS_FILL_MODE_UPPER : CUBLAS_FILL_MODE_LOWER;
    double *dw = nullptr, *work = nullptr;
    int *dinfo = nullptr, lwork = 0;
    SHIM_CUDA(cudaMalloc(&dw, sizeof(double) * n));
    SHIM_SOLVER(cusolverDnDsyevd_bufferSize(solver(), mode, fill, n, dA, ldda, dw, &lwork));
    SHIM_CUDA(cudaMalloc(&work, sizeof(double) * (lwork > 0 ? lwork : 1)));
    SHIM_CUDA(cudaMalloc(&dinfo, sizeof(int)));
    SHIM_SOLVER(cusolverDnDsyevd(solver(), mode, fill, n, dA, ldda, dw, work, lwork, dinfo));
    SHIM_CUDA(cudaDeviceSynchronize());
    SHIM_CUDA(cudaMemcpy(w, dw, sizeof(double) * n, cudaMemcpyDeviceToHost));
    SHIM_CUDA(cudaMemcpy(info, dinfo, sizeof(int), cudaMemcpyDeviceToHost));
    cudaFree(dw); cudaFree(work); cudaFree(dinfo);
    return MAGMA_SUCCESS;
}

extern "C" magma_int_t magma_dgesv_gpu(magma_int_t n, magma_int_t nrhs, double *dA,
                                       magma_int_t ldda, magma_int_t *ipiv, double *dB,
                                       magma_int_t lddb, magma_int_t *info) {
    SHIM_CUDA(cudaDeviceSynchronize());
    int lwork = 0;
    SHIM_SOLVER(cusolverDnDgetrf_bufferSize(solver(), n, n, dA, ldda, &lwork));
    double *work = nullptr;
    int *dipiv = nullptr, *dinfo = nullptr;
    SHIM_CUDA(cudaMalloc(&work, sizeof(double) * (lwork > 0 ? lwork : 1)));
    SHIM_CUDA(cudaMalloc(&dipiv, sizeof(int) * n));
    SHIM_CUDA(cudaMalloc(&dinfo, sizeof(int)));
    SHIM_SOLVER(cusolverDnDgetrf(solver(), n, n, dA, ldda, work, dipiv, dinfo));
    SHIM_SOLVER(cusolverDnDgetrs(solver(), CUBLAS_OP_N, n, nrhs, dA, ldda, dipiv, dB, lddb, dinfo));
    SHIM_CUDA(cudaDeviceSynchronize());
    SHIM_CUDA(cudaMemcpy(ipiv, dipiv, sizeof(int) * n, cudaMemcpyDeviceToHost));
    SHIM_CUDA(cudaMemcpy(info, dinfo, sizeof(int), cudaMemcpyDeviceToHost));
    cudaFree(work); cudaFree(dipiv); cudaFree(dinfo);
    return MAGMA_SUCCESS;
}

/* Full SVD of a host column-major m x n matrix (m >= n), through cuSOLVER. */
extern "C" int LAPACKE_dgesvd(int layout, char jobu, char jobvt, int m, int n,
                              double *a, int lda, double *s, double *u, int ldu,
                              double *vt, int ldvt, double *superb) {
    if (layout != LAPACK_COL_MAJOR || m < n) return -1;
    SHIM_CUDA(cudaDeviceSynchronize());
    double *da, *ds, *du, *dvt, *work, *rwork;
    int *dinfo, lwork = 0, info = 0;
    SHIM_CUDA(cudaMalloc(&da, sizeof(double) * (size_t)lda * n));
    SHIM_CUDA(cudaMalloc(&ds, sizeof(double) * n));
    SHIM_CUDA(cudaMalloc(&du, sizeof(double) * (size_t)ldu * m));
    SHIM_CUDA(cudaMalloc(&dvt, sizeof(double) * (size_t)ldvt * n));
    SHIM_CUDA(cudaMalloc(&rwork, sizeof(double) * n));
    SHIM_CUDA(cudaMalloc(&dinfo, sizeof(int)));
    SHIM_CUDA(cudaMemcpy(da, a, sizeof(double) * (size_t)lda * n, cudaMemcpyHostToDevice));
    SHIM_SOLVER(cusolverDnDgesvd_bufferSize(solver(), m, n, &lwork));
    SHIM_CUDA(cudaMalloc(&work, sizeof(double) * (lwork > 0 ? lwork : 1)));
    SHIM_SOLVER(cusolverDnDgesvd(solver(), jobu, jobvt, m, n, da, lda, ds, du, ldu,
                                 dvt, ldvt, work, lwork, rwork, dinfo));
    SHIM_CUDA(cudaDeviceSynchronize());
    SHIM_CUDA(cudaMemcpy(s, ds, sizeof(double) * n, cudaMemcpyDeviceToHost));
    SHIM_CUDA(cudaMemcpy(u, du, sizeof(double) * (size_t)ldu * m, cudaMemcpyDeviceToHost));
    SHIM_CUDA(cudaMemcpy(vt, dvt, sizeof(double) * (size_t)ldvt * n, cudaMemcpyDeviceToHost));
    SHIM_CUDA(cudaMemcpy(&info, dinfo, sizeof(int), cudaMemcpyDeviceToHost));
    if (superb) memset(superb, 0, sizeof(double) * (n > 1 ? n - 1 : 1));
    cudaFree(da); cudaFree(ds); cudaFree(du); cudaFree(dvt); cudaFree(work);
    cudaFree(rwork); cudaFree(dinfo);
    return info;
}

/* C = alpha * op(A) * op(B) + beta * C, column-major, host memory. */
extern "C" void cblas_dgemm(CBLAS_LAYOUT layout, CBLAS_TRANSPOSE ta, CBLAS_TRANSPOSE tb,
                            int m, int n, int k, double alpha, const double *a, int lda,
                            const double *b, int ldb, double beta, double *c, int ldc) {
    if (layout != CblasColMajor) shim_fail("cblas_dgemm row-major", 0);
    for (int j = 0; j < n; j++) {
        for (int i = 0; i < m; i++) {
            double acc = 0.0;
            for (int p = 0; p < k; p++) {
                double av = (ta == CblasNoTrans) ? a[i + (size_t)p * lda] : a[p + (size_t)i * lda];
                double bv = (tb == CblasNoTrans) ? b[p + (size_t)j * ldb] : b[j + (size_t)p * ldb];
                acc += av * bv;
            }
            double prev = (beta == 0.0) ? 0.0 : beta * c[i + (size_t)j * ldc];
            c[i + (size_t)j * ldc] = alpha * acc + prev;
        }
    }
}
