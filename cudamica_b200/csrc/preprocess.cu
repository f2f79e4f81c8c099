// Centring and sphering on the GPU in FP64 (replaces center() and whiten(),
// src/preprocess.cu:31-420 of the reference, which use a float-accumulated
// mean, cuBLAS Dsyrk and MAGMA dsyevd / dgesv / dgetrf).
//
//   mean      FP64 column sums, per-CTA partials reduced in fixed order
//   C         X_c^T X_c / T in FP64 (register-blocked, per-CTA partials)
//   S         do_sphere 1: 2 C^{-1/2} from a parallel-ordered cyclic Jacobi
//             eigendecomposition (one CTA, round-robin disjoint rotations);
//             do_sphere 2: diag(1/std) (std with T-1, src/kernels.cu:148-161);
//             do_sphere 0: I
//   ldetS     -log|det S| = -sum log of the eigen-scales
//   x         S (x - mean) in FP64, rounded once to FP32 into the padded
//             sample-major layout the E-step reads.
#include <cmath>
#include <cstdint>

#include "common.cuh"

namespace {

constexpr int kChunk = 2048;   // samples per CTA in the reductions

__global__ void k_colsum(const float* __restrict__ x, int64_t T, int n, double* __restrict__ part) {
    const int64_t t0 = (int64_t)blockIdx.x * kChunk;
    const int64_t t1 = t0 + kChunk < T ? t0 + kChunk : T;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        double s = 0.0;
        for (int64_t t = t0; t < t1; t++) s += (double)x[t * n + i];
        part[(size_t)blockIdx.x * n + i] = s;
    }
}

__global__ void k_mean(const double* __restrict__ part, int nblk, int n, int64_t T,
                       double* __restrict__ mean) {
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        double s = 0.0;
        for (int b = 0; b < nblk; b++) s += part[(size_t)b * n + i];
        mean[i] = s / (double)T;
    }
}

// Partial covariance over one chunk: each thread owns an RB x RB block of C.
template <int RB>
__global__ void __launch_bounds__(256) k_cov(const float* __restrict__ x, int64_t T, int n,
                                             const double* __restrict__ mean,
                                             double* __restrict__ part) {
    extern __shared__ double xs[];   // [32][n]
    const int nb = (n + RB - 1) / RB;
    const int64_t t0 = (int64_t)blockIdx.x * kChunk;
    const int64_t t1 = t0 + kChunk < T ? t0 + kChunk : T;
    // every thread handles up to ceil(nb*nb / 256) blocks
    double acc[4][RB][RB];
    const int nblocks = nb * nb;
#pragma unroll
    for (int q = 0; q < 4; q++)
#pragma unroll
        for (int a = 0; a < RB; a++)
#pragma unroll
            for (int b = 0; b < RB; b++) acc[q][a][b] = 0.0;
    for (int64_t tb = t0; tb < t1; tb += 32) {
        __syncthreads();
        for (int e = threadIdx.x; e < 32 * n; e += blockDim.x) {
            const int r = e / n, i = e % n;
            const int64_t t = tb + r;
            xs[e] = (t < t1) ? (double)x[t * n + i] - mean[i] : 0.0;
        }
        __syncthreads();
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const int blk = threadIdx.x + q * blockDim.x;
            if (blk >= nblocks) break;
            const int bi = (blk % nb) * RB, bk = (blk / nb) * RB;
            for (int r = 0; r < 32; r++) {
                double xi[RB], xk[RB];
#pragma unroll
                for (int a = 0; a < RB; a++) xi[a] = (bi + a < n) ? xs[r * n + bi + a] : 0.0;
#pragma unroll
                for (int b = 0; b < RB; b++) xk[b] = (bk + b < n) ? xs[r * n + bk + b] : 0.0;
#pragma unroll
                for (int a = 0; a < RB; a++)
#pragma unroll
                    for (int b = 0; b < RB; b++) acc[q][a][b] += xi[a] * xk[b];
            }
        }
    }
#pragma unroll
    for (int q = 0; q < 4; q++) {
        const int blk = threadIdx.x + q * blockDim.x;
        if (blk >= nblocks) break;
        const int bi = (blk % nb) * RB, bk = (blk / nb) * RB;
#pragma unroll
        for (int a = 0; a < RB; a++)
#pragma unroll
            for (int b = 0; b < RB; b++)
                if (bi + a < n && bk + b < n)
                    part[(size_t)blockIdx.x * n * n + (size_t)(bk + b) * n + bi + a] = acc[q][a][b];
    }
}

__global__ void k_cov_reduce(const double* __restrict__ part, int nblk, int n, int64_t T,
                             double* __restrict__ C) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n * n) return;
    double s = 0.0;
    for (int b = 0; b < nblk; b++) s += part[(size_t)b * n * n + e];
    C[e] = s / (double)T;
}

// Parallel-ordered cyclic Jacobi: per round, n/2 disjoint (p,q) rotations from
// a round-robin schedule; J^T A J applied as column then row updates.
// a: n x n column-major (overwritten, becomes diagonal); V: eigenvectors.
__global__ void __launch_bounds__(1024) k_jacobi(double* a, double* V, int n, double* evals) {
    const int tid = threadIdx.x;
    const int ne = (n % 2) ? n + 1 : n;   // pad to even with a dummy index
    __shared__ double cs[256], sn[256];
    __shared__ int pp[256], qq[256];
    __shared__ double red[32];
    __shared__ int stop;
    for (int e = tid; e < n * n; e += blockDim.x) V[e] = ((e % n) == (e / n)) ? 1.0 : 0.0;
    __syncthreads();
    for (int sweep = 0; sweep < 40; sweep++) {
        // convergence: off-diagonal vs Frobenius
        double off = 0.0, fro = 0.0;
        for (int e = tid; e < n * n; e += blockDim.x) {
            const double v = a[e];
            fro += v * v;
            if ((e % n) != (e / n)) off += v * v;
        }
        for (int o = 16; o > 0; o >>= 1) {
            off += __shfl_xor_sync(0xffffffffu, off, o);
            fro += __shfl_xor_sync(0xffffffffu, fro, o);
        }
        if (tid % 32 == 0) { red[tid / 32] = off; }
        __syncthreads();
        if (tid == 0) {
            double s = 0.0;
            for (int w = 0; w < (int)(blockDim.x / 32); w++) s += red[w];
            red[0] = s;
        }
        __syncthreads();
        const double offt = red[0];
        __syncthreads();
        if (tid % 32 == 0) red[tid / 32] = fro;
        __syncthreads();
        if (tid == 0) {
            double s = 0.0;
            for (int w = 0; w < (int)(blockDim.x / 32); w++) s += red[w];
            stop = (offt <= 1e-30 * s);
        }
        __syncthreads();
        if (stop) break;
        for (int round = 0; round < ne - 1; round++) {
            const int half = ne / 2;
            for (int k = tid; k < half; k += blockDim.x) {
                auto pos = [&](int j) { return j == 0 ? 0 : 1 + ((j - 1 + round) % (ne - 1)); };
                int p = pos(k), q = pos(ne - 1 - k);
                if (p > q) { int t = p; p = q; q = t; }
                double c = 1.0, s = 0.0;
                if (q < n) {
                    const double apq = a[(size_t)q * n + p];
                    if (fabs(apq) >= 1e-300) {
                        const double app = a[(size_t)p * n + p], aqq = a[(size_t)q * n + q];
                        const double th = (aqq - app) / (2.0 * apq);
                        const double t = (th >= 0 ? 1.0 : -1.0) / (fabs(th) + sqrt(th * th + 1.0));
                        c = 1.0 / sqrt(t * t + 1.0);
                        s = t * c;
                    }
                }
                pp[k] = p; qq[k] = q; cs[k] = c; sn[k] = s;
            }
            __syncthreads();
            // columns p, q (and V)
            for (int e = tid; e < half * n; e += blockDim.x) {
                const int k = e / n, r = e % n;
                const int p = pp[k], q = qq[k];
                if (q >= n || sn[k] == 0.0) continue;
                const double c = cs[k], s = sn[k];
                const double arp = a[(size_t)p * n + r], arq = a[(size_t)q * n + r];
                a[(size_t)p * n + r] = c * arp - s * arq;
                a[(size_t)q * n + r] = s * arp + c * arq;
                const double vrp = V[(size_t)p * n + r], vrq = V[(size_t)q * n + r];
                V[(size_t)p * n + r] = c * vrp - s * vrq;
                V[(size_t)q * n + r] = s * vrp + c * vrq;
            }
            __syncthreads();
            // rows p, q
            for (int e = tid; e < half * n; e += blockDim.x) {
                const int k = e / n, col = e % n;
                const int p = pp[k], q = qq[k];
                if (q >= n || sn[k] == 0.0) continue;
                const double c = cs[k], s = sn[k];
                const double apc = a[(size_t)col * n + p], aqc = a[(size_t)col * n + q];
                a[(size_t)col * n + p] = c * apc - s * aqc;
                a[(size_t)col * n + q] = s * apc + c * aqc;
            }
            __syncthreads();
        }
    }
    for (int i = tid; i < n; i += blockDim.x) evals[i] = a[(size_t)i * n + i];
}

// S = V diag(2/sqrt(d)) V^T (do_sphere 1), diag(1/std) (2) or I (0); ldetS.
__global__ void k_sphere(const double* __restrict__ V, const double* __restrict__ evals,
                         const double* __restrict__ var, int n, int do_sphere,
                         double* __restrict__ S, double* __restrict__ ldetS) {
    for (int e = threadIdx.x + blockIdx.x * blockDim.x; e < n * n; e += blockDim.x * gridDim.x) {
        const int i = e % n, k = e / n;
        double v = 0.0;
        if (do_sphere == 1) {
            for (int q = 0; q < n; q++)
                v += V[(size_t)q * n + i] * (2.0 / sqrt(evals[q])) * V[(size_t)q * n + k];
        } else if (do_sphere == 2) {
            v = (i == k) ? 1.0 / sqrt(var[i]) : 0.0;
        } else {
            v = (i == k) ? 1.0 : 0.0;
        }
        S[e] = v;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        double ld = 0.0;
        for (int q = 0; q < n; q++) {
            if (do_sphere == 1) ld += log(2.0 / sqrt(evals[q]));
            else if (do_sphere == 2) ld += log(fabs(1.0 / sqrt(var[q])));
        }
        *ldetS = -ld;
    }
}

// per-channel variance about the (second) mean, divisor T-1 (do_sphere 2)
__global__ void k_var(const float* __restrict__ x, int64_t T, int n, const double* __restrict__ mean,
                      double* __restrict__ var) {
    const int i = blockIdx.x;
    __shared__ double sh[256];
    double s = 0.0;
    for (int64_t t = threadIdx.x; t < T; t += blockDim.x) s += (double)x[t * n + i] - mean[i];
    sh[threadIdx.x] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double tot = 0.0;
        for (int k = 0; k < (int)blockDim.x; k++) tot += sh[k];
        sh[0] = tot / (double)T;
    }
    __syncthreads();
    const double mu2 = sh[0];
    __syncthreads();
    double m2 = 0.0;
    for (int64_t t = threadIdx.x; t < T; t += blockDim.x) {
        const double d = fabs((double)x[t * n + i] - mean[i] - mu2);
        m2 += d * d;
    }
    sh[threadIdx.x] = m2;
    __syncthreads();
    if (threadIdx.x == 0) {
        double tot = 0.0;
        for (int k = 0; k < (int)blockDim.x; k++) tot += sh[k];
        var[i] = tot / (double)(T - 1);
    }
}

// x_out[t][i] = sum_k S(i,k) (x[t][k] - mean[k]) in FP64, rounded to FP32;
// padded channels are zero.
// Round to the TF32 grid, nearest with ties away from zero (the tensor cores
// read only the top 19 bits of an FP32 operand, i.e. truncate; storing the data
// pre-rounded makes the TF32 contraction see an unbiased value).
__device__ __forceinline__ float round_tf32(float v) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(v));
    return __uint_as_float(r);
}

__global__ void __launch_bounds__(256) k_apply_sphere(const float* __restrict__ x, int64_t T, int n,
                                                      const double* __restrict__ mean,
                                                      const double* __restrict__ S,
                                                      float* __restrict__ xo, int ldx, int tf32) {
    extern __shared__ double xc[];   // [16][n]
    const int64_t t0 = (int64_t)blockIdx.x * 16;
    for (int e = threadIdx.x; e < 16 * n; e += blockDim.x) {
        const int r = e / n, k = e % n;
        const int64_t t = t0 + r;
        xc[e] = (t < T) ? (double)x[t * n + k] - mean[k] : 0.0;
    }
    __syncthreads();
    for (int e = threadIdx.x; e < 16 * ldx; e += blockDim.x) {
        const int r = e / ldx, i = e % ldx;
        const int64_t t = t0 + r;
        if (t >= T) continue;
        double acc = 0.0;
        if (i < n)
            for (int k = 0; k < n; k++) acc += S[(size_t)k * n + i] * xc[r * n + k];
        xo[t * ldx + i] = tf32 ? round_tf32((float)acc) : (float)acc;
    }
}

__global__ void k_convert(const double* __restrict__ xs, int64_t T, int n, float* __restrict__ xo,
                          int ldx, int tf32) {
    const int64_t total = T * (int64_t)ldx;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t t = e / ldx;
        const int i = (int)(e % ldx);
        const float v = (i < n) ? (float)xs[t * n + i] : 0.f;
        xo[e] = tf32 ? round_tf32(v) : v;
    }
}

}  // namespace

namespace amica {

// evwork: >= 4 n^2 + 4 n doubles
cudaError_t launch_preprocess(const float* raw, int64_t T, int n, int do_sphere, double* means,
                              double* cov, double* sphere, double* evwork, double* ldetS_dev,
                              float* x, int ldx, int tf32, cudaStream_t st) {
    if (n > 256) return cudaErrorInvalidValue;
    const int nblk = (int)((T + kChunk - 1) / kChunk);
    double* part = nullptr;
    const size_t part_len = (size_t)nblk * n * n > (size_t)nblk * n ? (size_t)nblk * n * n : (size_t)nblk * n;
    cudaError_t e = cudaMallocAsync(&part, sizeof(double) * part_len, st);
    if (e != cudaSuccess) return e;
    k_colsum<<<nblk, 256, 0, st>>>(raw, T, n, part);
    k_mean<<<1, 256, 0, st>>>(part, nblk, n, T, means);
    double* V = evwork;
    double* ev = evwork + (size_t)n * n;
    double* var = ev + n;
    if (do_sphere == 1) {
        const int RB = 4;
        const int nb = (n + RB - 1) / RB;
        if (nb * nb > 4 * 256) { cudaFreeAsync(part, st); return cudaErrorInvalidValue; }
        const size_t smem = sizeof(double) * 32 * n;
        e = cudaFuncSetAttribute(k_cov<RB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) { cudaFreeAsync(part, st); return e; }
        k_cov<RB><<<nblk, 256, smem, st>>>(raw, T, n, means, part);
        k_cov_reduce<<<(n * n + 255) / 256, 256, 0, st>>>(part, nblk, n, T, cov);
        e = cudaMemcpyAsync(evwork + 2 * (size_t)n * n, cov, sizeof(double) * n * n,
                            cudaMemcpyDeviceToDevice, st);
        if (e != cudaSuccess) { cudaFreeAsync(part, st); return e; }
        k_jacobi<<<1, 1024, 0, st>>>(evwork + 2 * (size_t)n * n, V, n, ev);
    } else if (do_sphere == 2) {
        k_var<<<n, 256, 0, st>>>(raw, T, n, means, var);
    }
    k_sphere<<<(n * n + 255) / 256, 256, 0, st>>>(V, ev, var, n, do_sphere, sphere, ldetS_dev);
    const size_t smem2 = sizeof(double) * 16 * n;
    e = cudaFuncSetAttribute(k_apply_sphere, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem2);
    if (e != cudaSuccess) { cudaFreeAsync(part, st); return e; }
    k_apply_sphere<<<(unsigned)((T + 15) / 16), 256, smem2, st>>>(raw, T, n, means, sphere, x, ldx, tf32);
    cudaFreeAsync(part, st);
    return cudaGetLastError();
}

cudaError_t launch_convert_sphered(const double* xs, int64_t T, int n, float* x, int ldx, int tf32,
                                   cudaStream_t st) {
    k_convert<<<2048, 256, 0, st>>>(xs, T, n, x, ldx, tf32);
    return cudaGetLastError();
}

}  // namespace amica
