// Centring and sphering on the GPU in FP64 (replaces center() and whiten(),
// src/preprocess.cu:31-420 of the reference, which use a float-accumulated
// mean, cuBLAS Dsyrk and MAGMA dsyevd / dgesv / dgetrf).
//
//   mean      FP64 column sums, per-CTA partials reduced in fixed order
//   C         X_c^T X_c / T in FP64 (8 x 8 register blocks, one CTA per SM)
//   S         do_sphere 1: 2 C^{-1/2} from a parallel-ordered cyclic Jacobi
//             eigendecomposition (one CTA, round-robin disjoint rotations,
//             matrix and eigenvectors in shared memory);
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

// mean = (sum of the per-CTA partial sums) / div; div = 1 gives the sums
__global__ void k_mean(const double* __restrict__ part, int nblk, int n, double div,
                       double* __restrict__ mean) {
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        double s = 0.0;
        for (int b = 0; b < nblk; b++) s += part[(size_t)b * n + i];
        mean[i] = s / div;
    }
}

__global__ void k_cov_reduce(const double* __restrict__ part, int nblk, int n, double div,
                             double* __restrict__ C) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n * n) return;
    double s = 0.0;
    for (int b = 0; b < nblk; b++) s += part[(size_t)b * n * n + e];
    C[e] = s / div;
}

// The sharded form's inputs to k_sphere: the covariance (scatter / T) and, for
// do_sphere 2, the per-channel variance (scatter diagonal / (T - 1)) of all
// shards.
__global__ void k_scale_scatter(const double* __restrict__ scatter, int n, double T,
                                double* __restrict__ C, double* __restrict__ var) {
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n * n; e += blockDim.x * gridDim.x) {
        C[e] = scatter[e] / T;
        if (e % (n + 1) == 0) var[e / (n + 1)] = scatter[e] / (T - 1.0);
    }
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

// Partial covariance: one persistent CTA per SM over a contiguous sample range;
// thread (bi, bk) owns the 8 x 8 block C[8 bi .. 8 bi + 7][8 bk .. 8 bk + 7] in
// registers (n <= 128: 16 x 16 blocks, 256 threads).  Samples are staged 32 at
// a time, centred, in shared memory.
constexpr int kCovRows = 32;
__global__ void __launch_bounds__(256, 1) k_cov8(const float* __restrict__ x, int64_t T, int n,
                                                 int64_t chunk, const double* __restrict__ mean,
                                                 double* __restrict__ part) {
    __shared__ __align__(16) double xs[kCovRows][128];
    const int bi = threadIdx.x & 15, bk = threadIdx.x >> 4;
    const int64_t t0 = (int64_t)blockIdx.x * chunk;
    const int64_t t1 = t0 + chunk < T ? t0 + chunk : T;
    double acc[8][8];
#pragma unroll
    for (int a = 0; a < 8; a++)
#pragma unroll
        for (int b = 0; b < 8; b++) acc[a][b] = 0.0;
    for (int64_t tb = t0; tb < t1; tb += kCovRows) {
        __syncthreads();
        for (int e = threadIdx.x; e < kCovRows * 128; e += 256) {
            const int r = e >> 7, i = e & 127;
            const int64_t t = tb + r;
            xs[r][i] = (t < t1 && i < n) ? (double)x[t * n + i] - mean[i] : 0.0;
        }
        __syncthreads();
#pragma unroll 2
        for (int r = 0; r < kCovRows; r++) {
            double xi[8], xk[8];
#pragma unroll
            for (int a = 0; a < 8; a += 2) {
                const double2 u = *reinterpret_cast<const double2*>(&xs[r][8 * bi + a]);
                const double2 w = *reinterpret_cast<const double2*>(&xs[r][8 * bk + a]);
                xi[a] = u.x; xi[a + 1] = u.y; xk[a] = w.x; xk[a + 1] = w.y;
            }
#pragma unroll
            for (int a = 0; a < 8; a++)
#pragma unroll
                for (int b = 0; b < 8; b++) acc[a][b] = fma(xi[a], xk[b], acc[a][b]);
        }
    }
#pragma unroll
    for (int a = 0; a < 8; a++)
#pragma unroll
        for (int b = 0; b < 8; b++) {
            const int i = 8 * bi + a, k = 8 * bk + b;
            if (i < n && k < n) part[(size_t)blockIdx.x * n * n + (size_t)k * n + i] = acc[a][b];
        }
}

// Parallel-ordered cyclic Jacobi eigendecomposition of the symmetric n x n
// matrix C (n <= 128), one CTA, everything in shared memory: the upper
// triangle of the working matrix packed by columns and the eigenvector matrix
// V.  A round applies n/2 disjoint rotations (p_k, q_k) of the round-robin
// schedule at once.  Since J^T A J only mixes rows {p_K, q_K} with columns
// {p_L, q_L}, each 2 x 2 block (K, L), K <= L, is transformed independently by
// the thread that owns it; V <- V J rotates column pairs.  Sweeps stop when the
// off-diagonal energy is below 1e-30 of the total.
__device__ __forceinline__ int pk_idx(int i, int j) {   // i <= j
    return (j * (j + 1)) / 2 + i;
}
__device__ __forceinline__ int pk_sym(int i, int j) { return i <= j ? pk_idx(i, j) : pk_idx(j, i); }

constexpr int kJacThreads = 1024;
__global__ void __launch_bounds__(kJacThreads, 1) k_jacobi_smem(const double* __restrict__ C,
                                                                double* __restrict__ Vout,
                                                                double* __restrict__ evals, int n) {
    extern __shared__ __align__(16) double jsm[];
    const int np = (n * (n + 1)) / 2;
    double* ap = jsm;                                   // packed upper triangle
    double* V = jsm + ((np + 1) & ~1);                  // n x n, column-major
    __shared__ double cs[64], sn[64];
    __shared__ int pp[64], qq[64];
    __shared__ unsigned short blkKL[64 * 65 / 2];   // (K << 8) | L for the 2 x 2 blocks, K <= L
    __shared__ double red[32];
    __shared__ int stop;
    const int tid = threadIdx.x;
    const int ne = n + (n & 1), half = ne / 2;
    const int nblk = half * (half + 1) / 2;
    for (int e = tid; e < n * n; e += kJacThreads) {
        const int r = e % n, c = e / n;
        if (r <= c) ap[pk_idx(r, c)] = C[e];
        V[e] = (r == c) ? 1.0 : 0.0;
    }
    if (tid < half)
        for (int K = 0; K <= tid; K++) blkKL[tid * (tid + 1) / 2 + K] = (unsigned short)((K << 8) | tid);
    __syncthreads();
    for (int sweep = 0; sweep < 40; sweep++) {
        double off = 0.0, tot = 0.0;
        for (int e = tid; e < np; e += kJacThreads) {
            // column j of the packed triangle holds rows 0..j; the last one is diagonal
            int j = (int)((sqrt(8.0 * e + 1.0) - 1.0) * 0.5);
            while (pk_idx(0, j + 1) <= e) j++;
            while (pk_idx(0, j) > e) j--;
            const double v = ap[e];
            const bool diag = (e - pk_idx(0, j)) == j;
            tot += diag ? v * v : 2.0 * v * v;
            off += diag ? 0.0 : 2.0 * v * v;
        }
        for (int o = 16; o > 0; o >>= 1) {
            off += __shfl_xor_sync(0xffffffffu, off, o);
            tot += __shfl_xor_sync(0xffffffffu, tot, o);
        }
        if ((tid & 31) == 0) red[tid >> 5] = off;
        __syncthreads();
        if (tid == 0) {
            double s = 0.0;
            for (int w = 0; w < kJacThreads / 32; w++) s += red[w];
            red[0] = s;
        }
        __syncthreads();
        const double offt = red[0];
        __syncthreads();
        if ((tid & 31) == 0) red[tid >> 5] = tot;
        __syncthreads();
        if (tid == 0) {
            double s = 0.0;
            for (int w = 0; w < kJacThreads / 32; w++) s += red[w];
            stop = (offt <= 1e-30 * s);
        }
        __syncthreads();
        if (stop) break;
        for (int round = 0; round < ne - 1; round++) {
            if (tid < half) {
                auto pos = [&](int j) { return j == 0 ? 0 : 1 + ((j - 1 + round) % (ne - 1)); };
                int p = pos(tid), q = pos(ne - 1 - tid);
                if (p > q) { const int t = p; p = q; q = t; }
                double c = 1.0, s = 0.0;
                if (q < n) {
                    const double apq = ap[pk_idx(p, q)];
                    if (fabs(apq) >= 1e-300) {
                        const double app = ap[pk_idx(p, p)], aqq = ap[pk_idx(q, q)];
                        const double th = (aqq - app) / (2.0 * apq);
                        const double t = (th >= 0 ? 1.0 : -1.0) / (fabs(th) + sqrt(th * th + 1.0));
                        c = 1.0 / sqrt(t * t + 1.0);
                        s = t * c;
                    }
                }
                pp[tid] = p; qq[tid] = q; cs[tid] = c; sn[tid] = s;
            }
            __syncthreads();
            // A <- J^T A J, one 2 x 2 block (K <= L) per work item
            for (int e = tid; e < nblk; e += kJacThreads) {
                const int K = blkKL[e] >> 8, L = blkKL[e] & 0xff;
                const int pK = pp[K], qK = qq[K], pL = pp[L], qL = qq[L];
                const double cK = cs[K], sK = sn[K], cL = cs[L], sL = sn[L];
                if (K == L) {
                    if (qK < n && sK != 0.0) {
                        const double app = ap[pk_idx(pK, pK)], aqq = ap[pk_idx(qK, qK)];
                        const double apq = ap[pk_idx(pK, qK)];
                        ap[pk_idx(pK, pK)] = cK * cK * app - 2.0 * cK * sK * apq + sK * sK * aqq;
                        ap[pk_idx(qK, qK)] = sK * sK * app + 2.0 * cK * sK * apq + cK * cK * aqq;
                        ap[pk_idx(pK, qK)] = 0.0;
                    }
                    continue;
                }
                if (sK == 0.0 && sL == 0.0) continue;
                const bool hq = qK < n, hqL = qL < n;
                const double b11 = ap[pk_sym(pK, pL)];
                const double b12 = hqL ? ap[pk_sym(pK, qL)] : 0.0;
                const double b21 = hq ? ap[pk_sym(qK, pL)] : 0.0;
                const double b22 = (hq && hqL) ? ap[pk_sym(qK, qL)] : 0.0;
                // B J_L (columns), then J_K^T (rows); J = [[c, s], [-s, c]]
                const double d11 = cL * b11 - sL * b12, d12 = sL * b11 + cL * b12;
                const double d21 = cL * b21 - sL * b22, d22 = sL * b21 + cL * b22;
                ap[pk_sym(pK, pL)] = cK * d11 - sK * d21;
                if (hqL) ap[pk_sym(pK, qL)] = cK * d12 - sK * d22;
                if (hq) ap[pk_sym(qK, pL)] = sK * d11 + cK * d21;
                if (hq && hqL) ap[pk_sym(qK, qL)] = sK * d12 + cK * d22;
            }
            // V <- V J: 16 threads per rotation, rows r = lane16, lane16 + 16, ...
            for (int k = tid >> 4; k < half; k += kJacThreads / 16) {
                const int p = pp[k], q = qq[k];
                const double s = sn[k];
                if (q >= n || s == 0.0) continue;
                const double c = cs[k];
                for (int r = tid & 15; r < n; r += 16) {
                    const double vp = V[(size_t)p * n + r], vq = V[(size_t)q * n + r];
                    V[(size_t)p * n + r] = c * vp - s * vq;
                    V[(size_t)q * n + r] = s * vp + c * vq;
                }
            }
            __syncthreads();
        }
    }
    for (int e = tid; e < n * n; e += kJacThreads) Vout[e] = V[e];
    for (int i = tid; i < n; i += kJacThreads) evals[i] = ap[pk_idx(i, i)];
}

// ---------------------------------------------------------------------------
// 128 < n <= 256.  The n <= 128 kernels keep the whole problem in one SM; here
// the covariance runs k_cov8's register blocking on the four 128 x 128
// quadrants, the eigendecomposition spreads the same Jacobi rounds over a
// cooperative grid, and the sphering keeps a 64-row slice of S per CTA.

// k_cov8 for the quadrant (oi, ok) of C (rows oi .., columns ok ..): blockIdx.y
// selects the quadrant; both 128-channel sample slices are staged.
__global__ void __launch_bounds__(256, 1) k_cov8q(const float* __restrict__ x, int64_t T, int n,
                                                  int64_t chunk, const double* __restrict__ mean,
                                                  double* __restrict__ part) {
    extern __shared__ __align__(16) double cq[];
    double (*xi_s)[128] = reinterpret_cast<double (*)[128]>(cq);
    double (*xk_s)[128] = reinterpret_cast<double (*)[128]>(cq + kCovRows * 128);
    const int oi = 128 * (blockIdx.y & 1), ok = 128 * (blockIdx.y >> 1);
    const int bi = threadIdx.x & 15, bk = threadIdx.x >> 4;
    const int64_t t0 = (int64_t)blockIdx.x * chunk;
    const int64_t t1 = t0 + chunk < T ? t0 + chunk : T;
    double acc[8][8];
#pragma unroll
    for (int a = 0; a < 8; a++)
#pragma unroll
        for (int b = 0; b < 8; b++) acc[a][b] = 0.0;
    for (int64_t tb = t0; tb < t1; tb += kCovRows) {
        __syncthreads();
        for (int e = threadIdx.x; e < kCovRows * 128; e += 256) {
            const int r = e >> 7, i = e & 127;
            const int64_t t = tb + r;
            const bool in = t < t1;
            xi_s[r][i] = (in && oi + i < n) ? (double)x[t * n + oi + i] - mean[oi + i] : 0.0;
            xk_s[r][i] = (in && ok + i < n) ? (double)x[t * n + ok + i] - mean[ok + i] : 0.0;
        }
        __syncthreads();
#pragma unroll 2
        for (int r = 0; r < kCovRows; r++) {
            double xi[8], xk[8];
#pragma unroll
            for (int a = 0; a < 8; a += 2) {
                const double2 u = *reinterpret_cast<const double2*>(&xi_s[r][8 * bi + a]);
                const double2 w = *reinterpret_cast<const double2*>(&xk_s[r][8 * bk + a]);
                xi[a] = u.x; xi[a + 1] = u.y; xk[a] = w.x; xk[a + 1] = w.y;
            }
#pragma unroll
            for (int a = 0; a < 8; a++)
#pragma unroll
                for (int b = 0; b < 8; b++) acc[a][b] = fma(xi[a], xk[b], acc[a][b]);
        }
    }
#pragma unroll
    for (int a = 0; a < 8; a++)
#pragma unroll
        for (int b = 0; b < 8; b++) {
            const int i = oi + 8 * bi + a, k = ok + 8 * bk + b;
            if (i < n && k < n) part[(size_t)blockIdx.x * n * n + (size_t)k * n + i] = acc[a][b];
        }
}

// Grid-wide barrier for a cooperative launch: a monotonic arrival counter;
// barrier number b completes when it reaches (b + 1) * gridDim.x.  The wait is
// bounded (~1 s); on expiry it records kErrWaitTimeout and sets *abort, after
// which every block leaves its loops at the next barrier.
// (skip_arrival: the test hook of amica_test_arm_wait_fault, a block that does
// not arrive, so that the others' waits run out.)
__device__ __forceinline__ bool grid_barrier(unsigned* count, unsigned target, volatile int* abort,
                                             int* err, long long wait_cycles, bool skip_arrival = false) {
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        if (!skip_arrival) atomicAdd(count, 1u);
        const long long t0 = clock64();
        while (true) {
            const unsigned v = *(volatile unsigned*)count;
            if (v >= target || *abort) break;
            if (clock64() - t0 > wait_cycles) {
                *abort = 1;
                atomicOr(err, amica::kErrWaitTimeout);
                break;
            }
        }
        __threadfence();
    }
    __syncthreads();
    return *abort == 0;
}

// The Jacobi eigendecomposition of k_jacobi_smem (same round-robin schedule,
// rotation formula, 2 x 2 block transforms, eigenvector update and stopping
// rule) with the packed triangle and V in global memory, rounds spread over all
// blocks of a cooperative launch: every block forms the round's n/2 rotations
// from the packed triangle, a grid barrier, the blocks share out the 2 x 2 block
// and V updates, and a second grid barrier ends the round.  Loads of shared
// state bypass L1.
struct JacGlobal {
    double* ap;        // packed upper triangle, n (n + 1) / 2
    double* part;      // per-block partial sums of the stopping test, 2 per block
    unsigned* count;   // barrier counter (zero at launch)
    int* abort;        // zero at launch
    long long wait_cycles;   // bound of every barrier wait (~1 s)
    int skip_block;          // test hook: this block skips its first arrival (-1: none)
};
__global__ void __launch_bounds__(kJacThreads, 1) k_jacobi_grid(const double* __restrict__ C,
                                                                double* __restrict__ V,
                                                                double* __restrict__ evals, int n,
                                                                JacGlobal g, int* err) {
    __shared__ double cs[128], sn[128];
    __shared__ int pp[128], qq[128];
    __shared__ double red[32];
    const int tid = threadIdx.x;
    const int gtid = blockIdx.x * kJacThreads + tid, gthreads = gridDim.x * kJacThreads;
    const int np = (n * (n + 1)) / 2;
    const int ne = n + (n & 1), half = ne / 2;
    const int nblk = half * (half + 1) / 2;
    double* ap = g.ap;
    unsigned bar = 0;
    for (int e = gtid; e < n * n; e += gthreads) {
        const int r = e % n, c = e / n;
        if (r <= c) ap[pk_idx(r, c)] = C[e];
        V[e] = (r == c) ? 1.0 : 0.0;
    }
    if (!grid_barrier(g.count, (++bar) * gridDim.x, g.abort, err, g.wait_cycles,
                      (int)blockIdx.x == g.skip_block)) return;
    for (int sweep = 0; sweep < 40; sweep++) {
        double off = 0.0, tot = 0.0;
        for (int e = gtid; e < np; e += gthreads) {
            int j = (int)((sqrt(8.0 * e + 1.0) - 1.0) * 0.5);
            while (pk_idx(0, j + 1) <= e) j++;
            while (pk_idx(0, j) > e) j--;
            const double v = __ldcg(ap + e);
            const bool diag = (e - pk_idx(0, j)) == j;
            tot += diag ? v * v : 2.0 * v * v;
            off += diag ? 0.0 : 2.0 * v * v;
        }
        for (int o = 16; o > 0; o >>= 1) {
            off += __shfl_xor_sync(0xffffffffu, off, o);
            tot += __shfl_xor_sync(0xffffffffu, tot, o);
        }
        if ((tid & 31) == 0) red[tid >> 5] = off;
        __syncthreads();
        if (tid == 0) {
            double s = 0.0;
            for (int w = 0; w < kJacThreads / 32; w++) s += red[w];
            g.part[2 * blockIdx.x] = s;
        }
        __syncthreads();
        if ((tid & 31) == 0) red[tid >> 5] = tot;
        __syncthreads();
        if (tid == 0) {
            double s = 0.0;
            for (int w = 0; w < kJacThreads / 32; w++) s += red[w];
            g.part[2 * blockIdx.x + 1] = s;
        }
        if (!grid_barrier(g.count, (++bar) * gridDim.x, g.abort, err, g.wait_cycles)) return;
        // every block sums the partials in the same order and takes the same decision
        double offt = 0.0, tott = 0.0;
        for (int b = 0; b < (int)gridDim.x; b++) {
            offt += __ldcg(g.part + 2 * b);
            tott += __ldcg(g.part + 2 * b + 1);
        }
        if (offt <= 1e-30 * tott) break;
        // the partials are rewritten next sweep only after every block has read
        // them: the first round's barrier lies in between
        for (int round = 0; round < ne - 1; round++) {
            if (tid < half) {
                auto pos = [&](int j) { return j == 0 ? 0 : 1 + ((j - 1 + round) % (ne - 1)); };
                int p = pos(tid), q = pos(ne - 1 - tid);
                if (p > q) { const int t = p; p = q; q = t; }
                double c = 1.0, s = 0.0;
                if (q < n) {
                    const double apq = __ldcg(ap + pk_idx(p, q));
                    if (fabs(apq) >= 1e-300) {
                        const double app = __ldcg(ap + pk_idx(p, p)), aqq = __ldcg(ap + pk_idx(q, q));
                        const double th = (aqq - app) / (2.0 * apq);
                        const double t = (th >= 0 ? 1.0 : -1.0) / (fabs(th) + sqrt(th * th + 1.0));
                        c = 1.0 / sqrt(t * t + 1.0);
                        s = t * c;
                    }
                }
                pp[tid] = p; qq[tid] = q; cs[tid] = c; sn[tid] = s;
            }
            // every block has read the diagonal entries that the round's K = L
            // blocks are about to overwrite
            if (!grid_barrier(g.count, (++bar) * gridDim.x, g.abort, err, g.wait_cycles)) return;
            // A <- J^T A J: block (K, L), K <= L, numbered column by column
            for (int e = gtid; e < nblk; e += gthreads) {
                int L = (int)((sqrt(8.0 * e + 1.0) - 1.0) * 0.5);
                while ((L + 1) * (L + 2) / 2 <= e) L++;
                while (L * (L + 1) / 2 > e) L--;
                const int K = e - L * (L + 1) / 2;
                const int pK = pp[K], qK = qq[K], pL = pp[L], qL = qq[L];
                const double cK = cs[K], sK = sn[K], cL = cs[L], sL = sn[L];
                if (K == L) {
                    if (qK < n && sK != 0.0) {
                        const double app = __ldcg(ap + pk_idx(pK, pK)), aqq = __ldcg(ap + pk_idx(qK, qK));
                        const double apq = __ldcg(ap + pk_idx(pK, qK));
                        ap[pk_idx(pK, pK)] = cK * cK * app - 2.0 * cK * sK * apq + sK * sK * aqq;
                        ap[pk_idx(qK, qK)] = sK * sK * app + 2.0 * cK * sK * apq + cK * cK * aqq;
                        ap[pk_idx(pK, qK)] = 0.0;
                    }
                    continue;
                }
                if (sK == 0.0 && sL == 0.0) continue;
                const bool hq = qK < n, hqL = qL < n;
                const double b11 = __ldcg(ap + pk_sym(pK, pL));
                const double b12 = hqL ? __ldcg(ap + pk_sym(pK, qL)) : 0.0;
                const double b21 = hq ? __ldcg(ap + pk_sym(qK, pL)) : 0.0;
                const double b22 = (hq && hqL) ? __ldcg(ap + pk_sym(qK, qL)) : 0.0;
                const double d11 = cL * b11 - sL * b12, d12 = sL * b11 + cL * b12;
                const double d21 = cL * b21 - sL * b22, d22 = sL * b21 + cL * b22;
                ap[pk_sym(pK, pL)] = cK * d11 - sK * d21;
                if (hqL) ap[pk_sym(pK, qL)] = cK * d12 - sK * d22;
                if (hq) ap[pk_sym(qK, pL)] = sK * d11 + cK * d21;
                if (hq && hqL) ap[pk_sym(qK, qL)] = sK * d12 + cK * d22;
            }
            // V <- V J, one (rotation, row) pair per work item
            for (int e = gtid; e < half * n; e += gthreads) {
                const int k = e / n, r = e - k * n;
                const int p = pp[k], q = qq[k];
                const double s = sn[k];
                if (q >= n || s == 0.0) continue;
                const double c = cs[k];
                const double vp = __ldcg(V + (size_t)p * n + r), vq = __ldcg(V + (size_t)q * n + r);
                V[(size_t)p * n + r] = c * vp - s * vq;
                V[(size_t)q * n + r] = s * vp + c * vq;
            }
            if (!grid_barrier(g.count, (++bar) * gridDim.x, g.abort, err, g.wait_cycles)) return;
        }
    }
    for (int i = gtid; i < n; i += gthreads) evals[i] = __ldcg(ap + pk_idx(i, i));
}

// x_out[t][i] for 128 < n <= 256: blockIdx.y picks 64 output channels whose
// rows of S stay in shared memory; 16-sample tiles, one (sample, 2 channels)
// per thread; the same k-ascending FMA order as k_apply_sphere8.
constexpr int kSphTileQ = 16;
__global__ void __launch_bounds__(512, 1) k_apply_sphere_q(const float* __restrict__ x, int64_t T,
                                                           int n, const double* __restrict__ mean,
                                                           const double* __restrict__ S,
                                                           float* __restrict__ xo, int ldx, int tf32) {
    extern __shared__ __align__(16) double sq[];
    double* Sq = sq;                                   // [256][64]: S(i0 + il, k) at k * 64 + il
    double* xc = sq + 256 * 64;                        // [16][257]
    constexpr int XL = 257;
    const int i0 = 64 * blockIdx.y;
    for (int e = threadIdx.x; e < 256 * 64; e += 512) {
        const int k = e >> 6, il = e & 63, i = i0 + il;
        Sq[e] = (i < n && k < n) ? S[(size_t)k * n + i] : 0.0;
    }
    const int s = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t ntile = (T + kSphTileQ - 1) / kSphTileQ;
    for (int64_t tile = blockIdx.x; tile < ntile; tile += gridDim.x) {
        const int64_t t0 = tile * kSphTileQ;
        __syncthreads();
        for (int e = threadIdx.x; e < kSphTileQ * 256; e += 512) {
            const int r = e >> 8, k = e & 255;
            const int64_t t = t0 + r;
            xc[r * XL + k] = (t < T && k < n) ? (double)x[t * n + k] - mean[k] : 0.0;
        }
        __syncthreads();
        double acc0 = 0.0, acc1 = 0.0;
#pragma unroll 4
        for (int k = 0; k < n; k++) {
            const double xv = xc[s * XL + k];
            acc0 = fma(Sq[k * 64 + lane], xv, acc0);
            acc1 = fma(Sq[k * 64 + lane + 32], xv, acc1);
        }
        const int64_t t = t0 + s;
        if (t < T) {
            const double accs[2] = {acc0, acc1};
#pragma unroll
            for (int u = 0; u < 2; u++) {
                const int i = i0 + lane + 32 * u;
                if (i < ldx) {
                    const float v = (i < n) ? (float)accs[u] : 0.f;
                    xo[t * ldx + i] = tf32 ? round_tf32(v) : v;
                }
            }
        }
    }
}

// x_out[t][i] = sum_k S(i,k) (x[t][k] - mean[k]) in FP64, rounded once to FP32
// (padded channels zero).  Persistent CTAs of 512 threads; S staged in shared
// memory; a thread computes 4 channels x 4 samples of a 64-sample tile.
constexpr int kSphTile = 64;
__global__ void __launch_bounds__(512, 1) k_apply_sphere8(const float* __restrict__ x, int64_t T, int n,
                                                          const double* __restrict__ mean,
                                                          const double* __restrict__ S,
                                                          float* __restrict__ xo, int ldx, int tf32) {
    extern __shared__ __align__(16) double ssm[];
    double* Ss = ssm;
    double* xc = ssm + 128 * 128;
    constexpr int XL = 129;
    for (int e = threadIdx.x; e < 128 * 128; e += 512) {
        const int k = e >> 7, i = e & 127;
        Ss[e] = (i < n && k < n) ? S[(size_t)k * n + i] : 0.0;
    }
    const int ib = threadIdx.x & 31, tb = threadIdx.x >> 5;     // channels 4 ib.., samples 4 tb..
    const int64_t ntile = (T + kSphTile - 1) / kSphTile;
    for (int64_t tile = blockIdx.x; tile < ntile; tile += gridDim.x) {
        const int64_t t0 = tile * kSphTile;
        __syncthreads();
        for (int e = threadIdx.x; e < kSphTile * 128; e += 512) {
            const int r = e >> 7, k = e & 127;
            const int64_t t = t0 + r;
            xc[r * XL + k] = (t < T && k < n) ? (double)x[t * n + k] - mean[k] : 0.0;
        }
        __syncthreads();
        double acc[4][4];
#pragma unroll
        for (int a = 0; a < 4; a++)
#pragma unroll
            for (int b = 0; b < 4; b++) acc[a][b] = 0.0;
#pragma unroll 4
        for (int k = 0; k < n; k++) {
            double s4[4], x4[4];
#pragma unroll
            for (int b = 0; b < 4; b += 2) {
                const double2 v = *reinterpret_cast<const double2*>(&Ss[k * 128 + 4 * ib + b]);
                s4[b] = v.x; s4[b + 1] = v.y;
            }
#pragma unroll
            for (int a = 0; a < 4; a++) x4[a] = xc[(4 * tb + a) * XL + k];
#pragma unroll
            for (int a = 0; a < 4; a++)
#pragma unroll
                for (int b = 0; b < 4; b++) acc[a][b] = fma(s4[b], x4[a], acc[a][b]);
        }
#pragma unroll
        for (int a = 0; a < 4; a++) {
            const int64_t t = t0 + 4 * tb + a;
            if (t >= T) continue;
#pragma unroll
            for (int b = 0; b < 4; b++) {
                const int i = 4 * ib + b;
                if (i < ldx) {
                    const float v = (i < n) ? (float)acc[a][b] : 0.f;
                    xo[t * ldx + i] = tf32 ? round_tf32(v) : v;
                }
            }
        }
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

// The preprocessing of one fit in three steps, so that a fit whose samples are
// spread over several contexts can add the sums of every shard between them:
//   pp_colsum:  column sums / div of the raw data;
//   pp_scatter: sum_t (x_t - mean)(x_t - mean)^T / div (do_sphere 1 only);
//   pp_finish:  the eigendecomposition of the covariance, S and ldetS, and
//               the sphered data x = S (raw - mean) in the layout of the E-step.
// part: scratch of pp_part_len doubles; evwork: >= 4 n^2 + 4 n doubles.
int sm_count() {
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    return nsm;
}

size_t pp_part_len(int64_t T, int n) {
    const size_t nblk = (size_t)((T + kChunk - 1) / kChunk);
    const size_t a = nblk * n, b = (size_t)sm_count() * n * n;
    return a > b ? a : b;
}

cudaError_t pp_colsum(const float* raw, int64_t T, int n, double div, double* part, double* out,
                      cudaStream_t st) {
    const int nblk = (int)((T + kChunk - 1) / kChunk);
    k_colsum<<<nblk, 256, 0, st>>>(raw, T, n, part);
    k_mean<<<1, 256, 0, st>>>(part, nblk, n, div, out);
    return cudaGetLastError();
}

cudaError_t pp_scatter(const float* raw, int64_t T, int n, const double* means, double div,
                       double* part, double* out, cudaStream_t st) {
    const int ncov = sm_count();
    const int64_t chunk = ((T + ncov - 1) / ncov + kCovRows - 1) / kCovRows * kCovRows;
    if (n <= 128) {
        k_cov8<<<ncov, 256, 0, st>>>(raw, T, n, chunk, means, part);
    } else {
        const size_t csmem = sizeof(double) * 2 * kCovRows * 128;
        cudaError_t e = cudaFuncSetAttribute(k_cov8q, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)csmem);
        if (e != cudaSuccess) return e;
        k_cov8q<<<dim3(ncov, 4), 256, csmem, st>>>(raw, T, n, chunk, means, part);
    }
    k_cov_reduce<<<(n * n + 255) / 256, 256, 0, st>>>(part, ncov, n, div, out);
    return cudaGetLastError();
}

// var_ready: evwork's variance slot already holds the do_sphere 2 variances
cudaError_t pp_finish(const float* raw, int64_t T, int n, int do_sphere, const double* means,
                      const double* cov, double* sphere, double* evwork, double* ldetS_dev,
                      float* x, int ldx, int tf32, int* err, double* part, bool var_ready,
                      cudaStream_t st, long long fault_wait_cycles) {
    const bool big = n > 128;
    const int nsm = sm_count();
    cudaError_t e = cudaSuccess;
    double* V = evwork;
    double* ev = evwork + (size_t)n * n;
    double* var = ev + n;
    if (do_sphere == 1 && !big) {
        const size_t jsmem = sizeof(double) * (size_t)((((n * (n + 1)) / 2 + 1) & ~1) + n * n);
        e = cudaFuncSetAttribute(k_jacobi_smem, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)jsmem);
        if (e != cudaSuccess) return e;
        k_jacobi_smem<<<1, kJacThreads, jsmem, st>>>(cov, V, ev, n);
    } else if (do_sphere == 1) {
        // Jacobi state in the partial buffer: packed triangle, the stopping-test
        // partials, the barrier counter and the abort flag
        int per_sm = 0;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_jacobi_grid, kJacThreads, 0);
        if (e != cudaSuccess || per_sm < 1) return e ? e : cudaErrorInvalidValue;
        const int nb = nsm < 64 ? nsm : 64;
        const size_t np = (size_t)n * (n + 1) / 2;
        JacGlobal jg;
        jg.ap = part;
        jg.part = part + np;
        jg.count = reinterpret_cast<unsigned*>(part + np + 2 * nb);
        jg.abort = reinterpret_cast<int*>(part + np + 2 * nb + 1);
        jg.wait_cycles = fault_wait_cycles > 0 ? fault_wait_cycles : 2000000000LL;
        jg.skip_block = fault_wait_cycles > 0 ? 0 : -1;
        e = cudaMemsetAsync(part + np + 2 * nb, 0, 2 * sizeof(double), st);
        if (e != cudaSuccess) return e;
        double* covp = const_cast<double*>(cov);
        void* args[] = {(void*)&covp, (void*)&V, (void*)&ev, (void*)&n, (void*)&jg, (void*)&err};
        e = cudaLaunchCooperativeKernel((const void*)k_jacobi_grid, dim3(nb), dim3(kJacThreads), args, 0, st);
        if (e != cudaSuccess) return e;
    } else if (do_sphere == 2 && !var_ready) {
        k_var<<<n, 256, 0, st>>>(raw, T, n, means, var);
    }
    k_sphere<<<(n * n + 255) / 256, 256, 0, st>>>(V, ev, var, n, do_sphere, sphere, ldetS_dev);
    if (big) {
        const size_t smemq = sizeof(double) * (256 * 64 + kSphTileQ * 257);
        e = cudaFuncSetAttribute(k_apply_sphere_q, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smemq);
        if (e != cudaSuccess) return e;
        const int64_t ntq = (T + kSphTileQ - 1) / kSphTileQ;
        const int gq = (int)(ntq < nsm ? ntq : nsm);
        k_apply_sphere_q<<<dim3(gq, (ldx + 63) / 64), 512, smemq, st>>>(raw, T, n, means, sphere, x, ldx, tf32);
        return cudaGetLastError();
    }
    const size_t smem2 = sizeof(double) * (128 * 128 + kSphTile * 129);
    e = cudaFuncSetAttribute(k_apply_sphere8, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem2);
    if (e != cudaSuccess) return e;
    const int64_t ntile = (T + kSphTile - 1) / kSphTile;
    const int gsph = (int)(ntile < nsm ? ntile : nsm);
    k_apply_sphere8<<<gsph, 512, smem2, st>>>(raw, T, n, means, sphere, x, ldx, tf32);
    return cudaGetLastError();
}

}  // namespace

namespace amica {

// fault_wait_cycles > 0 arms the test hook of amica_test_arm_wait_fault for
// this launch (cooperative eigensolver only: block 0 skips its first arrival,
// every wait is bounded by fault_wait_cycles).
cudaError_t launch_preprocess(const float* raw, int64_t T, int n, int do_sphere, double* means,
                              double* cov, double* sphere, double* evwork, double* ldetS_dev,
                              float* x, int ldx, int tf32, int* err, cudaStream_t st,
                              long long fault_wait_cycles) {
    if (n > 256 || ldx > 256) return cudaErrorInvalidValue;
    double* part = nullptr;
    cudaError_t e = cudaMallocAsync(&part, sizeof(double) * pp_part_len(T, n), st);
    if (e != cudaSuccess) return e;
    e = pp_colsum(raw, T, n, (double)T, part, means, st);
    if (e == cudaSuccess && do_sphere == 1) e = pp_scatter(raw, T, n, means, (double)T, part, cov, st);
    if (e == cudaSuccess)
        e = pp_finish(raw, T, n, do_sphere, means, cov, sphere, evwork, ldetS_dev, x, ldx, tf32, err, part,
                      false, st, fault_wait_cycles);
    cudaFreeAsync(part, st);
    return e;
}

// Sharded preprocessing: the column sums of this shard's raw data (n doubles).
cudaError_t launch_shard_colsum(const float* raw, int64_t T, int n, double* sums, cudaStream_t st) {
    if (n > 256) return cudaErrorInvalidValue;
    double* part = nullptr;
    cudaError_t e = cudaMallocAsync(&part, sizeof(double) * pp_part_len(T, n), st);
    if (e != cudaSuccess) return e;
    e = pp_colsum(raw, T, n, 1.0, part, sums, st);
    cudaFreeAsync(part, st);
    return e;
}

// means = sums / T_total (the column sums of all shards), then the scatter of
// this shard's raw data about them, n x n doubles.
cudaError_t launch_shard_scatter(const float* raw, int64_t T, int n, const double* sums, int64_t T_total,
                                 double* means, double* scatter, cudaStream_t st) {
    if (n > 256 || T_total < 1) return cudaErrorInvalidValue;
    double* part = nullptr;
    cudaError_t e = cudaMallocAsync(&part, sizeof(double) * pp_part_len(T, n), st);
    if (e != cudaSuccess) return e;
    k_mean<<<1, 256, 0, st>>>(sums, 1, n, (double)T_total, means);
    e = pp_scatter(raw, T, n, means, 1.0, part, scatter, st);
    cudaFreeAsync(part, st);
    return e;
}

// S and ldetS from the scatter of all shards (T_total samples; do_sphere 1 and
// 2 read it, 0 ignores it), applied to this shard's samples.
cudaError_t launch_shard_finish(const float* raw, int64_t T, int n, int do_sphere, const double* means,
                                const double* scatter, int64_t T_total, double* cov, double* sphere,
                                double* evwork, double* ldetS_dev, float* x, int ldx, int tf32, int* err,
                                cudaStream_t st) {
    if (n > 256 || ldx > 256 || T_total < 2) return cudaErrorInvalidValue;
    double* part = nullptr;
    cudaError_t e = cudaMallocAsync(&part, sizeof(double) * pp_part_len(T, n), st);
    if (e != cudaSuccess) return e;
    if (do_sphere != 0)
        k_scale_scatter<<<(n * n + 255) / 256, 256, 0, st>>>(scatter, n, (double)T_total, cov,
                                                             evwork + (size_t)n * n + n);
    e = cudaGetLastError();
    if (e == cudaSuccess)
        e = pp_finish(raw, T, n, do_sphere, means, cov, sphere, evwork, ldetS_dev, x, ldx, tf32, err, part,
                      true, st, 0);
    cudaFreeAsync(part, st);
    return e;
}

cudaError_t launch_convert_sphered(const double* xs, int64_t T, int n, float* x, int ldx, int tf32,
                                   cudaStream_t st) {
    k_convert<<<2048, 256, 0, st>>>(xs, T, n, x, ldx, tf32);
    return cudaGetLastError();
}

}  // namespace amica
