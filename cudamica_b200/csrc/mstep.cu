// FP64 device-side M-step of the AMICA EM iteration, plus the per-iteration
// preparation of the E-step constants and the deterministic reduction of the
// E-step's per-CTA partial sums.
//
// The reference runs this part as ~40 small FP64 kernels, cuBLAS/MAGMA calls
// and host round trips per iteration (src/amica.cu:835-924 and :1981-2512:
// host SVD for pinv, a synchronous bflag copy, ...).  Here it is six small
// kernels that stay on the device, so that a whole iteration can be captured
// in one CUDA graph and no host synchronisation is needed between iterations.
#include <algorithm>
#include <cmath>
#include <cstdint>

#include "common.cuh"

using namespace amica;

namespace {

constexpr int kT = 256;

__device__ double block_sum(double v, double* sh) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int w = threadIdx.x / 32, l = threadIdx.x % 32;
    __syncthreads();
    if (l == 0) sh[w] = v;
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x == 0) {
        for (int i = 0; i < (int)(blockDim.x / 32); i++) s += sh[i];
        sh[32] = s;
    }
    __syncthreads();
    return sh[32];
}

// ---------------------------------------------------------------------------
// k_inverse_derive: W_h = A_h^{-1}, ldet_h = -log|det A_h| and the FP32 E-step
// constants, one CTA of 512 threads per model (n <= 128).  Replaces pinv() and
// the LU log-determinant (src/amica.cu:27-127, :864-924).
//
// Gauss-Jordan elimination with partial pivoting and no row interchanges: the
// pivot of column k is a not yet used row p_k of (nearly) largest |a(p_k, k)|.
// Sweeping (p_k, k) in place,
//   a(p, k) <- 1 / a(p, k),   a(p, j) <- a(p, j) / a(p, k),
//   a(i, k) <- -a(i, k) / a(p, k),   a(i, j) <- a(i, j) - a(i, k) a(p, j) / a(p, k),
// turns column k into column p_k of P.A^{-1}, so at the end W(j, p_k) = a(p_j, k).
//
// Columns are swept in panels of 16.  Warps 0-1 sweep a panel's columns alone
// (thread r holds rows r and r + 64 of the panel in registers): the pivot of
// column k only depends on column k as updated by the earlier pivots, and those
// updates only read the pivot rows' panel entries.  The pivot key of a row is
// the high word of |a| with its low 7 bits replaced by 127 - row (so the pivot
// is within 2^-13 of the column's largest |a|, lowest row on ties); each warp's
// best row publishes its panel row and its reciprocal (every row forms the
// reciprocal of its candidate while the warp max runs), and after one 64-thread
// barrier every thread takes the larger key, updates the next column first and
// starts the next search before the rest of its rows.
//
// Sweeping a panel's pivots (P, K) one after another is, on the other columns
// C, the block sweep
//   a(i, C) <- [i not in P] a(i, C) + sum_t X(i, t) a_old(p_t, C),
// X being the swept panel: FP64 products on the tensor cores (mma.sync
// m8n8k4; tcgen05 has no FP64 kind) with operands in shared memory.  The
// next panel's columns get it first (all warps), then warps 4-15 apply it to
// the remaining columns while warps 0-1 sweep the next panel.
constexpr int kInvThreads = 512;
constexpr int kInvN = 128;                            // padded order
constexpr int kPanel = 16;                            // columns per panel
constexpr int kLdA = kInvN + 1;                       // odd: a warp reading a column of 32 rows hits distinct banks
constexpr int kLdX = kPanel + 4;                      // 16-byte rows; 40-word stride puts an 8 x 4 fragment on distinct banks
constexpr size_t kInvSmem = sizeof(double) * ((size_t)kInvN * kLdA + 3 * (size_t)kInvN * kLdX);

__device__ __forceinline__ void bar_panel() { asm volatile("bar.sync 1, 64;" ::: "memory"); }

// D(8x8) += A(8x4) B(4x8) in FP64: lane (g, q) = (lane / 4, lane % 4) holds
// A(g, q), B(q, g) and D(g, 2q), D(g, 2q + 1)
__device__ __forceinline__ void dmma884(double& d0, double& d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

// pivot key of row r holding v (0: not a candidate)
__device__ __forceinline__ uint32_t pivot_key(double v, bool usable, int r) {
    return usable ? ((((uint32_t)__double2hiint(v)) & 0x7fffff80u) | (uint32_t)(127 - r)) + 128u : 0u;
}

// a(i, 8 ct + [0, 8)) for the 16 rows tiles rt0 + [0, 8) <- [i not in P] a + X Pt^T, P the
// pivot rows of the panel at k0, X its swept columns, Pt the pivot rows' old
// entries (Pt[j][t] = a_old(p_t, j)); one warp
__device__ __forceinline__ void block_sweep_strip(double* __restrict__ As, const double* __restrict__ X,
                                                  const double* __restrict__ Pt, const int* pinv, int k0,
                                                  int ct, int rt0, int nrt, int lane) {
    const int g = lane >> 2, q = lane & 3;
    const int j = 8 * ct + 2 * q;
    double acc[8][2];
#pragma unroll
    for (int u = 0; u < 8; u++) {
        if (u < nrt) {
            const int i = 8 * (rt0 + u) + g;
            // rows pivoted in this panel have pinv in [k0, k0 + 16); other rows'
            // pinv is either not set yet or outside that range
            const bool prow = (unsigned)(pinv[i] - k0) < (unsigned)kPanel;
            acc[u][0] = prow ? 0.0 : As[i * kLdA + j];
            acc[u][1] = prow ? 0.0 : As[i * kLdA + j + 1];
        }
    }
#pragma unroll
    for (int s = 0; s < kPanel; s += 4) {
        const double bf = Pt[(8 * ct + g) * kLdX + s + q];
#pragma unroll
        for (int u = 0; u < 8; u++)
            if (u < nrt) dmma884(acc[u][0], acc[u][1], X[(8 * (rt0 + u) + g) * kLdX + s + q], bf);
    }
#pragma unroll
    for (int u = 0; u < 8; u++) {
        if (u < nrt) {
            const int i = 8 * (rt0 + u) + g;
            As[i * kLdA + j] = acc[u][0];
            As[i * kLdA + j + 1] = acc[u][1];
        }
    }
}

__global__ void __launch_bounds__(kInvThreads, 1) k_inverse_derive(
    const double* __restrict__ A, const double* __restrict__ c, const double* __restrict__ alpha,
    const double* __restrict__ mu, const double* __restrict__ beta, const double* __restrict__ rho,
    const double* __restrict__ gm, double ldetS, double* __restrict__ W, double* __restrict__ ldet,
    double* __restrict__ ltc64, float* __restrict__ Wf, float* __restrict__ wcf,
    MixParam* __restrict__ mp, int n, int m, int NP, int* err) {
    extern __shared__ __align__(16) double smem_inv[];
    double* As = smem_inv;                            // a(r, j) at As[r * kLdA + j]
    double* Xs = As + kInvN * kLdA;                   // swept panels, two buffers: Xs[b & 1][r * kLdX + t]
    double* Pt = Xs + 2 * kInvN * kLdX;               // Pt[j * kLdX + t] = a(p_t, j) before the panel's update
    __shared__ __align__(16) double crow_v[2][2][kPanel];   // each panel warp's candidate row
    __shared__ uint32_t ckey[2][2];
    __shared__ double cpiv[2][2], cinv[2][2];
    __shared__ double pivs[kInvN], wcs[kInvN], cperm[kInvN], cs[kInvN];
    __shared__ float sb_cl2[kMaxMix * kInvN];      // log2 normaliser per (mixture, channel)
    __shared__ int perm[kInvN], pinv[kInvN];
    __shared__ int s_bad;
    __shared__ double s_lgm;
    const int h = blockIdx.x, tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const double* Ah = A + (size_t)h * n * n;
    for (int e = tid; e < kInvN * kInvN; e += kInvThreads) {
        const int j = e >> 7, r = e & (kInvN - 1);
        As[r * kLdA + j] = (r < n && j < n) ? Ah[(size_t)j * n + r] : 0.0;
    }
    if (tid < kInvN) pinv[tid] = 0x7fffffff;
    if (tid == 0) s_bad = 0;
    // panel threads (tid < 64): rows r0 = tid and r1 = tid + 64, not yet pivot rows
    const int r0 = tid, r1 = tid + 64;
    bool us0 = r0 < n, us1 = r1 < n;
    const int npan = (n + kPanel - 1) / kPanel;
    __syncthreads();
    for (int b = 0; b <= npan; b++) {
        const int k0 = kPanel * b;
        if (b < npan && warp < 2) {
            double* Xb = Xs + (b & 1) * kInvN * kLdX;
            double pa[kPanel], pb[kPanel];            // rows r0 and r1
#pragma unroll
            for (int t = 0; t < kPanel; t++) {
                pa[t] = As[r0 * kLdA + k0 + t];
                pb[t] = As[r1 * kLdA + k0 + t];
            }
            bool bad = false;
            uint32_t ka = pivot_key(pa[0], us0, r0), kb = pivot_key(pb[0], us1, r1);
            uint32_t key = max(ka, kb);
            double v = kb > ka ? pb[0] : pa[0];
            double rv = 1.0 / v;
            uint32_t wkey = __reduce_max_sync(0xffffffffu, key);
#pragma unroll
            for (int t = 0; t < kPanel; t++) {
                if (k0 + t >= n) break;               // uniform
                const int buf = t & 1;
                if (wkey == 0u) {
                    if (lane == 0) ckey[buf][warp] = 0u;
                } else if (key == wkey) {             // one thread: the key names its row
                    const bool second = kb == key;
#pragma unroll
                    for (int j = 0; j < kPanel; j += 2)
                        *reinterpret_cast<double2*>(&crow_v[buf][warp][j]) =
                            second ? make_double2(pb[j], pb[j + 1]) : make_double2(pa[j], pa[j + 1]);
                    ckey[buf][warp] = key;
                    cpiv[buf][warp] = v;
                    cinv[buf][warp] = rv;
                }
                bar_panel();
                const uint32_t kw0 = ckey[buf][0], kw1 = ckey[buf][1];
                const int wb = kw1 > kw0 ? 1 : 0;     // distinct unless both 0
                const uint32_t best = max(kw0, kw1);
                const double piv = wb ? cpiv[buf][1] : cpiv[buf][0];
                const double inv = wb ? cinv[buf][1] : cinv[buf][0];
                const int tn = t + 1 < kPanel ? t + 1 : t;
                const double pn = wb ? crow_v[buf][1][tn] : crow_v[buf][0][tn];
                if (best == 0u || piv == 0.0) { bad = true; break; }   // same in every panel thread
                const int p = 127 - (int)((best - 128u) & 127u);
                const double* pp = crow_v[buf][wb];
                if (tid == 0) { perm[k0 + t] = p; pinv[p] = k0 + t; pivs[k0 + t] = piv; }
                const bool pa_is_p = r0 == p, pb_is_p = r1 == p;
                us0 = us0 && !pa_is_p;
                us1 = us1 && !pb_is_p;
                const double fa = pa[t] * inv, fb = pb[t] * inv;
                if (t + 1 < kPanel) {                 // the next column first, and the next search
                    pa[t + 1] = fma(-fa, pn, pa[t + 1]);
                    pb[t + 1] = fma(-fb, pn, pb[t + 1]);
                    ka = pivot_key(pa[t + 1], us0, r0);
                    kb = pivot_key(pb[t + 1], us1, r1);
                    key = max(ka, kb);
                    v = kb > ka ? pb[t + 1] : pa[t + 1];
                    rv = 1.0 / v;
                    wkey = __reduce_max_sync(0xffffffffu, key);
                }
                double ppv[kPanel];                   // the pivot row, read once for both rows
#pragma unroll
                for (int j = 0; j < kPanel; j += 2) {
                    const double2 d = *reinterpret_cast<const double2*>(pp + j);
                    ppv[j] = d.x;
                    ppv[j + 1] = d.y;
                }
#pragma unroll
                for (int j = 0; j < kPanel; j++)
                    if (j != t && j != t + 1) {
                        pa[j] = fma(-fa, ppv[j], pa[j]);
                        pb[j] = fma(-fb, ppv[j], pb[j]);
                    }
                pa[t] = -fa;
                pb[t] = -fb;
                if (pa_is_p) {                        // the pivot row: its own entries over the pivot
#pragma unroll
                    for (int j = 0; j < kPanel; j++) pa[j] = j == t ? inv : ppv[j] * inv;
                }
                if (pb_is_p) {
#pragma unroll
                    for (int j = 0; j < kPanel; j++) pb[j] = j == t ? inv : ppv[j] * inv;
                }
            }
            if (bad && tid == 0) s_bad = 1;
#pragma unroll
            for (int t = 0; t < kPanel; t++) {
                As[r0 * kLdA + k0 + t] = pa[t];
                As[r1 * kLdA + k0 + t] = pb[t];
            }
#pragma unroll
            for (int t = 0; t < kPanel; t += 2) {
                *reinterpret_cast<double2*>(&Xb[r0 * kLdX + t]) = make_double2(pa[t], pa[t + 1]);
                *reinterpret_cast<double2*>(&Xb[r1 * kLdX + t]) = make_double2(pb[t], pb[t + 1]);
            }
        } else if (b == 0) {
            // parameter-only work of the E-step constants, off the elimination's path
            for (int e = tid - 64; e < m * NP; e += kInvThreads - 64) {
                const int j = e / NP, i = e - j * NP;
                float cl = 0.f;
                if (i < n) {
                    const size_t idx = ((size_t)h * m + j) * n + i;
                    cl = (float)((log(alpha[idx]) + 0.5 * log(beta[idx]) - M_LN2 -
                                  lgamma(1.0 + 1.0 / rho[idx])) * 1.4426950408889634);
                }
                sb_cl2[e] = cl;
            }
            if (tid >= 64 && tid < 64 + kInvN) cs[tid - 64] = tid - 64 < n ? c[(size_t)h * n + tid - 64] : 0.0;
            if (tid == 64 + kInvN) s_lgm = log(gm[h]);
        } else if (b >= 1 && (b == npan || warp >= 4)) {
            // the previous panel's block sweep on the columns outside it and
            // outside this panel (which got it already), in column strips of 8
            const int kp = k0 - kPanel;
            const double* Xp = Xs + ((b - 1) & 1) * kInvN * kLdX;
            const int w0 = b == npan ? 0 : 4, nw = b == npan ? 16 : 12;
            for (int ct = warp - w0; ct < kInvN / 8; ct += nw) {
                const int j0 = 8 * ct;
                if ((unsigned)(j0 - kp) < (unsigned)kPanel || (unsigned)(j0 - k0) < (unsigned)kPanel) continue;
                block_sweep_strip(As, Xp, Pt, pinv, kp, ct, 0, 8, lane);
                block_sweep_strip(As, Xp, Pt, pinv, kp, ct, 8, 8, lane);
            }
        }
        __syncthreads();
        if (s_bad || b == npan) break;
        // Pt for this panel: its pivot rows' entries outside it, now final up to it
        const int w = min(kPanel, n - k0);
        for (int e = tid; e < kPanel * kInvN; e += kInvThreads) {
            const int j = e >> 4, t = e & (kPanel - 1);
            if ((unsigned)(j - k0) < (unsigned)kPanel) continue;
            Pt[j * kLdX + t] = t < w ? As[perm[k0 + t] * kLdA + j] : 0.0;
        }
        __syncthreads();
        if (b + 1 < npan) {
            // the next panel's 16 columns: 2 strips x 16 row tiles, 2 tiles per warp
            const double* Xb = Xs + (b & 1) * kInvN * kLdX;
            block_sweep_strip(As, Xb, Pt, pinv, k0, 2 * (b + 1) + (warp & 1), 2 * (warp >> 1), 2, lane);
        }
        __syncthreads();
    }
    if (s_bad) {
        if (tid == 0) atomicOr(err, kErrSingular);
        return;
    }
    // W(j, q) = a(perm[j], pinv[q]).  W_h column-major: thread j = tid % 128 holds
    // its row index perm[j] and walks the columns
    double* Wh = W + (size_t)h * n * n;
    {
        const int j = tid & (kInvN - 1);
        if (j < n) {
            const double* Wr = As + perm[j] * kLdA;
#pragma unroll 4
            for (int q = tid >> 7; q < n; q += kInvThreads / kInvN) Wh[(size_t)q * n + j] = Wr[pinv[q]];
        }
    }
    if (tid < n) {
        pivs[tid] = log(fabs(pivs[tid]));
        cperm[tid] = cs[perm[tid]];                  // c at the column that holds its W column
    }
    __syncthreads();
    if (warp == 0) {
        double ld = 0.0;
        for (int k = lane; k < n; k += 32) ld += pivs[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) ld += __shfl_xor_sync(0xffffffffu, ld, o);
        if (lane == 0) {
            ldet[h] = -ld;
            ltc64[h] = s_lgm - ld + ldetS;            // src/amica.cu:1009
        }
    }
    // E-step constants: W in FP32 (row-major, NP x NP, zero padded), w_c = W c,
    // and per (mixture, channel) sqrt(beta), sqrt(beta)(mu + w_c), the log2
    // normaliser and rho.  w_c(i) = sum_col a(perm[i], col) c(perm[col]): four
    // threads per row, each a quarter of the columns
    {
        const int i = tid >> 2, part = tid & 3;
        double s = 0.0;
        if (i < n) {
            const double* Wr = As + perm[i] * kLdA;
#pragma unroll 8
            for (int col = part; col < n; col += 4) s = fma(Wr[col], cperm[col], s);
        }
        s += __shfl_xor_sync(0xffffffffu, s, 1);
        s += __shfl_xor_sync(0xffffffffu, s, 2);
        if (part == 0 && i < NP) {
            wcs[i] = s;
            wcf[(size_t)h * NP + i] = (float)s;
        }
    }
    float* Wfh = Wf + (size_t)h * NP * NP;
    {
        // NP divides the block: thread k = tid % NP keeps pinv[k] and walks the rows
        const int k = tid % NP;
        const int pk = k < n ? pinv[k] : 0;
#pragma unroll 4
        for (int i = tid / NP; i < NP; i += kInvThreads / NP)
            Wfh[(size_t)i * NP + k] = (i < n && k < n) ? (float)As[perm[i] * kLdA + pk] : 0.f;
    }
    __syncthreads();
    for (int e = tid; e < m * NP; e += kInvThreads) {
        const int j = e / NP, i = e - j * NP;
        MixParam q;
        if (i < n) {
            const size_t idx = ((size_t)h * m + j) * n + i;
            const double s = sqrt(beta[idx]);
            const double r = rho[idx];
            q.s = (float)s;
            q.off = (float)(s * (mu[idx] + wcs[i]));
            q.cl2 = sb_cl2[e];
            q.rho = (float)r;
        } else {
            q.s = 0.f; q.off = 0.f; q.cl2 = 0.f; q.rho = 1.f;
        }
        mp[((size_t)h * m + j) * NP + i] = q;
    }
}

// ---------------------------------------------------------------------------
// k_inverse_big: W_h = A_h^{-1} and log|pivots| for 128 < n <= 256, where the
// n x n FP64 matrix no longer fits in one SM's shared memory.  The blocked
// Gauss-Jordan elimination of k_inverse_derive (16-column panels, the same
// pivot keys with 8 row bits, the block sweep on the FP64 tensor cores with
// look-ahead) on a row-major working copy in global memory (L2-resident, 512
// KB at n = 256); one CTA of 512 threads per model.  Warps 0-3 sweep a panel
// (thread r holds rows r and r + 128, one 128-thread barrier per pivot);
// warps 4-15 apply the previous panel's block sweep to the other columns,
// reading and writing their accumulators in global memory.
constexpr int kMaxN = 256;
constexpr int kBigN = kMaxN;
constexpr size_t kBigSmem = sizeof(double) * 3 * (size_t)kBigN * kLdX;

__device__ __forceinline__ void bar_panel4() { asm volatile("bar.sync 1, 128;" ::: "memory"); }

__device__ __forceinline__ uint32_t pivot_key8(double v, bool usable, int r) {
    return usable ? ((((uint32_t)__double2hiint(v)) & 0x7fffff00u) | (uint32_t)(255 - r)) + 256u : 0u;
}

// the global-memory form of block_sweep_strip: a(i, 8 ct + [0, 8)) for the
// row tiles rt0 + [0, nrt) of G (row-major, stride n; rows and columns at and
// beyond n are skipped)
__device__ __forceinline__ void block_sweep_strip_g(double* __restrict__ G, int n, const double* __restrict__ X,
                                                    const double* __restrict__ Pt, const int* pinv, int k0,
                                                    int ct, int rt0, int nrt, int lane) {
    const int g = lane >> 2, q = lane & 3;
    const int j = 8 * ct + 2 * q;
    const bool ok0 = j < n, ok1 = j + 1 < n;
    double acc[8][2];
#pragma unroll
    for (int u = 0; u < 8; u++) {
        if (u < nrt) {
            const int i = 8 * (rt0 + u) + g;
            const bool ok = i < n && !((unsigned)(pinv[i] - k0) < (unsigned)kPanel);
            acc[u][0] = ok && ok0 ? G[(size_t)i * n + j] : 0.0;
            acc[u][1] = ok && ok1 ? G[(size_t)i * n + j + 1] : 0.0;
        }
    }
#pragma unroll
    for (int s = 0; s < kPanel; s += 4) {
        const double bf = Pt[(8 * ct + g) * kLdX + s + q];
#pragma unroll
        for (int u = 0; u < 8; u++)
            if (u < nrt) dmma884(acc[u][0], acc[u][1], X[(8 * (rt0 + u) + g) * kLdX + s + q], bf);
    }
#pragma unroll
    for (int u = 0; u < 8; u++) {
        if (u < nrt) {
            const int i = 8 * (rt0 + u) + g;
            if (i < n) {
                if (ok0) G[(size_t)i * n + j] = acc[u][0];
                if (ok1) G[(size_t)i * n + j + 1] = acc[u][1];
            }
        }
    }
}

__global__ void __launch_bounds__(kInvThreads, 1) k_inverse_big(const double* __restrict__ A,
                                                               double* __restrict__ work,
                                                               double* __restrict__ W,
                                                               double* __restrict__ pivlog, int n,
                                                               int* err) {
    extern __shared__ __align__(16) double smem_big[];
    double* Xs = smem_big;                            // swept panels, two buffers of 256 x kLdX
    double* Pt = Xs + 2 * kBigN * kLdX;               // Pt[j * kLdX + t] = a(p_t, j) before the panel's update
    __shared__ __align__(16) double crow_v[2][4][kPanel];
    __shared__ uint32_t ckey[2][4];
    __shared__ double cpiv[2][4], cinv[2][4];
    __shared__ double pivs[kBigN];
    __shared__ int perm[kBigN], pinv[kBigN];
    __shared__ int s_bad;
    const int h = blockIdx.x, tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const double* Ah = A + (size_t)h * n * n;         // column-major a(r, j) = Ah[j n + r]
    double* G = work + (size_t)h * n * n;             // row-major a(r, j) = G[r n + j]
    for (int e = tid; e < n * n; e += kInvThreads) {
        const int j = e / n, r = e - j * n;
        G[(size_t)r * n + j] = Ah[e];
    }
    if (tid < kBigN) pinv[tid] = 0x7fffffff;
    if (tid == 0) s_bad = 0;
    const int r0 = tid, r1 = tid + 128;               // panel threads (tid < 128)
    bool us0 = r0 < n, us1 = r1 < n;
    const int npan = (n + kPanel - 1) / kPanel, ncs = (n + 7) / 8;
    __syncthreads();
    for (int b = 0; b <= npan; b++) {
        const int k0 = kPanel * b;
        if (b < npan && warp < 4) {
            double* Xb = Xs + (b & 1) * kBigN * kLdX;
            double pa[kPanel], pb[kPanel];
#pragma unroll
            for (int t = 0; t < kPanel; t++) {
                const bool cok = k0 + t < n;
                pa[t] = cok && r0 < n ? G[(size_t)r0 * n + k0 + t] : 0.0;
                pb[t] = cok && r1 < n ? G[(size_t)r1 * n + k0 + t] : 0.0;
            }
            bool bad = false;
            uint32_t ka = pivot_key8(pa[0], us0, r0), kb = pivot_key8(pb[0], us1, r1);
            uint32_t key = max(ka, kb);
            double v = kb > ka ? pb[0] : pa[0];
            double rv = 1.0 / v;
            uint32_t wkey = __reduce_max_sync(0xffffffffu, key);
#pragma unroll
            for (int t = 0; t < kPanel; t++) {
                if (k0 + t >= n) break;               // uniform
                const int buf = t & 1;
                if (wkey == 0u) {
                    if (lane == 0) ckey[buf][warp] = 0u;
                } else if (key == wkey) {             // one thread: the key names its row
                    const bool second = kb == key;
#pragma unroll
                    for (int j = 0; j < kPanel; j += 2)
                        *reinterpret_cast<double2*>(&crow_v[buf][warp][j]) =
                            second ? make_double2(pb[j], pb[j + 1]) : make_double2(pa[j], pa[j + 1]);
                    ckey[buf][warp] = key;
                    cpiv[buf][warp] = v;
                    cinv[buf][warp] = rv;
                }
                bar_panel4();
                const int tn = t + 1 < kPanel ? t + 1 : t;
                uint32_t best = ckey[buf][0];
                int wb = 0;
                double piv = cpiv[buf][0], inv = cinv[buf][0], pn = crow_v[buf][0][tn];
#pragma unroll
                for (int qq = 1; qq < 4; qq++) {
                    const uint32_t kq = ckey[buf][qq];
                    const double pq = cpiv[buf][qq], iq = cinv[buf][qq], nq = crow_v[buf][qq][tn];
                    if (kq > best) { best = kq; wb = qq; piv = pq; inv = iq; pn = nq; }
                }
                if (best == 0u || piv == 0.0) { bad = true; break; }   // same in every panel thread
                const int p = 255 - (int)((best - 256u) & 255u);
                const double* pp = crow_v[buf][wb];
                if (tid == 0) { perm[k0 + t] = p; pinv[p] = k0 + t; pivs[k0 + t] = piv; }
                const bool pa_is_p = r0 == p, pb_is_p = r1 == p;
                us0 = us0 && !pa_is_p;
                us1 = us1 && !pb_is_p;
                const double fa = pa[t] * inv, fb = pb[t] * inv;
                if (t + 1 < kPanel) {                 // the next column first, and the next search
                    pa[t + 1] = fma(-fa, pn, pa[t + 1]);
                    pb[t + 1] = fma(-fb, pn, pb[t + 1]);
                    ka = pivot_key8(pa[t + 1], us0, r0);
                    kb = pivot_key8(pb[t + 1], us1, r1);
                    key = max(ka, kb);
                    v = kb > ka ? pb[t + 1] : pa[t + 1];
                    rv = 1.0 / v;
                    wkey = __reduce_max_sync(0xffffffffu, key);
                }
                double ppv[kPanel];                   // the pivot row, read once for both rows
#pragma unroll
                for (int j = 0; j < kPanel; j += 2) {
                    const double2 d = *reinterpret_cast<const double2*>(pp + j);
                    ppv[j] = d.x;
                    ppv[j + 1] = d.y;
                }
#pragma unroll
                for (int j = 0; j < kPanel; j++)
                    if (j != t && j != t + 1) {
                        pa[j] = fma(-fa, ppv[j], pa[j]);
                        pb[j] = fma(-fb, ppv[j], pb[j]);
                    }
                pa[t] = -fa;
                pb[t] = -fb;
                if (pa_is_p) {                        // the pivot row: its own entries over the pivot
#pragma unroll
                    for (int j = 0; j < kPanel; j++) pa[j] = j == t ? inv : ppv[j] * inv;
                }
                if (pb_is_p) {
#pragma unroll
                    for (int j = 0; j < kPanel; j++) pb[j] = j == t ? inv : ppv[j] * inv;
                }
            }
            if (bad && tid == 0) s_bad = 1;
#pragma unroll
            for (int t = 0; t < kPanel; t++) {
                if (k0 + t < n) {
                    if (r0 < n) G[(size_t)r0 * n + k0 + t] = pa[t];
                    if (r1 < n) G[(size_t)r1 * n + k0 + t] = pb[t];
                }
            }
#pragma unroll
            for (int t = 0; t < kPanel; t += 2) {
                *reinterpret_cast<double2*>(&Xb[r0 * kLdX + t]) = make_double2(pa[t], pa[t + 1]);
                *reinterpret_cast<double2*>(&Xb[r1 * kLdX + t]) = make_double2(pb[t], pb[t + 1]);
            }
        } else if (b >= 1 && (b == npan || warp >= 4)) {
            // the previous panel's block sweep outside it and outside this panel
            const int kp = k0 - kPanel;
            const double* Xp = Xs + ((b - 1) & 1) * kBigN * kLdX;
            const int w0 = b == npan ? 0 : 4, nw = b == npan ? 16 : 12;
            for (int ct = warp - w0; ct < ncs; ct += nw) {
                const int j0 = 8 * ct;
                if ((unsigned)(j0 - kp) < (unsigned)kPanel || (unsigned)(j0 - k0) < (unsigned)kPanel) continue;
                for (int rt0 = 0; 8 * rt0 < n; rt0 += 8) block_sweep_strip_g(G, n, Xp, Pt, pinv, kp, ct, rt0, 8, lane);
            }
        }
        __syncthreads();
        if (s_bad || b == npan) break;
        // Pt for this panel: its pivot rows' entries outside it, now final up to it
        const int w = min(kPanel, n - k0);
        for (int e = tid; e < kPanel * kBigN; e += kInvThreads) {
            const int j = e >> 4, t = e & (kPanel - 1);
            if ((unsigned)(j - k0) < (unsigned)kPanel) continue;
            Pt[j * kLdX + t] = t < w && j < n ? G[(size_t)perm[k0 + t] * n + j] : 0.0;
        }
        __syncthreads();
        if (b + 1 < npan) {
            // the next panel's columns: 2 strips x 32 row tiles, 4 tiles per warp
            const double* Xb = Xs + (b & 1) * kBigN * kLdX;
            const int rt0 = 4 * (warp >> 1);
            if (8 * rt0 < n) block_sweep_strip_g(G, n, Xb, Pt, pinv, k0, 2 * (b + 1) + (warp & 1), rt0, 4, lane);
        }
        __syncthreads();
    }
    if (s_bad) {
        if (tid == 0) atomicOr(err, kErrSingular);
        return;
    }
    // W(j, q) = a(perm[j], pinv[q]), column-major W_h
    double* Wh = W + (size_t)h * n * n;
    {
        const int j = tid & (kBigN - 1);
        if (j < n) {
            const double* Gr = G + (size_t)perm[j] * n;
            for (int q = tid >> 8; q < n; q += kInvThreads / kBigN) Wh[(size_t)q * n + j] = Gr[pinv[q]];
        }
    }
    for (int k = tid; k < n; k += kInvThreads) pivlog[(size_t)h * n + k] = log(fabs(pivs[k]));
}

// k_derive: log|det W_h|, the Lt constant and the FP32 E-step constants from a
// column-major W (the tail of k_inverse_derive for the n > 128 path).  One CTA
// of 256 threads per model.
__global__ void __launch_bounds__(256) k_derive(
    const double* __restrict__ W, const double* __restrict__ pivlog, const double* __restrict__ c,
    const double* __restrict__ alpha, const double* __restrict__ mu, const double* __restrict__ beta,
    const double* __restrict__ rho, const double* __restrict__ gm, double ldetS,
    double* __restrict__ ldet, double* __restrict__ ltc64, float* __restrict__ Wf,
    float* __restrict__ wcf, MixParam* __restrict__ mp, int n, int m, int NP) {
    const int h = blockIdx.x, tid = threadIdx.x;
    const double* Wh = W + (size_t)h * n * n;
    __shared__ double wcs[kMaxN];
    if (tid == 0) {
        double ld = 0.0;
        for (int k = 0; k < n; k++) ld += pivlog[(size_t)h * n + k];
        ldet[h] = -ld;
        ltc64[h] = log(gm[h]) - ld + ldetS;           // src/amica.cu:1009
    }
    for (int i = tid; i < NP; i += blockDim.x) {
        double wc = 0.0;
        if (i < n)
            for (int k = 0; k < n; k++) wc += Wh[(size_t)k * n + i] * c[(size_t)h * n + k];
        wcs[i] = wc;
        wcf[(size_t)h * NP + i] = (float)wc;
    }
    float* Wfh = Wf + (size_t)h * NP * NP;
    for (int e = tid; e < NP * NP; e += blockDim.x) {
        const int i = e / NP, k = e - i * NP;
        Wfh[e] = (i < n && k < n) ? (float)Wh[(size_t)k * n + i] : 0.f;
    }
    __syncthreads();
    for (int e = tid; e < m * NP; e += blockDim.x) {
        const int j = e / NP, i = e - j * NP;
        MixParam q;
        if (i < n) {
            const size_t idx = ((size_t)h * m + j) * n + i;
            const double s = sqrt(beta[idx]);
            const double r = rho[idx];
            q.s = (float)s;
            q.off = (float)(s * (mu[idx] + wcs[i]));
            q.cl2 = (float)((log(alpha[idx]) + 0.5 * log(beta[idx]) - M_LN2 - lgamma(1.0 + 1.0 / r)) *
                            1.4426950408889634);
            q.rho = (float)r;
        } else {
            q.s = 0.f; q.off = 0.f; q.cl2 = 0.f; q.rho = 1.f;
        }
        mp[((size_t)h * m + j) * NP + i] = q;
    }
}

// Entry (r, cc) of the A-update matrix B_h (src/amica.cu:2155-2279,
// src/kernels.cu:961-1014): the Newton form when this model takes the Newton
// step, else the natural gradient I - phi / vsum.
__device__ __forceinline__ double b_entry(const double* __restrict__ phi, double ivs,
                                          const double* __restrict__ kappa,
                                          const double* __restrict__ lambda,
                                          const double* __restrict__ sig2, int newton, int r, int cc,
                                          int n) {
    const double prc = phi[(size_t)cc * n + r] * ivs;      // phi(r, c) / vsum
    if (newton) {
        if (r == cc) return (1.0 - prc) / lambda[r];
        const double pcr = phi[(size_t)r * n + cc] * ivs;
        const double nom = -sig2[r] * kappa[cc];
        return (nom * (-prc) + (-pcr)) / ((kappa[r] * sig2[r]) * (kappa[cc] * sig2[cc]) - 1.0);
    }
    return (r == cc ? 1.0 : 0.0) - prc;
}

// Batched FP64 32x32-tiled products on n x n column-major matrices, one
// (tile, model) per CTA of 256 threads:
//   kind 0 (A update, src/amica.cu:2330-2342):  Out = X + s_h X B_h,
//          s_h = +lrate (Newton) or -lrate (natural gradient), B_h formed
//          on the fly from phi, kappa, lambda and sigma2
//   kind 1 (phi from Psi):  Out = (Psi - gsum c^T) W^T, written into the
//          statistics vector's phi block
struct GemmArgs {
    int kind, n, m;
    const double* X; size_t strideX;
    const double* Y; size_t strideY;        // kind 1: W
    double* Out; size_t strideOut;
    const double* gs; size_t strideG;       // kind 1
    const double* c;                        // kind 1
    const int* use_newton;                  // kind 0
    const Ctrl* ctrl;                       // kind 0
    const double* stats;                    // kind 0: phi and vsum
    const double* work;                     // kind 0: kappa, lambda, sigma2
};

__global__ void __launch_bounds__(256) k_gemm64(GemmArgs g) {
    __shared__ double xs[32][33], ys[32][33];
    const int n = g.n;
    const int h = blockIdx.z;
    const int r0 = blockIdx.x * 32, c0 = blockIdx.y * 32;
    const int tx = threadIdx.x % 32, ty = threadIdx.x / 32;   // ty: 0..7
    const double* Xh = g.X + g.strideX * h;
    const double* Yh = g.kind == 1 ? g.Y + g.strideY * h : nullptr;
    StatLayout SL{n, g.m};
    const double* phi = g.kind == 0 ? g.stats + SL.base(h) + SL.phi() : nullptr;
    const double ivs = g.kind == 0 ? 1.0 / g.stats[SL.base(h) + SL.vs()] : 0.0;
    const double* kappa = g.kind == 0 ? g.work + (size_t)h * 4 * n : nullptr;
    const int newton = g.kind == 0 ? g.use_newton[h] : 0;
    if (newton < 0) {                                 // frozen model: A unchanged
        const int r = r0 + tx;
        for (int q = 0; q < 4; q++) {
            const int col = c0 + ty + 8 * q;
            if (r < n && col < n) g.Out[g.strideOut * h + (size_t)col * n + r] = Xh[(size_t)col * n + r];
        }
        return;
    }
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    for (int k0 = 0; k0 < n; k0 += 32) {
        for (int q = 0; q < 4; q++) {
            const int rr = ty + 8 * q;                 // tile-local k (for X) / k (for Y)
            // X(r0 + tx, k0 + rr)
            const int r = r0 + tx, k = k0 + rr;
            double xv = 0.0;
            if (r < n && k < n) {
                xv = Xh[(size_t)k * n + r];
                if (g.kind == 1) xv -= g.gs[g.strideG * h + r] * g.c[(size_t)h * n + k];
            }
            xs[tx][rr] = xv;
            // Y(k0 + rr, c0 + tx): kind 0 -> B_h(k, col); kind 1 -> W^T(k, col) = W(col, k)
            const int col = c0 + tx;
            double yv = 0.0;
            if (k < n && col < n)
                yv = (g.kind == 0) ? b_entry(phi, ivs, kappa, kappa + n, kappa + 2 * n, newton, k, col, n)
                                   : Yh[(size_t)k * n + col];
            ys[rr][tx] = yv;
        }
        __syncthreads();
#pragma unroll 8
        for (int kk = 0; kk < 32; kk++) {
            const double xv = xs[tx][kk];
#pragma unroll
            for (int q = 0; q < 4; q++) acc[q] += xv * ys[kk][ty + 8 * q];
        }
        __syncthreads();
    }
    const int r = r0 + tx;
    if (r >= n) return;
    double s = 1.0;
    if (g.kind == 0) s = newton ? g.ctrl->lrate : -g.ctrl->lrate;
    for (int q = 0; q < 4; q++) {
        const int col = c0 + ty + 8 * q;
        if (col >= n) continue;
        double* o = g.Out + g.strideOut * h + (size_t)col * n + r;
        if (g.kind == 0) *o = Xh[(size_t)col * n + r] + s * acc[q];
        else *o = acc[q];
    }
}

// Reparametrisation and c update after the A update (src/amica.cu:2367-2512):
// unit columns of A, mu *= norm, beta /= norm^2, mu -= W_old (cnew - c), c = cnew.
// One CTA of 1024 threads per model (n <= 256).
// With phi_split = 2, every CTA also reports ||A_new - A||_F / ||A||_F of its
// model (frozen models report nothing), and the last CTA to finish switches the
// split correction of phi on for good once a Newton iteration changed no
// model's A by more than phi_split_rel.
__global__ void __launch_bounds__(1024) k_reparm(int update_A, int do_reparm, double* A,
                                                 const double* __restrict__ Anew,
                                                 const double* __restrict__ W, double* c,
                                                 double* mu, double* beta,
                                                 const double* __restrict__ work,
                                                 const int* __restrict__ use_newton, int n, int m,
                                                 int phi_split, double phi_split_rel, Ctrl* ctrl) {
    const int h = blockIdx.x, tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    auto report = [&](double rel, bool frozen) {
        if (phi_split != 2 || tid != 0) return;
        if (!frozen) atomicMax((unsigned long long*)&ctrl->newton_rel_bits,
                               (unsigned long long)__double_as_longlong(rel));
        __threadfence();
        if (atomicAdd((unsigned long long*)&ctrl->reparm_done, 1ull) == (unsigned long long)(gridDim.x - 1)) {
            __threadfence();
            const double mx = __longlong_as_double((long long)atomicMax(
                (unsigned long long*)&ctrl->newton_rel_bits, 0ull));
            if (update_A && ctrl->newton && mx < phi_split_rel) ctrl->phi_split = 1;
        }
    };
    if (use_newton[h] < 0) {                          // frozen model: A, c, mu, beta unchanged
        report(0.0, true);
        return;
    }
    const double* cnew = work + (size_t)h * 4 * n + 3 * n;
    double* ch = c + (size_t)h * n;
    __shared__ double norms[kMaxN], shift[kMaxN], dc[kMaxN];
    __shared__ double red[2][32];
    double rel = 0.0;
    if (update_A) {
        double* Ah = A + (size_t)h * n * n;
        const double* An = Anew + (size_t)h * n * n;
        if (phi_split == 2) {
            double dd = 0.0, aa = 0.0;
            for (int e = tid; e < n * n; e += blockDim.x) {
                const double d = An[e] - Ah[e];
                dd += d * d;
                aa += Ah[e] * Ah[e];
            }
            for (int o = 16; o > 0; o >>= 1) {
                dd += __shfl_xor_sync(0xffffffffu, dd, o);
                aa += __shfl_xor_sync(0xffffffffu, aa, o);
            }
            if (lane == 0) { red[0][warp] = dd; red[1][warp] = aa; }
            __syncthreads();
            if (tid == 0) {
                double sd = 0.0, sa = 0.0;
                for (int w = 0; w < (int)(blockDim.x >> 5); w++) { sd += red[0][w]; sa += red[1][w]; }
                rel = sa > 0.0 ? sqrt(sd / sa) : 0.0;
            }
            __syncthreads();
        }
        if (do_reparm) {
            for (int cc = warp; cc < n; cc += 32) {
                double s = 0.0;
                for (int r = lane; r < n; r += 32) s += An[(size_t)cc * n + r] * An[(size_t)cc * n + r];
                for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
                if (lane == 0) norms[cc] = sqrt(s);
            }
            if (tid < n) dc[tid] = cnew[tid] - ch[tid];
            __syncthreads();
            for (int ib = 0; ib < n; ib += 128) {
                const int i = ib + (tid >> 3), part = tid & 7;
                const double* Wh = W + (size_t)h * n * n;
                double acc = 0.0;
                if (i < n)
                    for (int k = part; k < n; k += 8) acc += Wh[(size_t)k * n + i] * dc[k];
                acc += __shfl_xor_sync(0xffffffffu, acc, 1);
                acc += __shfl_xor_sync(0xffffffffu, acc, 2);
                acc += __shfl_xor_sync(0xffffffffu, acc, 4);
                if (part == 0 && i < n) shift[i] = acc;
            }
            __syncthreads();
            for (int cc = tid >> 7; cc < n; cc += 8)
                for (int r = tid & 127; r < n; r += 128)
                    Ah[(size_t)cc * n + r] = An[(size_t)cc * n + r] / norms[cc];
            for (int e = tid; e < m * n; e += blockDim.x) {
                const int i = e % n;
                const size_t idx = (size_t)h * m * n + e;
                double mv = mu[idx] * norms[i];
                beta[idx] /= (norms[i] * norms[i]);
                mu[idx] = mv - shift[i];
            }
        } else {
            for (int e = tid; e < n * n; e += blockDim.x) Ah[e] = An[e];
        }
        __syncthreads();
    }
    for (int i = tid; i < n; i += blockDim.x) ch[i] = cnew[i];   // src/amica.cu:2456-2462
    report(rel, false);
}

// ---------------------------------------------------------------------------
// k_reduce: raw[h][e] = sum over slots of partial[q][h][e], fixed order.  The
// n x n block is carried only by every psi_step-th slot (the tensor-core E-step
// keeps phi in one slot per cluster); when it already is phi it also goes
// straight into the statistics vector.  Replaces the block/device reductions of
// src/amica.cu:1618-1920.
__global__ void k_reduce(const double* __restrict__ partial, double* __restrict__ raw,
                         double* __restrict__ stats, int nslots, int M, int n, int m, int psi_step,
                         int psi_is_phi) {
    PartLayout PL{n, m};
    StatLayout SL{n, m};
    const int stride = PL.stride(), psi0 = PL.psi();
    const int64_t total = (int64_t)M * stride;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int h = (int)(e / stride);
        const int off = (int)(e - (int64_t)h * stride);
        const bool in_psi = off >= psi0;
        const int step = in_psi ? psi_step : 1;
        double s = 0.0;
#pragma unroll 4
        for (int q = 0; q < nslots; q += step) s += partial[(size_t)q * total + e];
        raw[e] = s;
        if (in_psi && psi_is_phi) stats[SL.base(h) + SL.phi() + (off - psi0)] = s;
    }
}

// ---------------------------------------------------------------------------
// k_finalize: raw per-model sums -> the flat statistics vector (oracle layout):
// phi = (Psi - gsum c^T) W^T, and the per-block factors of src/kernels.cu:616
// (kappa * beta), :745 (mu_denom * sqrt(beta)), :748-750 (rho * beta_denom).
__global__ void __launch_bounds__(kT) k_finalize(
    const double* __restrict__ raw, const double* __restrict__ W, const double* __restrict__ A,
    const double* __restrict__ c,
    const double* __restrict__ beta, const double* __restrict__ rho,
    const double* __restrict__ ltc64, const Ctrl* __restrict__ ctrl, double* __restrict__ stats,
    int n, int m, int psi_is_phi) {
    const int h = blockIdx.x, tid = threadIdx.x;
    PartLayout PL{n, m};
    StatLayout SL{n, m};
    const double* R = raw + (size_t)h * PL.stride();
    double* S = stats + SL.base(h);
    if (h == 0 && tid == 0) stats[0] = R[0] + (double)ctrl->nkeep * ltc64[0];
    if (tid == 0) S[SL.vs()] = R[1];
    const double* Ah = A + (size_t)h * n * n;
    for (int i = tid; i < n; i += kT) {
        // sum_t v x_i = (A sum_t v b)_i + vsum c_i, since x - c = A b
        double acc = R[1] * c[(size_t)h * n + i];
        for (int k = 0; k < n; k++) acc += Ah[(size_t)k * n + i] * R[PL.cn() + k];
        S[SL.cn() + i] = acc;
        S[SL.s2() + i] = R[PL.s2() + i];
    }
    for (int e = tid; e < m * n; e += kT) {
        const size_t idx = (size_t)h * m * n + e;
        const double bt = beta[idx], r = rho[idx];
        S[SL.mix(kUs) + e] = R[PL.mix(kUs) + e];
        S[SL.mix(kKn) + e] = R[PL.mix(kKn) + e] * bt;
        S[SL.mix(kLn) + e] = R[PL.mix(kLn) + e];
        S[SL.mix(kMn) + e] = R[PL.mix(kMn) + e];
        S[SL.mix(kMd) + e] = R[PL.mix(kMd) + e] * sqrt(bt);
        S[SL.mix(kBd) + e] = R[PL.mix(kBd) + e] * (r > 2.0 ? r : 1.0);
        S[SL.mix(kRn) + e] = R[PL.mix(kRn) + e];
    }
}

// ---------------------------------------------------------------------------
struct MCfg {
    int n, m, M;
    int do_newton, update_rho, rho_start_iter, newt_start_iter, maxdec;
    int update_gm, update_alpha, update_A, update_mu, update_beta, do_reparm;
    int do_reject, rejstart, rejint, maxrej;
    int phi_split;
    double lratemax, lnatrate, lratefact, rholrate, rhomin, rhomax, rejsig;
};

__device__ double psi_series(double x) {
    // digamma: psi(x) = psi(x+6) - sum_{k<6} 1/(x+k), asymptotic series at x+6
    // with the Bernoulli coefficients B_2k/(2k) up to x^-18 (the method of the
    // reference's psi(), src/kernels.cu:906-929)
    const double coef[9] = {1.0 / 12.0, -1.0 / 120.0, 1.0 / 252.0, -1.0 / 240.0, 1.0 / 132.0,
                            -691.0 / 32760.0, 1.0 / 12.0, -3617.0 / 8160.0, 43867.0 / 14364.0};
    const double s = x + 6.0;
    double r = log(s) - 1.0 / (2.0 * s);
    const double s2 = s * s;
    double p = s2;
    for (int k = 0; k < 9; k++) { r -= coef[k] / p; p *= s2; }
    for (int k = 5; k >= 0; k--) r -= 1.0 / (x + k);
    return r;
}

// Per-model parameter updates (src/amica.cu:1995-2154) and the Newton
// condition bflag (src/amica.cu:2155-2230).  One CTA of 1024 threads per model;
// kappa, lambda, sigma2 and cnew go to `work` for the A update.
constexpr int kMT = 1024;
__global__ void __launch_bounds__(kMT) k_mstep_params(
    MCfg cf, const double* __restrict__ stats, Ctrl* ctrl, double* gm, double* alpha, double* mu,
    double* beta, double* rho, double* work, int64_t* bflag, int* use_newton) {
    const int h = blockIdx.x, tid = threadIdx.x;
    const int n = cf.n, m = cf.m, mn = m * n;
    StatLayout SL{n, m};
    const double* S = stats + SL.base(h);
    const int64_t iter = ctrl->iter + 1;
    const double Tk = (double)ctrl->nkeep;
    double* kappa = work + (size_t)h * 4 * n;
    double* lambda = kappa + n;
    double* sig2 = kappa + 2 * n;
    double* cnew = kappa + 3 * n;
    __shared__ double sh[33];
    __shared__ double ks[kMaxN];
    const double vsum = S[SL.vs()];
    const double ivs = 1.0 / vsum;
    if (!(vsum >= kMinModelVsum)) {                   // a model that explains no data: frozen
        if (tid == 0) {
            if (cf.update_gm) gm[h] = fmax(vsum / Tk, kMinGm);
            bflag[h] = 0;
            use_newton[h] = -1;
        }
        return;
    }
    if (tid == 0 && cf.update_gm) gm[h] = vsum / Tk;
    if (tid == 0 && !cf.update_A) use_newton[h] = 0;
    // alpha = usum / vsum; then kappa / lambda with the new alpha and old mu
    for (int i = tid; i < n; i += kMT) {
        const double s2 = S[SL.s2() + i] * ivs;
        sig2[i] = s2;
        cnew[i] = S[SL.cn() + i] * ivs;
        double kap = 0.0, lam = 0.0;
        for (int j = 0; j < m; j++) {
            const int mi = j * n + i;
            const size_t idx = (size_t)h * mn + mi;
            const double us = S[SL.mix(kUs) + mi];
            if (cf.update_alpha) alpha[idx] = us * ivs;
            if (!(us > 0.0)) continue;                // a component with no responsibility
            const double dk = S[SL.mix(kKn) + mi] / us;
            const double a = alpha[idx];
            kap += dk * a;
            const double muv = mu[idx];
            lam += (muv * muv * dk + S[SL.mix(kLn) + mi] / us) * a;
        }
        kappa[i] = kap;
        lambda[i] = lam;
        ks[i] = kap * s2;
    }
    __syncthreads();
    for (int mi = tid; mi < mn; mi += kMT) {
        const size_t idx = (size_t)h * mn + mi;
        if (!(S[SL.mix(kUs) + mi] > 0.0)) continue;  // no responsibility: mu, beta, rho kept
        if (cf.update_mu) mu[idx] += S[SL.mix(kMn) + mi] / S[SL.mix(kMd) + mi];
        if (cf.update_beta) {
            const double bnum = (rho[idx] > 2.0) ? 0.0 : S[SL.mix(kUs) + mi];
            beta[idx] *= bnum / S[SL.mix(kBd) + mi];
        }
        if (cf.update_rho && iter >= cf.rho_start_iter) {
            double r = rho[idx];
            const double ps = psi_series(1.0 + 1.0 / r);
            const double d = 1.0 - (r / ps) * S[SL.mix(kRn) + mi] / S[SL.mix(kUs) + mi];
            r = r + cf.rholrate * d;
            if (r > cf.rhomax) r = cf.rhomax;
            else if (r < cf.rhomin) r = cf.rhomin;
            rho[idx] = r;
        }
    }
    if (!cf.update_A) return;
    // bflag: entries of (kappa sigma2)(kappa sigma2)^T that are <= 1, diagonal included
    double cnt = 0.0;
    for (int r = tid & 127; r < n; r += 128)
        for (int cc = tid >> 7; cc < n; cc += kMT / 128)
            if (ks[r] * ks[cc] <= 1.0) cnt += 1.0;
    cnt = block_sum(cnt, sh);
    const int64_t bf = (int64_t)cnt;
    const int newton = (bf == 0 && cf.do_newton && iter >= cf.newt_start_iter);
    if (tid == 0) { bflag[h] = bf; use_newton[h] = newton; }
}

// LL bookkeeping and the learning-rate schedule (src/amica.cu:1981-1993,
// :2281-2285).  One thread.
__global__ void k_ctrl(MCfg cf, const double* __restrict__ stats, Ctrl* ctrl,
                       const int64_t* __restrict__ bflag, IterRec* hist, int64_t hist_cap) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    Ctrl c = *ctrl;
    const int64_t iter = c.iter + 1;
    const double ll = stats[0] / ((double)cf.n * (double)c.nkeep);
    const double lrate_print = c.lrate;
    c.ll_decreased = 0;
    if (iter > 1 && ll < c.ll_prev) {
        c.lrate *= cf.lratefact;
        c.numdec += 1;
        c.ll_decreased = 1;
        if (c.numdec > cf.maxdec) {
            c.lratemax *= cf.lratefact;
            c.numdec = 0;
        }
    }
    c.ll = ll;
    c.ll_prev = ll;
    c.newton = 0;
    if (cf.update_A) {
        int no_newt = 0;
        for (int h = 0; h < cf.M; h++) no_newt |= (bflag[h] > 0);
        const double step = c.lrate < 0.1 ? c.lrate : 0.1;
        if (iter >= cf.newt_start_iter && cf.do_newton && !no_newt) {
            c.lrate = fmin(cf.lratemax, c.lrate + step);
            c.newton = 1;
        } else {
            c.lrate = fmin(cf.lnatrate, c.lrate + step);
        }
        c.no_newt = no_newt;
    }
    c.iter = iter;
    c.last_rejected = 0;
    // the A update of this iteration reports its relative change (k_reparm)
    c.newton_rel_bits = 0;
    c.reparm_done = 0;
    if (cf.phi_split != 2) c.phi_split = cf.phi_split;
    *ctrl = c;
    if (hist && iter - 1 < hist_cap) {
        IterRec r;
        r.ll = ll;
        r.lrate = lrate_print;
        r.iter = iter;
        r.newton = c.newton;
        r.ll_decreased = c.ll_decreased;
        r.nkeep = c.nkeep;
        r.nrejected = 0;
        r.phi_split = c.phi_split;          // the form this iteration's E-step ran
        hist[iter - 1] = r;
    }
}

// Rejection pass (engine-defined; the reference has none): over kept samples,
// mean and std (n-1) of P in FP64, 4096-sample chunks summed in order, then the
// chunk sums in order; drop kept samples with P < mean - rejsig * std.  Runs
// only on the iterations the schedule selects.  One CTA.
__global__ void __launch_bounds__(kT) k_reject(MCfg cf, Ctrl* ctrl, const float* __restrict__ P,
                                               uint8_t* keep, int64_t T, double* chunk,
                                               IterRec* hist, int64_t hist_cap, int force) {
    const int tid = threadIdx.x;
    __shared__ int run;
    __shared__ double mean_s, thr_s;
    __shared__ long long nk_s;
    if (tid == 0) {
        const Ctrl c = *ctrl;
        const int64_t it = c.iter;
        run = force || (cf.do_reject && c.rej_passes < cf.maxrej && it >= cf.rejstart &&
                        ((it - cf.rejstart) % (cf.rejint > 0 ? cf.rejint : 1)) == 0);
    }
    __syncthreads();
    if (!run) return;
    const int64_t CH = 4096;
    const int64_t nch = (T + CH - 1) / CH;
    long long* cnt = reinterpret_cast<long long*>(chunk + nch);
    for (int64_t q = tid; q < nch; q += kT) {
        double s = 0.0;
        long long k = 0;
        const int64_t e = (q + 1) * CH < T ? (q + 1) * CH : T;
        for (int64_t t = q * CH; t < e; t++)
            if (keep[t]) { s = __dadd_rn(s, (double)P[t]); k++; }
        chunk[q] = s;
        cnt[q] = k;
    }
    __syncthreads();
    if (tid == 0) {
        double s = 0.0;
        long long k = 0;
        for (int64_t q = 0; q < nch; q++) { s = __dadd_rn(s, chunk[q]); k += cnt[q]; }
        nk_s = k;
        mean_s = (k > 0) ? __ddiv_rn(s, (double)k) : 0.0;
    }
    __syncthreads();
    if (nk_s < 2) return;
    const double mean = mean_s;
    for (int64_t q = tid; q < nch; q += kT) {
        double s = 0.0;
        const int64_t e = (q + 1) * CH < T ? (q + 1) * CH : T;
        for (int64_t t = q * CH; t < e; t++)
            if (keep[t]) {
                const double d = __dsub_rn((double)P[t], mean);
                s = __dadd_rn(s, __dmul_rn(d, d));
            }
        chunk[q] = s;
    }
    __syncthreads();
    if (tid == 0) {
        double s = 0.0;
        for (int64_t q = 0; q < nch; q++) s = __dadd_rn(s, chunk[q]);
        const double sd = __dsqrt_rn(__ddiv_rn(s, (double)(nk_s - 1)));
        thr_s = __dsub_rn(mean, __dmul_rn(cf.rejsig, sd));
        ctrl->rej_mean = mean;
        ctrl->rej_std = sd;
    }
    __syncthreads();
    const double thr = thr_s;
    long long dropped = 0;
    for (int64_t t = tid; t < T; t += kT)
        if (keep[t] && (double)P[t] < thr) { keep[t] = 0; dropped++; }
    __shared__ double shd[33];
    const double dd = block_sum((double)dropped, shd);
    if (tid == 0) {
        const int64_t d = (int64_t)dd;
        ctrl->nkeep -= d;
        ctrl->nrej_total += d;
        ctrl->rej_passes += 1;
        ctrl->last_rejected = d;
        const int64_t it = ctrl->iter;
        if (hist && it >= 1 && it - 1 < hist_cap) hist[it - 1].nrejected = d;
    }
}

}  // namespace

namespace amica {



static MCfg to_mcfg(const MStepCfgHost& h) {
    MCfg c;
    c.n = h.n; c.m = h.m; c.M = h.M;
    c.do_newton = h.do_newton; c.update_rho = h.update_rho; c.rho_start_iter = h.rho_start_iter;
    c.newt_start_iter = h.newt_start_iter; c.maxdec = h.maxdec; c.update_gm = h.update_gm;
    c.update_alpha = h.update_alpha; c.update_A = h.update_A; c.update_mu = h.update_mu;
    c.update_beta = h.update_beta; c.do_reparm = h.do_reparm; c.do_reject = h.do_reject;
    c.rejstart = h.rejstart; c.rejint = h.rejint; c.maxrej = h.maxrej; c.phi_split = h.phi_split;
    c.lratemax = h.lratemax; c.lnatrate = h.lnatrate; c.lratefact = h.lratefact;
    c.rholrate = h.rholrate; c.rhomin = h.rhomin; c.rhomax = h.rhomax; c.rejsig = h.rejsig;
    return c;
}

cudaError_t launch_prep(const MStepBuffers& b, const MStepCfgHost& h, cudaStream_t st) {
    if (h.n > kMaxN) return cudaErrorInvalidValue;
    if (h.n > 128) {
        if (!b.gj) return cudaErrorInvalidValue;
        double* pivlog = b.gj + (size_t)h.M * h.n * h.n;
        cudaError_t e = cudaFuncSetAttribute(k_inverse_big, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)kBigSmem);
        if (e != cudaSuccess) return e;
        k_inverse_big<<<h.M, kInvThreads, kBigSmem, st>>>(b.A, b.gj, b.W, pivlog, h.n, b.err);
        k_derive<<<h.M, 256, 0, st>>>(b.W, pivlog, b.c, b.alpha, b.mu, b.beta, b.rho, b.gm, h.ldetS,
                                      b.ldet, b.ltc64, b.Wf, b.wcf, b.mp, h.n, h.m, h.NP);
        return cudaGetLastError();
    }
    if (h.NP > 128 || kInvThreads % h.NP || h.m > kMaxMix) return cudaErrorInvalidValue;
    cudaError_t e = cudaFuncSetAttribute(k_inverse_derive, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)kInvSmem);
    if (e != cudaSuccess) return e;
    k_inverse_derive<<<h.M, kInvThreads, kInvSmem, st>>>(b.A, b.c, b.alpha, b.mu, b.beta, b.rho, b.gm,
                                                     h.ldetS, b.W, b.ldet, b.ltc64, b.Wf, b.wcf, b.mp,
                                                     h.n, h.m, h.NP, b.err);
    return cudaGetLastError();
}

cudaError_t launch_reduce_finalize(const MStepBuffers& b, const MStepCfgHost& h, int nclusters,
                                   cudaStream_t st) {
    PartLayout PL{h.n, h.m};
    StatLayout SL{h.n, h.m};
    const int64_t total = (int64_t)h.M * PL.stride();
    int grid = (int)((total + 255) / 256);
    if (grid > 4096) grid = 4096;
    k_reduce<<<grid, 256, 0, st>>>(b.partial, b.raw, b.stats, nclusters, h.M, h.n, h.m,
                                   h.psi_step > 0 ? h.psi_step : 1, h.psi_is_phi);
    k_finalize<<<h.M, kT, 0, st>>>(b.raw, b.W, b.A, b.c, b.beta, b.rho, b.ltc64, b.ctrl, b.stats,
                                   h.n, h.m, h.psi_is_phi);
    if (!h.psi_is_phi) {
        dim3 g((h.n + 31) / 32, (h.n + 31) / 32, h.M);
        GemmArgs ga{};
        ga.kind = 1; ga.n = h.n; ga.m = h.m;
        ga.X = b.raw + PL.psi(); ga.strideX = PL.stride();
        ga.Y = b.W; ga.strideY = (size_t)h.n * h.n;
        ga.Out = b.stats + SL.base(0) + SL.phi(); ga.strideOut = SL.S();
        ga.gs = b.raw + PL.gs(); ga.strideG = PL.stride();
        ga.c = b.c;
        k_gemm64<<<g, 256, 0, st>>>(ga);
    }
    return cudaGetLastError();
}

// Flags a non-finite parameter after the M-step, so that the host rolls the
// iteration back (the next E-step would otherwise carry NaN into the LL).
__global__ void k_check_finite(const double* __restrict__ A, const double* __restrict__ c,
                               const double* __restrict__ alpha, const double* __restrict__ mu,
                               const double* __restrict__ beta, const double* __restrict__ rho,
                               const double* __restrict__ gm, int64_t nA, int64_t nc, int64_t nmix,
                               int M, int* err) {
    bool bad = false;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int64_t t0 = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    for (int64_t e = t0; e < nA; e += stride) bad |= !isfinite(A[e]);
    for (int64_t e = t0; e < nc; e += stride) bad |= !isfinite(c[e]);
    for (int64_t e = t0; e < nmix; e += stride)
        bad |= !isfinite(alpha[e]) || !isfinite(mu[e]) || !isfinite(beta[e]) || !isfinite(rho[e]);
    for (int64_t e = t0; e < M; e += stride) bad |= !isfinite(gm[e]);
    if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(err, kErrNonFinite);
}

cudaError_t launch_mstep(const MStepBuffers& b, const MStepCfgHost& h, const float* P_rel,
                         uint8_t* keep, int64_t T, cudaStream_t st) {
    const MCfg cf = to_mcfg(h);
    k_mstep_params<<<h.M, kMT, 0, st>>>(cf, b.stats, b.ctrl, b.gm, b.alpha, b.mu, b.beta, b.rho,
                                        b.work, b.bflag, b.use_newton);
    k_ctrl<<<1, 32, 0, st>>>(cf, b.stats, b.ctrl, b.bflag, b.hist, b.hist_cap);
    if (h.update_A) {
        dim3 g((h.n + 31) / 32, (h.n + 31) / 32, h.M);
        GemmArgs ga{};
        ga.kind = 0; ga.n = h.n; ga.m = h.m;
        ga.X = b.A; ga.strideX = (size_t)h.n * h.n;
        ga.Out = b.Anew; ga.strideOut = (size_t)h.n * h.n;
        ga.use_newton = b.use_newton; ga.ctrl = b.ctrl;
        ga.stats = b.stats; ga.work = b.work;
        k_gemm64<<<g, 256, 0, st>>>(ga);
    }
    k_reparm<<<h.M, 1024, 0, st>>>(h.update_A, h.do_reparm, b.A, b.Anew, b.W, b.c, b.mu, b.beta,
                                  b.work, b.use_newton, h.n, h.m, h.phi_split, h.phi_split_rel, b.ctrl);
    {
        const int64_t nA = (int64_t)h.M * h.n * h.n, nmix = (int64_t)h.M * h.m * h.n;
        const int grid = (int)std::min<int64_t>((nA + 255) / 256, 148);
        k_check_finite<<<grid, 256, 0, st>>>(b.A, b.c, b.alpha, b.mu, b.beta, b.rho, b.gm, nA,
                                             (int64_t)h.M * h.n, nmix, h.M, b.err);
    }
    if (h.do_reject && P_rel && keep)
        k_reject<<<1, kT, 0, st>>>(cf, b.ctrl, P_rel, keep, T, b.chunk, b.hist, b.hist_cap, 0);
    return cudaGetLastError();
}

cudaError_t launch_reject_now(const MStepBuffers& b, const MStepCfgHost& h, const float* P_rel,
                              uint8_t* keep, int64_t T, cudaStream_t st) {
    const MCfg cf = to_mcfg(h);
    k_reject<<<1, kT, 0, st>>>(cf, b.ctrl, P_rel, keep, T, b.chunk, b.hist, b.hist_cap, 1);
    return cudaGetLastError();
}

}  // namespace amica
