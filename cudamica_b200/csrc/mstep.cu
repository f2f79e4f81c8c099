// FP64 device-side M-step of the AMICA EM iteration, plus the per-iteration
// preparation of the E-step constants and the deterministic reduction of the
// E-step's per-CTA partial sums.
//
// The reference runs this part as ~40 small FP64 kernels, cuBLAS/MAGMA calls
// and host round trips per iteration (src/amica.cu:835-924 and :1981-2512:
// host SVD for pinv, a synchronous bflag copy, ...).  Here it is six small
// kernels that stay on the device, so that a whole iteration can be captured
// in one CUDA graph and no host synchronisation is needed between iterations.
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
// k_prep: W_h = A_h^{-1} (Gauss-Jordan, partial pivoting), ldet_h = -log|det A_h|
// and the FP32 constants of the E-step.  One CTA per model.
// Replaces pinv() + the ldet computation (src/amica.cu:27-127, :835-924).
__global__ void __launch_bounds__(kT) k_prep(
    const double* __restrict__ A, const double* __restrict__ c, const double* __restrict__ alpha,
    const double* __restrict__ mu, const double* __restrict__ beta, const double* __restrict__ rho,
    const double* __restrict__ gm, double ldetS, double* __restrict__ aug, double* __restrict__ W,
    double* __restrict__ ldet, double* __restrict__ ltc64, float* __restrict__ Wf,
    float* __restrict__ wcf, MixParam* __restrict__ mp, int n, int m, int NP, int* err) {
    const int h = blockIdx.x, tid = threadIdx.x;
    const int n2 = 2 * n;
    double* a = aug + (size_t)h * n * n2;              // row-major [r][c], c < 2n
    const double* Ah = A + (size_t)h * n * n;          // column-major
    __shared__ double fcol[256];
    __shared__ double sh[33];
    __shared__ int piv_s;
    __shared__ double pv_s;
    for (int e = tid; e < n * n2; e += kT) {
        const int r = e / n2, cc = e % n2;
        a[e] = (cc < n) ? Ah[(size_t)cc * n + r] : ((cc - n) == r ? 1.0 : 0.0);
    }
    __syncthreads();
    double logdet = 0.0;
    bool singular = false;
    for (int k = 0; k < n; k++) {
        // pivot: argmax_{r >= k} |a(r,k)| (lowest index on ties)
        double best = -1.0;
        int bi = k;
        for (int r = k + tid; r < n; r += kT) {
            const double v = fabs(a[(size_t)r * n2 + k]);
            if (v > best) { best = v; bi = r; }
        }
        for (int o = 16; o > 0; o >>= 1) {
            const double ov = __shfl_xor_sync(0xffffffffu, best, o);
            const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
            if (ov > best || (ov == best && oi < bi)) { best = ov; bi = oi; }
        }
        __shared__ double wb[8];
        __shared__ int wi[8];
        if (tid % 32 == 0) { wb[tid / 32] = best; wi[tid / 32] = bi; }
        __syncthreads();
        if (tid == 0) {
            double b = wb[0];
            int i = wi[0];
            for (int w = 1; w < kT / 32; w++)
                if (wb[w] > b || (wb[w] == b && wi[w] < i)) { b = wb[w]; i = wi[w]; }
            piv_s = i;
        }
        __syncthreads();
        const int p = piv_s;
        if (p != k)
            for (int cc = tid; cc < n2; cc += kT) {
                const double t = a[(size_t)k * n2 + cc];
                a[(size_t)k * n2 + cc] = a[(size_t)p * n2 + cc];
                a[(size_t)p * n2 + cc] = t;
            }
        __syncthreads();
        if (tid == 0) pv_s = a[(size_t)k * n2 + k];
        __syncthreads();
        const double pv = pv_s;
        if (pv == 0.0) { singular = true; break; }
        logdet += log(fabs(pv));
        const double inv = 1.0 / pv;
        for (int cc = tid; cc < n2; cc += kT) a[(size_t)k * n2 + cc] *= inv;
        for (int r = tid; r < n; r += kT) fcol[r] = a[(size_t)r * n2 + k];
        __syncthreads();
        for (int e = tid; e < n * n2; e += kT) {
            const int r = e / n2, cc = e % n2;
            if (r != k) a[e] -= fcol[r] * a[(size_t)k * n2 + cc];
        }
        __syncthreads();
    }
    if (singular) {
        if (tid == 0) atomicOr(err, kErrSingular);
        return;
    }
    double* Wh = W + (size_t)h * n * n;
    for (int e = tid; e < n * n; e += kT) {
        const int r = e % n, cc = e / n;
        Wh[e] = a[(size_t)r * n2 + n + cc];             // column-major W(r, cc)
    }
    if (tid == 0) {
        ldet[h] = -logdet;
        ltc64[h] = log(gm[h]) - logdet + ldetS;         // src/amica.cu:1009
    }
    __syncthreads();
    // FP32 copies for the E-step
    float* Wfh = Wf + (size_t)h * NP * NP;
    for (int e = tid; e < NP * NP; e += kT) {
        const int i = e / NP, k = e % NP;
        Wfh[e] = (i < n && k < n) ? (float)Wh[(size_t)k * n + i] : 0.f;
    }
    for (int i = tid; i < NP; i += kT) {
        double wc = 0.0;
        if (i < n)
            for (int k = 0; k < n; k++) wc += Wh[(size_t)k * n + i] * c[(size_t)h * n + k];
        wcf[(size_t)h * NP + i] = (float)wc;
        for (int j = 0; j < m; j++) {
            MixParam q;
            if (i < n) {
                const size_t idx = ((size_t)h * m + j) * n + i;
                const double s = sqrt(beta[idx]);
                const double r = rho[idx];
                q.s = (float)s;
                q.off = (float)(s * (mu[idx] + wc));
                q.cl2 = (float)((log(alpha[idx]) + 0.5 * log(beta[idx]) - M_LN2 - lgamma(1.0 + 1.0 / r)) *
                                1.4426950408889634);
                q.rho = (float)r;
            } else {
                q.s = 0.f; q.off = 0.f; q.cl2 = 0.f; q.rho = 1.f;
            }
            mp[((size_t)h * m + j) * NP + i] = q;
        }
    }
}

// ---------------------------------------------------------------------------
// k_inverse_smem: W_h = A_h^{-1} by in-place Gauss-Jordan with partial pivoting,
// the whole n x n FP64 matrix resident in shared memory (n <= 128), one CTA of
// 1024 threads per model; ldet_h = -sum log|pivot|.  Replaces pinv() and the
// LU log-determinant (src/amica.cu:27-127, :864-924).
__global__ void __launch_bounds__(1024) k_inverse_smem(const double* __restrict__ A,
                                                       const double* __restrict__ gm, double ldetS,
                                                       double* __restrict__ W,
                                                       double* __restrict__ ldet,
                                                       double* __restrict__ ltc64, int n, int* err) {
    extern __shared__ double gj[];                       // [n][n] row-major, then fcol[n]
    double* fcol = gj + n * n;
    __shared__ int perm[128];
    __shared__ double wb[32];
    __shared__ int wi[32];
    __shared__ double piv_s, logdet_s;
    __shared__ int p_s, bad_s;
    const int h = blockIdx.x, tid = threadIdx.x, nt = blockDim.x;
    const double* Ah = A + (size_t)h * n * n;
    for (int e = tid; e < n * n; e += nt) {
        const int r = e / n, c = e % n;
        gj[e] = Ah[(size_t)c * n + r];
    }
    if (tid == 0) { logdet_s = 0.0; bad_s = 0; }
    __syncthreads();
    for (int k = 0; k < n; k++) {
        // pivot row: argmax_{r >= k} |a(r,k)|, lowest index on ties
        double best = -1.0;
        int bi = k;
        for (int r = k + tid; r < n; r += nt) {
            const double v = fabs(gj[r * n + k]);
            if (v > best) { best = v; bi = r; }
        }
        for (int o = 16; o > 0; o >>= 1) {
            const double ov = __shfl_xor_sync(0xffffffffu, best, o);
            const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
            if (ov > best || (ov == best && oi < bi)) { best = ov; bi = oi; }
        }
        if ((tid & 31) == 0) { wb[tid >> 5] = best; wi[tid >> 5] = bi; }
        __syncthreads();
        if (tid == 0) {
            double b = wb[0];
            int i = wi[0];
            for (int w = 1; w < nt / 32; w++)
                if (wb[w] > b || (wb[w] == b && wi[w] < i)) { b = wb[w]; i = wi[w]; }
            p_s = i;
            perm[k] = i;
        }
        __syncthreads();
        const int p = p_s;
        if (p != k)
            for (int c = tid; c < n; c += nt) {
                const double t = gj[k * n + c];
                gj[k * n + c] = gj[p * n + c];
                gj[p * n + c] = t;
            }
        __syncthreads();
        if (tid == 0) {
            piv_s = gj[k * n + k];
            if (piv_s == 0.0) bad_s = 1;
            else logdet_s += log(fabs(piv_s));
        }
        for (int r = tid; r < n; r += nt) fcol[r] = gj[r * n + k];
        __syncthreads();
        if (bad_s) break;
        const double inv = 1.0 / piv_s;
        for (int c = tid; c < n; c += nt) gj[k * n + c] = (c == k ? 1.0 : gj[k * n + c]) * inv;
        __syncthreads();
        for (int e = tid; e < n * n; e += nt) {
            const int r = e / n, c = e % n;
            if (r != k) gj[e] = (c == k ? 0.0 : gj[e]) - fcol[r] * gj[k * n + c];
        }
        __syncthreads();
    }
    if (bad_s) {
        if (tid == 0) atomicOr(err, kErrSingular);
        return;
    }
    // undo the row interchanges as column interchanges, last first
    for (int k = n - 1; k >= 0; k--) {
        const int p = perm[k];
        if (p != k)
            for (int r = tid; r < n; r += nt) {
                const double t = gj[r * n + k];
                gj[r * n + k] = gj[r * n + p];
                gj[r * n + p] = t;
            }
        __syncthreads();
    }
    double* Wh = W + (size_t)h * n * n;
    for (int e = tid; e < n * n; e += nt) {
        const int r = e % n, c = e / n;
        Wh[e] = gj[r * n + c];                          // column-major W(r, c)
    }
    if (tid == 0) {
        ldet[h] = -logdet_s;
        ltc64[h] = log(gm[h]) - logdet_s + ldetS;       // src/amica.cu:1009
    }
}

// FP32 E-step constants from W and the parameters (grid: models x channel blocks).
__global__ void __launch_bounds__(128) k_derive(
    const double* __restrict__ W, const double* __restrict__ c, const double* __restrict__ alpha,
    const double* __restrict__ mu, const double* __restrict__ beta, const double* __restrict__ rho,
    float* __restrict__ Wf, float* __restrict__ wcf, MixParam* __restrict__ mp, int n, int m,
    int NP) {
    const int h = blockIdx.x;
    const int i = blockIdx.y * blockDim.x + threadIdx.x;   // channel
    if (i >= NP) return;
    const double* Wh = W + (size_t)h * n * n;
    float* Wfh = Wf + (size_t)h * NP * NP;
    for (int k = 0; k < NP; k++) Wfh[(size_t)i * NP + k] = (i < n && k < n) ? (float)Wh[(size_t)k * n + i] : 0.f;
    double wc = 0.0;
    if (i < n)
        for (int k = 0; k < n; k++) wc += Wh[(size_t)k * n + i] * c[(size_t)h * n + k];
    wcf[(size_t)h * NP + i] = (float)wc;
    for (int j = 0; j < m; j++) {
        MixParam q;
        if (i < n) {
            const size_t idx = ((size_t)h * m + j) * n + i;
            const double s = sqrt(beta[idx]);
            const double r = rho[idx];
            q.s = (float)s;
            q.off = (float)(s * (mu[idx] + wc));
            q.cl2 = (float)((log(alpha[idx]) + 0.5 * log(beta[idx]) - M_LN2 - lgamma(1.0 + 1.0 / r)) *
                            1.4426950408889634);
            q.rho = (float)r;
        } else {
            q.s = 0.f; q.off = 0.f; q.cl2 = 0.f; q.rho = 1.f;
        }
        mp[((size_t)h * m + j) * NP + i] = q;
    }
}

// Batched FP64 32x32-tiled products on n x n column-major matrices, one
// (tile, model) per CTA of 256 threads:
//   kind 0 (A update, src/amica.cu:2330-2342):  Out = X + s_h X Y,
//          s_h = +lrate (Newton) or -lrate (natural gradient)
//   kind 1 (phi from Psi):  Out = (Psi - gsum c^T) W^T, written into the
//          statistics vector's phi block
__global__ void __launch_bounds__(256) k_gemm64(int kind, const double* __restrict__ X,
                                                size_t strideX, const double* __restrict__ Y,
                                                size_t strideY, double* __restrict__ Out,
                                                size_t strideOut, const double* __restrict__ gs,
                                                size_t strideG, const double* __restrict__ c,
                                                const int* __restrict__ use_newton,
                                                const Ctrl* __restrict__ ctrl, int n) {
    __shared__ double xs[32][33], ys[32][33];
    const int h = blockIdx.z;
    const int r0 = blockIdx.x * 32, c0 = blockIdx.y * 32;
    const int tx = threadIdx.x % 32, ty = threadIdx.x / 32;   // ty: 0..7
    const double* Xh = X + strideX * h;
    const double* Yh = Y + strideY * h;
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    for (int k0 = 0; k0 < n; k0 += 32) {
        for (int q = 0; q < 4; q++) {
            const int rr = ty + 8 * q;                 // tile-local k (for X) / k (for Y)
            // X(r0 + tx, k0 + rr)
            const int r = r0 + tx, k = k0 + rr;
            double xv = 0.0;
            if (r < n && k < n) {
                xv = Xh[(size_t)k * n + r];
                if (kind == 1) xv -= gs[strideG * h + r] * c[(size_t)h * n + k];
            }
            xs[tx][rr] = xv;
            // Y(k0 + rr, c0 + tx): kind 0 -> Y col-major; kind 1 -> W^T(k, col) = W(col, k)
            const int col = c0 + tx;
            double yv = 0.0;
            if (k < n && col < n) yv = (kind == 0) ? Yh[(size_t)col * n + k] : Yh[(size_t)k * n + col];
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
    if (kind == 0) s = use_newton[h] ? ctrl->lrate : -ctrl->lrate;
    for (int q = 0; q < 4; q++) {
        const int col = c0 + ty + 8 * q;
        if (col >= n) continue;
        double* o = Out + strideOut * h + (size_t)col * n + r;
        if (kind == 0) *o = Xh[(size_t)col * n + r] + s * acc[q];
        else *o = acc[q];
    }
}

// Reparametrisation and c update after the A update (src/amica.cu:2367-2512):
// unit columns of A, mu *= norm, beta /= norm^2, mu -= W_old (cnew - c), c = cnew.
__global__ void __launch_bounds__(256) k_reparm(int update_A, int do_reparm, double* A,
                                                const double* __restrict__ Anew,
                                                const double* __restrict__ W, double* c,
                                                double* mu, double* beta,
                                                const double* __restrict__ work, int n, int m) {
    const int h = blockIdx.x, tid = threadIdx.x;
    const double* cnew = work + (size_t)h * 4 * n + 3 * n;
    double* ch = c + (size_t)h * n;
    __shared__ double norms[256];
    __shared__ double shift[256];
    if (update_A) {
        double* Ah = A + (size_t)h * n * n;
        const double* An = Anew + (size_t)h * n * n;
        if (do_reparm) {
            for (int cc = tid; cc < n; cc += blockDim.x) {
                double s = 0.0;
                for (int r = 0; r < n; r++) s += An[(size_t)cc * n + r] * An[(size_t)cc * n + r];
                norms[cc] = sqrt(s);
            }
            const double* Wh = W + (size_t)h * n * n;
            for (int i = tid; i < n; i += blockDim.x) {
                double acc = 0.0;
                for (int k = 0; k < n; k++) acc += Wh[(size_t)k * n + i] * (cnew[k] - ch[k]);
                shift[i] = acc;
            }
            __syncthreads();
            for (int e = tid; e < n * n; e += blockDim.x) Ah[e] = An[e] / norms[e / n];
            for (int e = tid; e < m * n; e += blockDim.x) {
                const int i = e % n;
                const size_t idx = (size_t)h * m * n + e;
                mu[idx] *= norms[i];
                beta[idx] /= (norms[i] * norms[i]);
                mu[idx] -= shift[i];
            }
        } else {
            for (int e = tid; e < n * n; e += blockDim.x) Ah[e] = An[e];
        }
        __syncthreads();
    }
    for (int i = tid; i < n; i += blockDim.x) ch[i] = cnew[i];   // src/amica.cu:2456-2462
}

// ---------------------------------------------------------------------------
// k_reduce: raw[h][e] = sum over clusters of partial[q][h][e], fixed order.
// Replaces the block/device reductions of src/amica.cu:1618-1920.
__global__ void k_reduce(const double* __restrict__ partial, double* __restrict__ raw, int nclusters,
                         int M, int stride) {
    const int64_t total = (int64_t)M * stride;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total;
         e += (int64_t)gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int q = 0; q < nclusters; q++) s += partial[(size_t)q * total + e];
        raw[e] = s;
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
    const double* Psi = R + PL.psi();
    const double* gs = R + PL.gs();
    const double* Wh = W + (size_t)h * n * n;
    const double* ch = c + (size_t)h * n;
    for (int e = tid; e < n * n; e += kT) {
        const int i = e % n, k = e / n;
        if (psi_is_phi) S[SL.phi() + (size_t)k * n + i] = Psi[e];
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

// Per-model parameter updates (src/amica.cu:1995-2154) and the Newton /
// natural-gradient matrix B (src/amica.cu:2155-2279, src/kernels.cu:961-1014).
__global__ void __launch_bounds__(kT) k_mstep_params(
    MCfg cf, const double* __restrict__ stats, Ctrl* ctrl, double* gm, double* alpha, double* mu,
    double* beta, double* rho, double* work, double* B, int64_t* bflag, int* use_newton) {
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
    const double vsum = S[SL.vs()];
    const double ivs = 1.0 / vsum;
    if (tid == 0 && cf.update_gm) gm[h] = vsum / Tk;
    for (int i = tid; i < n; i += kT) {
        sig2[i] = S[SL.s2() + i] * ivs;
        cnew[i] = S[SL.cn() + i] * ivs;
    }
    // alpha = usum / vsum; then kappa / lambda with the new alpha and old mu
    for (int i = tid; i < n; i += kT) {
        double kap = 0.0, lam = 0.0;
        for (int j = 0; j < m; j++) {
            const int mi = j * n + i;
            const size_t idx = (size_t)h * mn + mi;
            const double us = S[SL.mix(kUs) + mi];
            if (cf.update_alpha) alpha[idx] = us * ivs;
            const double dk = S[SL.mix(kKn) + mi] / us;
            const double a = alpha[idx];
            kap += dk * a;
            const double muv = mu[idx];
            lam += (muv * muv * dk + S[SL.mix(kLn) + mi] / us) * a;
        }
        kappa[i] = kap;
        lambda[i] = lam;
    }
    __syncthreads();
    for (int mi = tid; mi < mn; mi += kT) {
        const size_t idx = (size_t)h * mn + mi;
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
    for (int e = tid; e < n * n; e += kT) {
        const int r = e % n, cc = e / n;
        const double d = (kappa[r] * sig2[r]) * (kappa[cc] * sig2[cc]);
        if (d <= 1.0) cnt += 1.0;
    }
    cnt = block_sum(cnt, sh);
    const int64_t bf = (int64_t)cnt;
    const int newton = (bf == 0 && cf.do_newton && iter >= cf.newt_start_iter);
    if (tid == 0) { bflag[h] = bf; use_newton[h] = newton; }
    const double* phi = S + SL.phi();
    double* Bh = B + (size_t)h * n * n;
    for (int e = tid; e < n * n; e += kT) {
        const int r = e % n, cc = e / n;
        const double prc = phi[(size_t)cc * n + r] * ivs;      // phi(r, c) / vsum
        double v;
        if (newton) {
            if (r == cc) {
                v = (1.0 - prc) / lambda[r];
            } else {
                const double pcr = phi[(size_t)r * n + cc] * ivs;
                const double nom = -sig2[r] * kappa[cc];
                v = (nom * (-prc) + (-pcr)) / ((kappa[r] * sig2[r]) * (kappa[cc] * sig2[cc]) - 1.0);
            }
        } else {
            v = (r == cc ? 1.0 : 0.0) - prc;
        }
        Bh[e] = v;
    }
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
        r.pad = 0;
        hist[iter - 1] = r;
    }
}

// A update and reparametrisation (src/amica.cu:2288-2447, src/kernels.cu:1023-1065).
__global__ void __launch_bounds__(kT) k_mstep_A(MCfg cf, const Ctrl* __restrict__ ctrl, double* A,
                                                double* Anew, const double* __restrict__ B,
                                                const int* __restrict__ use_newton,
                                                const double* __restrict__ W, double* c, double* mu,
                                                double* beta, const double* __restrict__ work) {
    const int h = blockIdx.x, tid = threadIdx.x;
    const int n = cf.n, m = cf.m;
    const double* cnew = work + (size_t)h * 4 * n + 3 * n;
    double* ch = c + (size_t)h * n;
    __shared__ double norms[256];
    __shared__ double shift[256];
    if (cf.update_A) {
        double* Ah = A + (size_t)h * n * n;
        double* An = Anew + (size_t)h * n * n;
        const double* Bh = B + (size_t)h * n * n;
        const double al = use_newton[h] ? ctrl->lrate : -ctrl->lrate;
        for (int e = tid; e < n * n; e += kT) {
            const int r = e % n, cc = e / n;
            double acc = 0.0;
            for (int k = 0; k < n; k++) acc += Ah[(size_t)k * n + r] * Bh[(size_t)cc * n + k];
            An[e] = al * acc + Ah[e];
        }
        __syncthreads();
        if (cf.do_reparm) {
            for (int cc = tid; cc < n; cc += kT) {
                double s = 0.0;
                for (int r = 0; r < n; r++) s += An[(size_t)cc * n + r] * An[(size_t)cc * n + r];
                norms[cc] = sqrt(s);
            }
            // W (cnew - c) with the W of the start of the iteration
            const double* Wh = W + (size_t)h * n * n;
            for (int i = tid; i < n; i += kT) {
                double acc = 0.0;
                for (int k = 0; k < n; k++) acc += Wh[(size_t)k * n + i] * (cnew[k] - ch[k]);
                shift[i] = acc;
            }
            __syncthreads();
            for (int e = tid; e < n * n; e += kT) Ah[e] = An[e] / norms[e / n];
            for (int e = tid; e < m * n; e += kT) {
                const int i = e % n;
                const size_t idx = (size_t)h * m * n + e;
                mu[idx] *= norms[i];
                beta[idx] /= (norms[i] * norms[i]);
                mu[idx] -= shift[i];
            }
        } else {
            for (int e = tid; e < n * n; e += kT) Ah[e] = An[e];
        }
        __syncthreads();
    }
    for (int i = tid; i < n; i += kT) ch[i] = cnew[i];   // src/amica.cu:2456-2462
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
    c.rejstart = h.rejstart; c.rejint = h.rejint; c.maxrej = h.maxrej;
    c.lratemax = h.lratemax; c.lnatrate = h.lnatrate; c.lratefact = h.lratefact;
    c.rholrate = h.rholrate; c.rhomin = h.rhomin; c.rhomax = h.rhomax; c.rejsig = h.rejsig;
    return c;
}

cudaError_t launch_prep(const MStepBuffers& b, const MStepCfgHost& h, cudaStream_t st) {
    if (h.n <= 128) {
        const size_t smem = sizeof(double) * ((size_t)h.n * h.n + h.n);
        cudaError_t e = cudaFuncSetAttribute(k_inverse_smem, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)smem);
        if (e != cudaSuccess) return e;
        k_inverse_smem<<<h.M, 1024, smem, st>>>(b.A, b.gm, h.ldetS, b.W, b.ldet, b.ltc64, h.n, b.err);
        dim3 grid(h.M, (h.NP + 127) / 128);
        k_derive<<<grid, 128, 0, st>>>(b.W, b.c, b.alpha, b.mu, b.beta, b.rho, b.Wf, b.wcf, b.mp, h.n,
                                       h.m, h.NP);
    } else {
        k_prep<<<h.M, kT, 0, st>>>(b.A, b.c, b.alpha, b.mu, b.beta, b.rho, b.gm, h.ldetS, b.aug, b.W,
                                   b.ldet, b.ltc64, b.Wf, b.wcf, b.mp, h.n, h.m, h.NP, b.err);
    }
    return cudaGetLastError();
}

cudaError_t launch_reduce_finalize(const MStepBuffers& b, const MStepCfgHost& h, int nclusters,
                                   cudaStream_t st) {
    PartLayout PL{h.n, h.m};
    StatLayout SL{h.n, h.m};
    const int64_t total = (int64_t)h.M * PL.stride();
    int grid = (int)((total + 255) / 256);
    if (grid > 4096) grid = 4096;
    k_reduce<<<grid, 256, 0, st>>>(b.partial, b.raw, nclusters, h.M, PL.stride());
    k_finalize<<<h.M, kT, 0, st>>>(b.raw, b.W, b.A, b.c, b.beta, b.rho, b.ltc64, b.ctrl, b.stats,
                                   h.n, h.m, h.psi_is_phi);
    if (!h.psi_is_phi) {
        dim3 g((h.n + 31) / 32, (h.n + 31) / 32, h.M);
        k_gemm64<<<g, 256, 0, st>>>(1, b.raw + PL.psi(), PL.stride(), b.W, (size_t)h.n * h.n,
                                    b.stats + SL.base(0) + SL.phi(), SL.S(), b.raw + PL.gs(),
                                    PL.stride(), b.c, nullptr, nullptr, h.n);
    }
    return cudaGetLastError();
}

cudaError_t launch_mstep(const MStepBuffers& b, const MStepCfgHost& h, const float* P_rel,
                         uint8_t* keep, int64_t T, cudaStream_t st) {
    const MCfg cf = to_mcfg(h);
    k_mstep_params<<<h.M, kT, 0, st>>>(cf, b.stats, b.ctrl, b.gm, b.alpha, b.mu, b.beta, b.rho,
                                       b.work, b.B, b.bflag, b.use_newton);
    k_ctrl<<<1, 32, 0, st>>>(cf, b.stats, b.ctrl, b.bflag, b.hist, b.hist_cap);
    if (h.update_A) {
        dim3 g((h.n + 31) / 32, (h.n + 31) / 32, h.M);
        k_gemm64<<<g, 256, 0, st>>>(0, b.A, (size_t)h.n * h.n, b.B, (size_t)h.n * h.n, b.Anew,
                                    (size_t)h.n * h.n, nullptr, 0, nullptr, b.use_newton, b.ctrl, h.n);
    }
    k_reparm<<<h.M, 256, 0, st>>>(h.update_A, h.do_reparm, b.A, b.Anew, b.W, b.c, b.mu, b.beta,
                                  b.work, h.n, h.m);
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
