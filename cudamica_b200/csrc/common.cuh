// Shared definitions for the AMICA EM engine's CUDA kernels (sm_100a).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace amica {

constexpr int kMaxModels = 8;     // thread-block cluster size limit (portable)
constexpr int kMaxMix = 8;
constexpr float kLog2e = 1.4426950408889634f;
constexpr float kLn2 = 0.6931471805599453f;
constexpr float kTinyAbs = 1.17549435e-38f;  // FLT_MIN: |y| == 0 guard

// Error flags written by kernels (bit set in ctx->d_err).
enum : int {
    kErrWaitTimeout = 1,      // a bounded mbarrier / flag wait gave up
    kErrShape = 2,            // launch received a shape it was not built for
    kErrSingular = 4,         // zero pivot while inverting A
    kErrNonFinite = 8,        // the M-step produced a non-finite parameter
};

// Per-(model, mixture, channel) E-step constants, derived in FP64 from the
// parameters once per iteration and rounded to FP32:
//   y  = s * (W x)_i - off          (s = sqrt(beta), off = s * (mu + (W c)_i))
//   Q  = (cl2 - |y|^rho * log2 e) * ln 2
struct __align__(16) MixParam {
    float s, off, cl2, rho;
};

// Per-iteration control block, device resident (FP64 where the reference
// keeps double on the host: src/amica.cu:800-806).
struct Ctrl {
    double lrate, lratemax, ll, ll_prev, ltc0;
    int64_t iter, numdec, nkeep, nrej_total, rej_passes;
    int64_t newton, ll_decreased, no_newt, last_rejected;
    double rej_mean, rej_std;
    // split correction of phi (tensor-core form): the largest relative change
    // ||A_new - A|| / ||A|| of this iteration's A update (bits of a
    // non-negative double, so that an integer max orders them), the M-step
    // CTAs that have reported it, and the flag the E-step reads
    uint64_t newton_rel_bits;
    int64_t reparm_done, phi_split;
};

// One history record per iteration (read back by the host after a run).
struct IterRec {
    double ll, lrate;
    int64_t iter, newton, ll_decreased, nkeep, nrejected, phi_split;
};

// Layout of one partial-sum slot (doubles), model h:
//   [0] LL numerator (model 0 only), [1] vsum, then per channel
//   sum v b (n; b = W(x - c), from which cnew = A sum(v b) / vsum + c),
//   s2 = sum v b^2 (n), gsum = sum g (n), then usum, kn, ln, mn, md, bd, rn
//   (m*n each, mixture-major), then the n*n contraction (column-major, (i,k)
//   at k*n + i): Psi = sum_t g x^T from the plain kernel, or phi = sum_t g b^T
//   from the tensor-core kernel.  Slots are summed in a fixed order by k_reduce.
struct PartLayout {
    int n, m;
    __host__ __device__ int cn() const { return 2; }
    __host__ __device__ int s2() const { return 2 + n; }
    __host__ __device__ int gs() const { return 2 + 2 * n; }
    __host__ __device__ int mix(int k) const { return 2 + 3 * n + k * m * n; }  // k = 0..6
    __host__ __device__ int psi() const { return 2 + 3 * n + 7 * m * n; }
    __host__ __device__ int stride() const { return 2 + 3 * n + 7 * m * n + n * n; }
};

// Flat statistics vector (identical to the oracle's): [0] LL numerator, then
// per model S = 1 + 2n + n*n + 7mn doubles: vsum, cnew (n), sigma2 num (n),
// phi (n*n), usum, kappa num, lambda num, mu num, mu den, beta den, rho num.
struct StatLayout {
    int n, m;
    __host__ __device__ int S() const { return 1 + 2 * n + n * n + 7 * m * n; }
    __host__ __device__ int base(int h) const { return 1 + h * S(); }
    __host__ __device__ int vs() const { return 0; }
    __host__ __device__ int cn() const { return 1; }
    __host__ __device__ int s2() const { return 1 + n; }
    __host__ __device__ int phi() const { return 1 + 2 * n; }
    __host__ __device__ int mix(int k) const { return 1 + 2 * n + n * n + k * m * n; }
};

enum MixStat { kUs = 0, kKn = 1, kLn = 2, kMn = 3, kMd = 4, kBd = 5, kRn = 6 };

// A model whose responsibilities sum to less than one sample (vsum_h < 1: it
// explains no data) is frozen: its A, c and mixture parameters keep their
// values and gm_h = max(vsum_h / T, kMinGm).  Likewise a mixture component
// with no responsibility at all (usum_hij = 0: every FP32 responsibility
// underflowed) keeps its mu, beta and rho and drops out of the kappa and
// lambda sums (its alpha is 0).  The reference divides by vsum_h and usum_hij
// regardless (src/amica.cu:1995-2154), which turns such parameters, and
// through kappa/lambda and the A update the whole model, non-finite.
constexpr double kMinModelVsum = 1.0;
constexpr double kMinGm = 1e-300;

// Everything the fused E-step kernel needs, by value.
struct EStepArgs {
    const float* x;          // T x ldx sphered data (channels >= n are zero)
    const float* Wf;         // M x NP x NP, W[h][i][k] row-major, zero padded
    const float* wc;         // M x NP, (W c)_i in FP32
    const MixParam* mp;      // M x m x NP
    const double* ltc64;     // M: log gm_h + ldet_h + ldetS (FP64)
    const uint8_t* keep;     // T (nullptr = all kept)
    float* Lt_out;           // M x T relative Lt (nullptr = skip)
    float* P_out;            // T relative P (nullptr = skip)
    double* partial;         // nclusters x M x stride
    int* err;
    int64_t T;
    int ldx, n, M, m;
    int ntiles, nclusters;
    int update_rho;
    int grad_mode;           // 1: beta-denominator slot holds sum u*f'*y for every rho (adjoint)
    // density-only form (contractions done outside the kernel): b = W x per
    // sample, [T][M][NP] with a row of ldb floats per sample; g written as the
    // operand image of the Psi contraction: per 32-sample block, model and
    // 128-channel half, a 128 x 32 K-major tile with the 128-byte swizzle
    // ([block][model][half][4096 floats], see sw128_off)
    const float* bext;
    float* gout;
    int ldb;
    // tensor-core form: device flag, nonzero = form phi from hi + lo parts of
    // both operands (split correction); nullptr = off
    const int64_t* split_phi;
};

// The cohort E-step (one persistent launch over many single-model fits): a
// subject's arguments and lane packing, and a run of its tiles.
struct TcCohortSub {
    EStepArgs a;   // the subject's E-step arguments (M = 1)
    int R;         // lane packing of its channel count (128 / padded channels)
};
struct TcCohortItem {
    int sub;       // subject
    int slot;      // partial-slot group in the subject's buffer
    int64_t tile0; // first tile
    int ntiles;    // consecutive tiles
};

// Device buffers and host-side settings of the FP64 M-step kernels.
struct MStepBuffers {
    double *A, *Anew, *c, *alpha, *mu, *beta, *rho, *gm, *W, *ldet, *ltc64;
    double *partial, *raw, *stats, *work, *chunk;
    double* gj;        // n > 128: M n^2 working matrices + M n pivot logs of the inverse
    int64_t* bflag;          // M: Newton-condition violations of the last M-step
    int* use_newton;         // M: 1 Newton step, 0 natural gradient, -1 frozen model (no update)
    float *Wf, *wcf;
    MixParam* mp;
    Ctrl* ctrl;
    IterRec* hist;
    int64_t hist_cap;
    int* err;
};
struct MStepCfgHost {
    int n, m, M, NP;
    int do_newton, update_rho, rho_start_iter, newt_start_iter, maxdec;
    int update_gm, update_alpha, update_A, update_mu, update_beta, do_reparm;
    int do_reject, rejstart, rejint, maxrej;
    double lratemax, lnatrate, lratefact, rholrate, rhomin, rhomax, rejsig, ldetS;
    int psi_is_phi;   // 1: the E-step's n x n slot already holds phi = sum g b^T (tensor-core form)
    int psi_step;     // only every psi_step-th partial slot carries the n x n block
    int phi_split;    // split correction of phi: 0 never, 1 always, 2 once a Newton step's relative change < phi_split_rel
    double phi_split_rel;
};
// Default relative change of A below which the split correction of phi
// switches on (phi_split = 2).
constexpr double kPhiSplitRel = 1e-4;

}  // namespace amica

// ---- small PTX helpers ----------------------------------------------------
__device__ __forceinline__ float ptx_ex2(float x) {
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float ptx_lg2(float x) {
    float y;
    asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float ptx_rcp(float x) {
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
