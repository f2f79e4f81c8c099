// Generalized-Gaussian mixture density math shared by the fused E-step
// kernels (src/kernels.cu:251-827 of the reference, restated in FP32 with
// MUFU ex2/lg2/rcp), written once so that both forms use the same arithmetic.
#pragma once

#include "common.cuh"

namespace amica {

// Mixture math on one float or on a float2 pair of mixtures (sm_100 packed
// FP32 instructions: one issue for two lanes of work).
__device__ __forceinline__ float splat_v(float a, float) { return a; }
__device__ __forceinline__ float2 splat_v(float a, float2) { return make_float2(a, a); }
__device__ __forceinline__ float vfma(float a, float b, float c) { return fmaf(a, b, c); }
__device__ __forceinline__ float2 vfma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float vmul(float a, float b) { return a * b; }
__device__ __forceinline__ float2 vmul(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float vadd(float a, float b) { return a + b; }
__device__ __forceinline__ float2 vadd(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float vabsmax(float y) { return fmaxf(fabsf(y), kTinyAbs); }
__device__ __forceinline__ float2 vabsmax(float2 y) { return make_float2(vabsmax(y.x), vabsmax(y.y)); }
__device__ __forceinline__ float vlg2(float x) { return ptx_lg2(x); }
__device__ __forceinline__ float2 vlg2(float2 x) { return make_float2(ptx_lg2(x.x), ptx_lg2(x.y)); }
__device__ __forceinline__ float vex2(float x) { return ptx_ex2(x); }
__device__ __forceinline__ float2 vex2(float2 x) { return make_float2(ptx_ex2(x.x), ptx_ex2(x.y)); }
// 1/y with |y| clamped to ay
__device__ __forceinline__ float vrcp_signed(float ay, float y) { return ptx_rcp(copysignf(ay, y)); }
__device__ __forceinline__ float2 vrcp_signed(float2 ay, float2 y) {
    return make_float2(ptx_rcp(copysignf(ay.x, y.x)), ptx_rcp(copysignf(ay.y, y.y)));
}

// Per-mixture parameters of one channel, as scalars or pairs.
template <class V>
struct MixV {
    V s, npo, pc, pr, sr;   // sqrt(beta), -sqrt(beta)(mu + w c), log2 normaliser, rho, sqrt(beta) rho
};

// Phase 1 for one sample: q = log2 of the mixture term, and log2|y|.
template <class V>
__device__ __forceinline__ V dens_q(const MixV<V>& P, float bx, V& L2) {
    const V y = vfma(P.s, splat_v(bx, V{}), P.npo);
    L2 = vlg2(vabsmax(y));
    const V p = vex2(vmul(P.pr, L2));
    return vfma(splat_v(-kLog2e, V{}), p, P.pc);
}

// Phase 2 for one sample: the seven sums A0..A6 and the g term.
template <class V, bool kHaveL2>
__device__ __forceinline__ void dens_acc(const MixV<V>& P, float bx, V L2, float nlse, float v, V* A,
                                         V& g) {
    const V y = vfma(P.s, splat_v(bx, V{}), P.npo);
    const V ay = vabsmax(y);
    if constexpr (!kHaveL2) L2 = vlg2(ay);
    const V p = vex2(vmul(P.pr, L2));
    const V z = vex2(vadd(vfma(splat_v(-kLog2e, V{}), p, P.pc), splat_v(nlse, V{})));
    const V uu = vmul(z, splat_v(v, V{}));
    const V ri = vrcp_signed(ay, y);
    const V w = vmul(uu, p);
    A[0] = vadd(A[0], uu);
    A[1] = vadd(A[1], w);
    A[2] = vfma(w, p, A[2]);
    A[3] = vfma(w, L2, A[3]);
    const V wr = vmul(w, ri);
    A[4] = vadd(A[4], wr);
    const V wr2 = vmul(wr, ri);
    A[5] = vadd(A[5], wr2);
    A[6] = vfma(wr2, p, A[6]);
    g = vfma(P.sr, wr, g);
}

// log-sum-exp over the mixtures in log2 units: qmax + log2(sum 2^(q - qmax)).
// The term of the maximum is exactly 1, so for m <= 3 its ex2 is skipped.
template <int MM>
__device__ __forceinline__ float lse2(const float* q) {
    if constexpr (MM == 1) {
        return q[0];
    } else if constexpr (MM == 2) {
        const float mx = fmaxf(q[0], q[1]), mn = fminf(q[0], q[1]);
        return mx + ptx_lg2(1.f + ptx_ex2(mn - mx));
    } else if constexpr (MM == 3) {
        const float m01 = fmaxf(q[0], q[1]), n01 = fminf(q[0], q[1]);
        const float mx = fmaxf(m01, q[2]), o1 = fminf(m01, q[2]);
        return mx + ptx_lg2(1.f + ptx_ex2(o1 - mx) + ptx_ex2(n01 - mx));
    } else {
        float mx = q[0];
#pragma unroll
        for (int j = 1; j < MM; j++) mx = fmaxf(mx, q[j]);
        float se = 0.f;
#pragma unroll
        for (int j = 0; j < MM; j++) se += ptx_ex2(q[j] - mx);
        return mx + ptx_lg2(se);
    }
}

// ---- the tensor-core E-step's form: one ex2 per element ----------------------
// With ay = max(|y|, FLT_MIN), L2 = log2 ay and q2 = ay^(rho - 2) = 2^((rho-2) L2):
//   p = |y|^rho = q2 y^2,   p / y = sign(y)|y|^(rho-1) = q2 y,   p / y^2 = q2,
// so the seven sums need no reciprocal of y:
//   A0 = sum u, A1 = sum u p, A2 = sum u p^2, A3 = sum u p L2,
//   A4 = sum u q2 y, A5 = sum u q2, A6 = sum u p q2,
// and g = sum_j sqrt(beta) rho u q2 y.  Every quantity is a pair: two mixtures
// of one sample, or one mixture (its parameters splatted) of two samples.
struct MixT2 {
    float2 s, npo, pc, pm2, sr;   // sqrt(beta), -sqrt(beta)(mu + w c), log2 normaliser, rho - 2, sqrt(beta) rho
};
__device__ __forceinline__ float2 f2s(float a) { return make_float2(a, a); }

// Phase 1: log2 of the mixture term q, with L2 and q2 for the cache.  Where
// y is 0 (FP32 cancellation of sqrt(beta) b and its offset), |y| is clamped
// to FLT_MIN for the logarithm and q2 is set to 0, so that the sample adds
// nothing to the sums that carry |y|^(rho-2) (p = |y|^rho underflows to 0
// there, as it does in the plain form's arithmetic).
__device__ __forceinline__ float2 tc_phase1(const MixT2& P, float2 bx, float2& L2, float2& q2) {
    const float2 y = __ffma2_rn(P.s, bx, P.npo);
    const float2 ay = make_float2(fmaxf(fabsf(y.x), kTinyAbs), fmaxf(fabsf(y.y), kTinyAbs));
    L2 = make_float2(ptx_lg2(ay.x), ptx_lg2(ay.y));
    const float2 e = __fmul2_rn(P.pm2, L2);
    const float ex = ptx_ex2(e.x), ey = ptx_ex2(e.y);
    q2 = make_float2(ay.x > kTinyAbs ? ex : 0.f, ay.y > kTinyAbs ? ey : 0.f);
    const float2 p = __fmul2_rn(q2, __fmul2_rn(ay, ay));
    return __ffma2_rn(f2s(-kLog2e), p, P.pc);
}

// L2 and q2 again from b (when they are not kept between the phases).
__device__ __forceinline__ void tc_recompute(const MixT2& P, float2 bx, float2& L2, float2& q2) {
    const float2 y = __ffma2_rn(P.s, bx, P.npo);
    const float2 ay = make_float2(fmaxf(fabsf(y.x), kTinyAbs), fmaxf(fabsf(y.y), kTinyAbs));
    L2 = make_float2(ptx_lg2(ay.x), ptx_lg2(ay.y));
    const float2 e = __fmul2_rn(P.pm2, L2);
    const float ex = ptx_ex2(e.x), ey = ptx_ex2(e.y);
    q2 = make_float2(ay.x > kTinyAbs ? ex : 0.f, ay.y > kTinyAbs ? ey : 0.f);
}

// Phase 2: the sums of one pair, given the responsibility z, q2, L2 and v.
__device__ __forceinline__ void tc_phase2(const MixT2& P, float2 bx, float2 z, float2 q2, float2 L2,
                                          float2 v, float2* A, float2& g) {
    const float2 u = __fmul2_rn(v, z);
    const float2 y = __ffma2_rn(P.s, bx, P.npo);
    const float2 w = __fmul2_rn(u, q2);
    const float2 gj = __fmul2_rn(w, y);
    A[4] = __fadd2_rn(A[4], gj);
    A[5] = __fadd2_rn(A[5], w);
    const float2 y2 = __fmul2_rn(y, y);
    const float2 wp = __fmul2_rn(w, y2);
    A[1] = __fadd2_rn(A[1], wp);
    const float2 p = __fmul2_rn(q2, y2);
    A[2] = __ffma2_rn(wp, p, A[2]);
    A[6] = __ffma2_rn(wp, q2, A[6]);
    A[3] = __ffma2_rn(wp, L2, A[3]);
    A[0] = __fadd2_rn(A[0], u);
    g = __ffma2_rn(P.sr, gj, g);
}

// Log-sum-exp over the mixtures (log2 units) and the responsibilities
// z_j = 2^(q_j - lse), from one set of exponentials: e_j = 2^(q_j - qmax),
// S = sum e_j, lse = qmax + log2 S, z_j = e_j / S; for two samples at once
// (x and y halves).
template <int MM>
__device__ __forceinline__ float2 tc_lse2(const float2* q, float2* z) {
    if constexpr (MM == 1) {
        z[0] = f2s(1.f);
        return q[0];
    } else {
        float2 mx = q[0];
#pragma unroll
        for (int j = 1; j < MM; j++) mx = make_float2(fmaxf(mx.x, q[j].x), fmaxf(mx.y, q[j].y));
        const float2 nmx = make_float2(-mx.x, -mx.y);
        float2 S = make_float2(0.f, 0.f);
#pragma unroll
        for (int j = 0; j < MM; j++) {
            const float2 d = __fadd2_rn(q[j], nmx);
            z[j] = make_float2(ptx_ex2(d.x), ptx_ex2(d.y));
            S = __fadd2_rn(S, z[j]);
        }
        const float2 rS = make_float2(ptx_rcp(S.x), ptx_rcp(S.y));
#pragma unroll
        for (int j = 0; j < MM; j++) z[j] = __fmul2_rn(z[j], rS);
        return __fadd2_rn(mx, make_float2(ptx_lg2(S.x), ptx_lg2(S.y)));
    }
}
template <int MM>
__device__ __forceinline__ float tc_lse(const float* q, float* z) {
    if constexpr (MM == 1) {
        z[0] = 1.f;
        return q[0];
    } else {
        float mx = q[0];
#pragma unroll
        for (int j = 1; j < MM; j++) mx = fmaxf(mx, q[j]);
        float S = 0.f;
#pragma unroll
        for (int j = 0; j < MM; j++) {
            z[j] = ptx_ex2(q[j] - mx);
            S += z[j];
        }
        const float rS = ptx_rcp(S);
#pragma unroll
        for (int j = 0; j < MM; j++) z[j] *= rS;
        return mx + ptx_lg2(S);
    }
}

// ---- the tensor-core E-step's phases, on pairs of consecutive samples ---------
// |y| is floored at kYFloor = 2^-23 (one FP32 ulp of 1) before the logarithm:
// an FP32 y that cancelled to 0 or to a few ulp then contributes
// |y|^(rho-2) <= 2^(23 (2 - rho)), the size its FP64 value has, instead of a
// value set by FLT_MIN (up to 2^126).  p = |y|^rho is then at most 2^-23, so
// the densities do not move.
constexpr float kYFloor = 1.1920928955078125e-07f;

// Phase 1: log2 of the mixture term for two samples, and L2 = log2 max(|y|, kYFloor).
__device__ __forceinline__ float2 tcp1(const MixT2& P, float2 bx, float2& L2) {
    const float2 y = __ffma2_rn(P.s, bx, P.npo);
    const float2 ay = make_float2(fmaxf(fabsf(y.x), kYFloor), fmaxf(fabsf(y.y), kYFloor));
    L2 = make_float2(ptx_lg2(ay.x), ptx_lg2(ay.y));
    const float2 e = __fmul2_rn(P.pm2, L2);
    const float2 q2 = make_float2(ptx_ex2(e.x), ptx_ex2(e.y));
    const float2 p = __fmul2_rn(q2, __fmul2_rn(ay, ay));
    return __ffma2_rn(f2s(-kLog2e), p, P.pc);
}

// Log-sum-exp over the mixtures of two samples (log2 units); the term of the
// maximum is exactly 1, so for m <= 3 its ex2 is skipped.
template <int MM>
__device__ __forceinline__ float2 tc_lse_pair(const float2* q) {
    if constexpr (MM == 1) {
        return q[0];
    } else if constexpr (MM == 2) {
        const float2 mx = make_float2(fmaxf(q[0].x, q[1].x), fmaxf(q[0].y, q[1].y));
        const float2 mn = make_float2(fminf(q[0].x, q[1].x), fminf(q[0].y, q[1].y));
        const float2 d = __fadd2_rn(mn, make_float2(-mx.x, -mx.y));
        const float2 sm = __fadd2_rn(f2s(1.f), make_float2(ptx_ex2(d.x), ptx_ex2(d.y)));
        return __fadd2_rn(mx, make_float2(ptx_lg2(sm.x), ptx_lg2(sm.y)));
    } else if constexpr (MM == 3) {
        const float2 m01 = make_float2(fmaxf(q[0].x, q[1].x), fmaxf(q[0].y, q[1].y));
        const float2 n01 = make_float2(fminf(q[0].x, q[1].x), fminf(q[0].y, q[1].y));
        const float2 mx = make_float2(fmaxf(m01.x, q[2].x), fmaxf(m01.y, q[2].y));
        const float2 o1 = make_float2(fminf(m01.x, q[2].x), fminf(m01.y, q[2].y));
        const float2 nmx = make_float2(-mx.x, -mx.y);
        const float2 d1 = __fadd2_rn(o1, nmx), d2 = __fadd2_rn(n01, nmx);
        float2 sm = __fadd2_rn(f2s(1.f), make_float2(ptx_ex2(d1.x), ptx_ex2(d1.y)));
        sm = __fadd2_rn(sm, make_float2(ptx_ex2(d2.x), ptx_ex2(d2.y)));
        return __fadd2_rn(mx, make_float2(ptx_lg2(sm.x), ptx_lg2(sm.y)));
    } else {
        float2 mx = q[0];
#pragma unroll
        for (int j = 1; j < MM; j++) mx = make_float2(fmaxf(mx.x, q[j].x), fmaxf(mx.y, q[j].y));
        const float2 nmx = make_float2(-mx.x, -mx.y);
        float2 sm = make_float2(0.f, 0.f);
#pragma unroll
        for (int j = 0; j < MM; j++) {
            const float2 d = __fadd2_rn(q[j], nmx);
            sm = __fadd2_rn(sm, make_float2(ptx_ex2(d.x), ptx_ex2(d.y)));
        }
        return __fadd2_rn(mx, make_float2(ptx_lg2(sm.x), ptx_lg2(sm.y)));
    }
}

// Phase 2 for two samples of one mixture: from b, the kept L2 and the
// per-sample lse and v, q2 = 2^((rho-2) L2) and the responsibility
// z = 2^(q - lse) (two ex2 per element, no reciprocal), then the seven sums
// (A0..A6 as in tc_phase2) and g.  (q - lse is formed as fma(lse, -1, q):
// exact negation, one rounding, the same value as q + (-lse).)
__device__ __forceinline__ void tcp2(const MixT2& P, float2 bx, float2 L2, float2 lse, float2 v,
                                     float2* A, float2& g) {
    const float2 y = __ffma2_rn(P.s, bx, P.npo);
    const float2 e = __fmul2_rn(P.pm2, L2);
    const float2 q2 = make_float2(ptx_ex2(e.x), ptx_ex2(e.y));
    const float2 y2 = __fmul2_rn(y, y);
    const float2 p = __fmul2_rn(q2, y2);
    const float2 t = __ffma2_rn(lse, f2s(-1.f), __ffma2_rn(f2s(-kLog2e), p, P.pc));
    const float2 z = make_float2(ptx_ex2(t.x), ptx_ex2(t.y));
    const float2 u = __fmul2_rn(v, z);
    const float2 w = __fmul2_rn(u, q2);
    const float2 gj = __fmul2_rn(w, y);
    A[4] = __fadd2_rn(A[4], gj);
    A[5] = __fadd2_rn(A[5], w);
    const float2 wp = __fmul2_rn(w, y2);
    A[1] = __fadd2_rn(A[1], wp);
    A[2] = __ffma2_rn(wp, p, A[2]);
    A[6] = __ffma2_rn(wp, q2, A[6]);
    A[3] = __ffma2_rn(wp, L2, A[3]);
    A[0] = __fadd2_rn(A[0], u);
    g = __ffma2_rn(P.sr, gj, g);
}

// Round to TF32, to nearest with ties away from zero, on the integer pipe
// (finite inputs): add half of the dropped range, then clear the 13 low bits.
__device__ __forceinline__ float tf32_rna_alu(float x) {
    return __uint_as_float((__float_as_uint(x) + 0x1000u) & 0xFFFFE000u);
}

// The seven per-(channel, mixture) sums A0..A6 of dens_acc mapped to the
// reference's statistics (usum, kappa num, lambda num, mu num, mu den, beta den,
// rho num; src/kernels.cu:495-827), with f' = rho p / y:
//   usum = A0, sum u f'^2 = rho^2 A6, sum u (f' y - 1)^2 = rho^2 A2 - 2 rho A1 + A0,
//   sum u f' = rho A4, mu den = sum u f'/y = rho A5 (rho <= 2) or sum u f'^2 (rho > 2),
//   beta den = sum u f' y = rho A1 (rho <= 2) or sum u |y|^rho = A1 (rho > 2),
//   sum u |y|^rho log|y|^rho = rho ln2 A3.
// In gradient mode mu den and beta den always take the rho <= 2 forms.
__device__ __forceinline__ void mix_stats_from_sums(double A0, double A1, double A2, double A3,
                                                    double A4, double A5, double A6, float rho_f,
                                                    int grad_mode, int update_rho, double& us,
                                                    double& kn, double& ln, double& mn, double& md,
                                                    double& bd, double& rn) {
    const double r = (double)rho_f;
    us = A0;
    kn = r * r * A6;
    ln = (r * r * A2 - 2.0 * r * A1) + A0;
    mn = r * A4;
    if (rho_f <= 2.f || grad_mode) {
        md = r * A5;
        bd = r * A1;
    } else {
        md = r * r * A6;
        bd = A1;
    }
    rn = update_rho ? r * kLn2 * A3 : 0.0;
}

}  // namespace amica
