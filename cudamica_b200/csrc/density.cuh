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
