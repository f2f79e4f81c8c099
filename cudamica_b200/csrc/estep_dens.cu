// Density-only E-step of the split mixed form (128 < n <= 256 channels).
//
// b = W x comes from the tensor-core contraction before this kernel and
// Psi = sum g x^T from the one after it; this kernel does the rest of the
// E-step of src/kernels.cu:251-827 (the mixture log-densities, log-sum-exp
// over mixtures, Lt per model, the posterior over models, responsibilities,
// score function and the per-(channel, mixture) sums) and writes g as the
// Psi contraction's operand image.
//
// Layout: one thread-block cluster of M CTAs (CTA h = model h) per tile
// stream, 256 threads per CTA (thread = channel, all 32 samples of a tile),
// 128 registers, two CTAs per SM: clusters of M place on any SM pair, so the
// grid covers every SM (one 512-thread CTA per SM left 16 of 148 SMs idle at
// M = 4), and one CTA's barrier waits are the other's issue slots.  The b rows
// of a tile arrive by bulk copies into one of two shared-memory stages; the
// copy of the next tile is issued as the current one starts.
//
// Arithmetic per element (no reciprocal): with ay = max(|y|, 2^-23),
// L2 = log2 ay and q2 = 2^((rho - 2) L2),
//   p = |y|^rho = q2 y^2,  p / y = q2 y,  p / y^2 = q2,
// phase 1 forms log2 of the mixture term from p, phase 2 forms L2 and q2
// again and the responsibility z = 2^(q - lse): 2 + 3 MUFU ops per element,
// plus m - 1 ex2 and one lg2 per (channel, sample) for the log-sum-exp.
//
// Sums: FP32 per thread over kFlush tiles, then added (red.global.add.f64)
// into FP64 running sums that each thread owns in the Psi region of its CTA's
// partial slot (which the Psi contraction after this kernel fills): one
// writer per entry, so the adds land in program order and results are
// deterministic.  A sample whose model responsibility v is exactly 0 adds
// exactly 0 to every sum and to g, and its phase 2 is skipped (v is the same
// for every thread of the CTA).
#include <cooperative_groups.h>
#include <cstdio>

#include "common.cuh"
#include "density.cuh"
#include "tc_ptx.cuh"

namespace cg = cooperative_groups;
using namespace amica;

namespace {

constexpr int kDT = 256;              // threads per CTA (one per channel); two CTAs per SM
constexpr int kDNP = 256;             // channels (padded)
constexpr int kDS = 32;               // samples per tile
constexpr int kDLL = kDNP + 16;       // padded row of the lse tile (conflict-free reduction)
constexpr int kFlush = 8;             // tiles between FP32 -> FP64 flushes

template <int MM>
struct DensShape {
    static constexpr int NACC = 7 * MM + 3;   // A0..A6 per mixture, sum v b, sum v b^2, sum g
    static constexpr size_t off_b = 0;                                          // [2][kDS][kDNP] float
    static constexpr size_t off_lse = off_b + 2 * (size_t)kDS * kDNP * 4;       // [kDS][kDLL] float
    static constexpr size_t off_slot = off_lse + (size_t)kDS * kDLL * 4;        // [2][kDS] float
    static constexpr size_t off_v = off_slot + 2 * kDS * 4;                     // [kDS] float
    static constexpr size_t off_bar = off_v + kDS * 4;                          // 2 mbarriers, abort flag
    static constexpr size_t bytes = off_bar + 32;
    static_assert(off_b % 16 == 0 && off_bar % 8 == 0, "alignment");
};

// Per-mixture constants of one channel for two mixtures at once.
struct MixQ2 {
    float2 s, npo, pc, pm2, sr;   // sqrt(beta), -sqrt(beta)(mu + w c), log2 normaliser, rho - 2, sqrt(beta) rho
};
struct MixQ1 {
    float s, npo, pc, pm2, sr;
};

// log2 sum_j 2^q_j over the mixtures: the maximum is found by a tournament
// that keeps the other m - 1 values, so the maximum's term (exactly 1) costs
// no ex2 for any m.
template <int MM>
__device__ __forceinline__ float lse_mix(const float* q) {
    if constexpr (MM <= 3) {
        return lse2<MM>(q);
    } else {
        const float m01 = fmaxf(q[0], q[1]), n01 = fminf(q[0], q[1]);
        const float m23 = fmaxf(q[2], q[3]), n23 = fminf(q[2], q[3]);
        float mx = fmaxf(m01, m23);
        const float nA = fminf(m01, m23);
        float o4 = -INFINITY;
        if constexpr (MM == 5) {
            o4 = fminf(mx, q[4]);
            mx = fmaxf(mx, q[4]);
        }
        float s = 1.f + ptx_ex2(n01 - mx);
        s += ptx_ex2(n23 - mx);
        s += ptx_ex2(nA - mx);
        if constexpr (MM == 5) s += ptx_ex2(o4 - mx);
        return mx + ptx_lg2(s);
    }
}

// Phase 1, two mixtures of one sample: log2 of the mixture terms.
__device__ __forceinline__ float2 dq_pair(const MixQ2& P, float bx) {
    const float2 y = __ffma2_rn(P.s, f2s(bx), P.npo);
    const float2 ay = make_float2(fmaxf(fabsf(y.x), kYFloor), fmaxf(fabsf(y.y), kYFloor));
    const float2 L2 = make_float2(ptx_lg2(ay.x), ptx_lg2(ay.y));
    const float2 e = __fmul2_rn(P.pm2, L2);
    const float2 q2 = make_float2(ptx_ex2(e.x), ptx_ex2(e.y));
    const float2 p = __fmul2_rn(q2, __fmul2_rn(ay, ay));
    return __ffma2_rn(f2s(-kLog2e), p, P.pc);
}
__device__ __forceinline__ float dq_one(const MixQ1& P, float bx) {
    const float y = fmaf(P.s, bx, P.npo);
    const float ay = fmaxf(fabsf(y), kYFloor);
    const float L2 = ptx_lg2(ay);
    const float q2 = ptx_ex2(P.pm2 * L2);
    return fmaf(-kLog2e, q2 * (ay * ay), P.pc);
}

// Phase 2, two mixtures of one sample: L2 and q2 again, the responsibility
// z = 2^(q - lse), then A0..A6 (A0 = sum u, A1 = sum u p, A2 = sum u p^2,
// A3 = sum u p L2, A4 = sum u q2 y, A5 = sum u q2, A6 = sum u p q2) and the
// sample's g term sum_j sqrt(beta) rho u q2 y.
__device__ __forceinline__ void da_pair(const MixQ2& P, float bx, float nlse, float v, float2* A,
                                        float2& g) {
    const float2 y = __ffma2_rn(P.s, f2s(bx), P.npo);
    const float2 ay = make_float2(fmaxf(fabsf(y.x), kYFloor), fmaxf(fabsf(y.y), kYFloor));
    const float2 L2 = make_float2(ptx_lg2(ay.x), ptx_lg2(ay.y));
    const float2 e = __fmul2_rn(P.pm2, L2);
    const float2 q2 = make_float2(ptx_ex2(e.x), ptx_ex2(e.y));
    const float2 y2 = __fmul2_rn(y, y);
    const float2 p = __fmul2_rn(q2, y2);
    const float2 t = __fadd2_rn(__ffma2_rn(f2s(-kLog2e), p, P.pc), f2s(nlse));
    const float2 z = make_float2(ptx_ex2(t.x), ptx_ex2(t.y));
    const float2 u = __fmul2_rn(f2s(v), z);
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
__device__ __forceinline__ void da_one(const MixQ1& P, float bx, float nlse, float v, float* A, float& g) {
    const float y = fmaf(P.s, bx, P.npo);
    const float ay = fmaxf(fabsf(y), kYFloor);
    const float L2 = ptx_lg2(ay);
    const float q2 = ptx_ex2(P.pm2 * L2);
    const float y2 = y * y;
    const float p = q2 * y2;
    const float z = ptx_ex2(fmaf(-kLog2e, p, P.pc) + nlse);
    const float u = v * z;
    const float w = u * q2;
    const float gj = w * y;
    A[4] += gj;
    A[5] += w;
    const float wp = w * y2;
    A[1] += wp;
    A[2] = fmaf(wp, p, A[2]);
    A[6] = fmaf(wp, q2, A[6]);
    A[3] = fmaf(wp, L2, A[3]);
    A[0] += u;
    g = fmaf(P.sr, gj, g);
}

// The b rows of one tile of model h into the b buffer: one 1 KB bulk copy per
// sample (rows past T are not copied; phase 1 reads them as 0).  Warp 0.
__device__ __forceinline__ void issue_b_tile(const EStepArgs& a, int h, int tile, float* bs, uint64_t* bar,
                                             int lane) {
    const int64_t t0 = (int64_t)tile * kDS;
    const int64_t left = a.T - t0;
    const int rows = left < kDS ? (int)left : kDS;
    if (lane == 0) mbar_expect_tx(bar, (uint32_t)rows * kDNP * 4);
    __syncwarp();
    if (lane < rows)
        bulk_load(smem_u32(bs + lane * kDNP), a.bext + (size_t)(t0 + lane) * a.ldb + (size_t)h * kDNP,
                  kDNP * 4, bar);
}

template <int MM>
__global__ void __launch_bounds__(kDT, 2) estep_dens_kernel(EStepArgs a) {
    using Sh = DensShape<MM>;
    constexpr int NACC = Sh::NACC;
    constexpr int NPR = MM / 2;
    constexpr bool kOdd = (MM & 1) != 0;
    constexpr int NPRA = NPR > 0 ? NPR : 1;
    extern __shared__ __align__(128) unsigned char dsm[];
    float* bs = reinterpret_cast<float*>(dsm + Sh::off_b);
    float* lse = reinterpret_cast<float*>(dsm + Sh::off_lse);
    float* slot = reinterpret_cast<float*>(dsm + Sh::off_slot);
    float* vS = reinterpret_cast<float*>(dsm + Sh::off_v);
    uint64_t* bar = reinterpret_cast<uint64_t*>(dsm + Sh::off_bar);   // [2]: b stage full
    volatile int* abort_flag = reinterpret_cast<volatile int*>(dsm + Sh::off_bar + 16);

    cg::cluster_group cluster = cg::this_cluster();
    const int h = (int)cluster.block_rank();
    const int M = a.M, n = a.n;
    const int cid = blockIdx.x / M;
    const int tid = threadIdx.x, lane = tid & 31;
    const int ch = tid;
    const bool ch_ok = ch < n;
    const int64_t T = a.T;
    const int ntiles = (int)((T + kDS - 1) / kDS);
    if (a.m != MM || n > kDNP || NACC > n || M > kMaxModels) {   // the same in every CTA: all return
        if (tid == 0) atomicOr(a.err, kErrShape);
        return;
    }
    // FP64 running sums: the thread of channel ch owns NACC entries (stride n)
    // in the Psi region of the CTA's partial slot, which the Psi contraction
    // after this kernel fills (NACC <= n).  Only the owning thread adds to an
    // entry, so its adds land in program order and the sums are deterministic.
    PartLayout L{n, MM};
    double* out = a.partial + ((size_t)cid * M + h) * L.stride();
    double* run = out + L.psi() + ch;
    if (ch_ok) {
#pragma unroll 1
        for (int e = 0; e < NACC; e++) run[(size_t)e * n] = 0.0;
    }
    if (tid == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    MixQ2 P2[NPRA];
    MixQ1 P1;
#pragma unroll
    for (int j = 0; j < MM; j++) {
        const MixParam q = a.mp[((size_t)h * MM + j) * kDNP + ch];
        const float vals[5] = {q.s, -q.off, q.cl2, q.rho - 2.f, q.s * q.rho};
        if (j < 2 * NPR) {
            float2* f[5] = {&P2[j / 2].s, &P2[j / 2].npo, &P2[j / 2].pc, &P2[j / 2].pm2, &P2[j / 2].sr};
#pragma unroll
            for (int e = 0; e < 5; e++) {
                if (j & 1) f[e]->y = vals[e];
                else f[e]->x = vals[e];
            }
        } else {
            P1.s = vals[0]; P1.npo = vals[1]; P1.pc = vals[2]; P1.pm2 = vals[3]; P1.sr = vals[4];
        }
    }
    const float wci = a.wc[(size_t)h * kDNP + ch];
    const float ltch = (float)(a.ltc64[h] - a.ltc64[0]);
    __syncthreads();
    if (tid < 32 && cid < ntiles) issue_b_tile(a, h, cid, bs, &bar[0], lane);

    float2 fP[NPRA][7];
    float fS1[7];
    float fCn, fS2, fGs;
    auto zero_f32 = [&]() {
#pragma unroll
        for (int k = 0; k < 7; k++) {
#pragma unroll
            for (int qq = 0; qq < NPRA; qq++) fP[qq][k] = make_float2(0.f, 0.f);
            fS1[k] = 0.f;
        }
        fCn = 0.f; fS2 = 0.f; fGs = 0.f;
    };
    // FP32 sums into this thread's FP64 running sums (fire-and-forget adds at
    // L2): entry k * MM + j is A_k of mixture j, then sum v b, sum v b^2, sum g
    auto flush = [&]() {
        if (ch_ok) {
#pragma unroll
            for (int k = 0; k < 7; k++) {
#pragma unroll
                for (int qq = 0; qq < NPR; qq++) {
                    red_add_f64(run + (size_t)(k * MM + 2 * qq) * n, (double)fP[qq][k].x);
                    red_add_f64(run + (size_t)(k * MM + 2 * qq + 1) * n, (double)fP[qq][k].y);
                }
                if constexpr (kOdd) red_add_f64(run + (size_t)(k * MM + MM - 1) * n, (double)fS1[k]);
            }
            red_add_f64(run + (size_t)(7 * MM + 0) * n, (double)fCn);
            red_add_f64(run + (size_t)(7 * MM + 1) * n, (double)fS2);
            red_add_f64(run + (size_t)(7 * MM + 2) * n, (double)fGs);
        }
        zero_f32();
    };
    zero_f32();
    double dLL = 0.0, dVs = 0.0;   // per-sample threads (tid < kDS)
    // warp 0: b stages whose copy was issued and not yet seen complete
    uint32_t pend = cid < ntiles ? 1u : 0u;   // bit s: stage s
    uint32_t pendpar = 0u;                    // bit s: the parity its copy completes

    int it = 0;
    for (int tile = cid; tile < ntiles; tile += a.nclusters, ++it) {
        const int64_t t0 = (int64_t)tile * kDS;
        const int par = it & 1, stg = it & 1;
        const float* bst = bs + stg * (kDS * kDNP);
        if (mbar_wait(&bar[stg], (uint32_t)(it >> 1) & 1u, abort_flag, a.err) && tid < 32) pend &= ~(1u << stg);
        // ---- the other stage was last read before the previous tile's final
        // barrier: fetch the next tile into it
        const int next = tile + a.nclusters;
        if (tid < 32) {
            const int go = __shfl_sync(0xffffffffu, (next < ntiles && !abort_get(abort_flag)) ? 1 : 0, 0);
            if (go) issue_b_tile(a, h, next, bs + (stg ^ 1) * (kDS * kDNP), &bar[stg ^ 1], lane);
            if (go) {
                pend |= 1u << (stg ^ 1);
                pendpar = (pendpar & ~(1u << (stg ^ 1))) | ((((uint32_t)(it + 1) >> 1) & 1u) << (stg ^ 1));
            }
        }
        // ---- phase 1: log-sum-exp over mixtures per (channel, sample), log2 units
#pragma unroll 4
        for (int t = 0; t < kDS; t++) {
            const float bx = (t0 + t < T) ? bst[t * kDNP + ch] : 0.f;
            float q[MM];
#pragma unroll
            for (int qq = 0; qq < NPR; qq++) {
                const float2 q2 = dq_pair(P2[qq], bx);
                q[2 * qq] = q2.x;
                q[2 * qq + 1] = q2.y;
            }
            if constexpr (kOdd) q[MM - 1] = dq_one(P1, bx);
            lse[t * kDLL + ch] = ch_ok ? lse_mix<MM>(q) : 0.f;
        }
        __syncthreads();
        // ---- Lt_h(t): in two rounds, sample t = 16 r + tid / 16 summed by 16
        // threads over channels j, j + 16, ... (fixed order, then a fixed
        // butterfly), published for the cluster
        float* myslot = slot + par * kDS;
#pragma unroll
        for (int t0r = 0; t0r < kDS; t0r += kDT / 16) {
            const int t = t0r + (tid >> 4), j = tid & 15;
            float s = 0.f;
#pragma unroll
            for (int c = 0; c < kDNP / 16; c++) s += lse[t * kDLL + c * 16 + j];
            s += __shfl_xor_sync(0xffffffffu, s, 8);
            s += __shfl_xor_sync(0xffffffffu, s, 4);
            s += __shfl_xor_sync(0xffffffffu, s, 2);
            s += __shfl_xor_sync(0xffffffffu, s, 1);
            if (j == 0) myslot[t] = ltch + kLn2 * s;
        }
        cluster.sync();
        // ---- P(t) and v_h(t) (identical arithmetic in every CTA of the cluster)
        if (tid < kDS) {
            float L[kMaxModels];
            float lmax = -INFINITY;
#pragma unroll
            for (int q = 0; q < kMaxModels; q++) {
                if (q < M) {
                    L[q] = cluster.map_shared_rank(myslot, q)[tid];
                    lmax = fmaxf(lmax, L[q]);
                }
            }
            float se = 0.f;
#pragma unroll
            for (int q = 0; q < kMaxModels; q++)
                if (q < M) se += ptx_ex2((L[q] - lmax) * kLog2e);
            const float P = lmax + kLn2 * ptx_lg2(se);
            const float Lh = myslot[tid];
            const float vh = ptx_ex2((Lh - P) * kLog2e);
            const int64_t tg = t0 + tid;
            const bool valid = tg < T && (a.keep == nullptr || a.keep[tg]);
            vS[tid] = valid ? vh : 0.f;
            if (valid) {
                dVs += (double)vh;
                if (h == 0) dLL += (double)P;
            }
            if (tg < T) {
                if (a.Lt_out) a.Lt_out[(size_t)h * T + tg] = Lh;
                if (a.P_out && h == 0) a.P_out[tg] = P;
            }
        }
        __syncthreads();
        // ---- phase 2: responsibilities, score function, sums; g of four
        // consecutive samples per 16-byte store into the operand image of the
        // Psi contraction (row = channel within its 128-channel half, column =
        // sample within its 32-sample block), rounded to TF32 (nearest, ties
        // away) so that the MMA reads it exactly; zero past T
        {
            const int rr = ch & 127, hc = ch >> 7;
            float* gblk = a.gout + (((size_t)tile * M + h) * 2 + hc) * 4096;
#pragma unroll 1
            for (int r4 = 0; r4 < kDS; r4 += 4) {
                float gq[4];
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    const int t = r4 + q;
                    const float v = vS[t];
                    float g = 0.f;
                    if (v != 0.f) {   // the same for every thread of the warp
                        const float nl = -lse[t * kDLL + ch];
                        const float bx = bst[t * kDNP + ch];   // v != 0: t0 + t < T
                        float2 g2 = make_float2(0.f, 0.f);
                        float g1 = 0.f;
#pragma unroll
                        for (int qq = 0; qq < NPR; qq++) da_pair(P2[qq], bx, nl, v, fP[qq], g2);
                        if constexpr (kOdd) da_one(P1, bx, nl, v, fS1, g1);
                        g = (g2.x + g2.y) + g1;
                        const float bb = bx - wci;
                        fCn = fmaf(v, bb, fCn);   // sum v b; cnew = A sum(v b) / vsum + c
                        fS2 = fmaf(v * bb, bb, fS2);
                        fGs += ch_ok ? g : 0.f;
                    }
                    gq[q] = (ch_ok && t0 + t < T) ? tf32_rna_alu(g) : 0.f;
                }
                *reinterpret_cast<float4*>(gblk + sw128_off(rr, r4, 128) / 4) =
                    make_float4(gq[0], gq[1], gq[2], gq[3]);
            }
        }
        if ((it + 1) % kFlush == 0) flush();
        __syncthreads();   // lse and v are rewritten by the next tile
    }
    flush();
    // a copy that a timed-out wait left in flight must land before the CTA exits
    if (tid == 0)
        for (int q = 0; q < 2; q++)
            if ((pend >> q) & 1u) mbar_wait(&bar[q], (pendpar >> q) & 1u, abort_flag, a.err, false, false);
    __syncthreads();

    // ---- this cluster's partial sums for model h: each channel's running sums
    // (read at L2, where the adds were made) mapped to the statistics
    if (ch_ok) {
        auto col = [&](int k) { return __ldcg(run + (size_t)k * n); };
#pragma unroll 1
        for (int j = 0; j < MM; j++) {
            const float rho = a.mp[((size_t)h * MM + j) * kDNP + ch].rho;
            double s[7];
            mix_stats_from_sums(col(0 * MM + j), col(1 * MM + j), col(2 * MM + j), col(3 * MM + j),
                                col(4 * MM + j), col(5 * MM + j), col(6 * MM + j), rho, a.grad_mode,
                                a.update_rho, s[kUs], s[kKn], s[kLn], s[kMn], s[kMd], s[kBd], s[kRn]);
#pragma unroll
            for (int k = 0; k < 7; k++) out[L.mix(k) + j * n + ch] = s[k];
        }
        out[L.cn() + ch] = col(7 * MM + 0);
        out[L.s2() + ch] = col(7 * MM + 1);
        out[L.gs() + ch] = col(7 * MM + 2);
    }
    // LL numerator and vsum: the per-sample threads' sums in a fixed order
    double* red = reinterpret_cast<double*>(lse);
    if (tid < kDS) { red[tid] = dLL; red[kDS + tid] = dVs; }
    __syncthreads();
    if (tid == 0) {
        double s0 = 0.0, s1 = 0.0;
        for (int t = 0; t < kDS; t++) { s0 += red[t]; s1 += red[kDS + t]; }
        out[0] = s0;
        out[1] = s1;
    }
    // Psi is summed by the contraction after this kernel into the first slot
    // (the running sums in its place are read: the barrier above)
    for (int e = tid; e < n * n; e += kDT) out[L.psi() + e] = 0.0;
    // peers may still read this CTA's slots: leave together
    cluster.sync();
}

template <int MM>
cudaError_t dens_config(int M, int nclusters, cudaStream_t st, cudaLaunchConfig_t& cfg,
                        cudaLaunchAttribute* attr) {
    using Sh = DensShape<MM>;
    auto kern = estep_dens_kernel<MM>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Sh::bytes);
    if (e != cudaSuccess) return e;
    cfg = {};
    cfg.gridDim = dim3(nclusters * M);
    cfg.blockDim = dim3(kDT);
    cfg.dynamicSmemBytes = Sh::bytes;
    cfg.stream = st;
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = M;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaSuccess;
}

template <int MM>
int dens_max_clusters_m(int M) {
    cudaLaunchConfig_t cfg;
    cudaLaunchAttribute attr[1];
    if (dens_config<MM>(M, 64, nullptr, cfg, attr) != cudaSuccess) return -1;
    int num = 0;
    if (cudaOccupancyMaxActiveClusters(&num, estep_dens_kernel<MM>, &cfg) != cudaSuccess) {
        cudaGetLastError();
        return -1;
    }
    return num;
}

template <int MM>
cudaError_t launch_dens_m(const EStepArgs& a, int nclusters, cudaStream_t st) {
    cudaLaunchConfig_t cfg;
    cudaLaunchAttribute attr[1];
    cudaError_t e = dens_config<MM>(a.M, nclusters, st, cfg, attr);
    if (e != cudaSuccess) return e;
    return cudaLaunchKernelEx(&cfg, estep_dens_kernel<MM>, a);
}

}  // namespace

namespace amica {

int dens_tile_samples() { return kDS; }

// Largest cluster count whose clusters (M CTAs, one per SM) are all resident.
int dens_max_clusters(int m, int M) {
    if (M < 1 || M > kMaxModels) return -1;
    switch (m) {
        case 1: return dens_max_clusters_m<1>(M);
        case 2: return dens_max_clusters_m<2>(M);
        case 3: return dens_max_clusters_m<3>(M);
        case 4: return dens_max_clusters_m<4>(M);
        case 5: return dens_max_clusters_m<5>(M);
        default: return -1;
    }
}

cudaError_t launch_estep_dens(const EStepArgs& a, int nclusters, cudaStream_t st) {
    if (!a.bext || !a.gout || a.ldb < a.M * kDNP || a.n > kDNP || a.M < 1 || a.M > kMaxModels ||
        nclusters < 1)
        return cudaErrorInvalidValue;
    switch (a.m) {
        case 1: return launch_dens_m<1>(a, nclusters, st);
        case 2: return launch_dens_m<2>(a, nclusters, st);
        case 3: return launch_dens_m<3>(a, nclusters, st);
        case 4: return launch_dens_m<4>(a, nclusters, st);
        case 5: return launch_dens_m<5>(a, nclusters, st);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace amica
