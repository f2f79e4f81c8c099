// Plain FP32 form of the fused AMICA E-step (SIMT FP32 contractions).
//
// One thread-block cluster per sample tile stream; CTA rank h of the cluster
// owns model h (cluster size = M).  Per tile of S samples each CTA:
//   1. stages the x tile in shared memory and computes b = W_h x on the FP32
//      pipe (register-blocked SIMT GEMM, W_h resident in shared memory);
//   2. evaluates the generalized-Gaussian mixture log-densities and the
//      log-sum-exp over mixtures per (channel, sample) -- the work of
//      betabyxminusmu / logalogblogpfun / updateltz (src/kernels.cu:251-366);
//   3. reduces over channels to Lt_h(t) and exchanges Lt over distributed
//      shared memory so that every CTA forms P(t) and v_h(t) (updatell,
//      src/kernels.cu:376-450) without touching global memory;
//   4. accumulates the sufficient statistics of src/kernels.cu:473-827 in
//      registers and Psi_h += g x^T (the sum behind phi = g b^T of
//      src/amica.cu:1535-1550, with phi formed from Psi in the FP64 M-step).
// Partial sums go to a per-CTA slot of `partial`; a separate kernel reduces
// the slots in a fixed order, so results are deterministic.
#include <cooperative_groups.h>
#include <cstdio>

#include <algorithm>

#include "common.cuh"
#include "density.cuh"

namespace cg = cooperative_groups;
using namespace amica;

namespace {

constexpr int kThreads = 256;
constexpr int kS = 64;  // samples per tile

// NP: channels padded (32, 64, 128 or 256).  Up to 128 channels one CTA per
// model holds them all; at 256 the Q = 4 CTAs of a model each own NPL = 64
// channels (their rows of W, their densities, their rows of Psi) and read the
// full x tile; their per-sample channel sums are added in the cluster.
template <int NP>
struct PlainShape {
    static constexpr int NPL = NP <= 128 ? NP : 64; // channels of this CTA
    static constexpr int Q = NP / NPL;              // CTAs per model
    static constexpr int SPLIT = kThreads / NPL;    // sample groups per channel
    static constexpr int SUB = kS / SPLIT;          // samples per thread per tile
    static constexpr int WLD = NPL + 4;             // padded row of W^T in smem
    static constexpr int XLD = NP + 4;              // padded row of the x tile
    // GEMM b = W x: each thread 4 channels x CT samples
    static constexpr int NTI = NPL / 4;
    static constexpr int NTT = kThreads / NTI;
    static constexpr int CT = kS / NTT;
    static_assert(NTI * NTT == kThreads && NTT * CT == kS, "b = W x tiling");
    // Psi update: each thread RI x RK block
    static constexpr int RI = NPL / 16;
    static constexpr int RK = NP / 16;
    static constexpr int LLD = NPL + 1;             // padded row of the lse tile
    static constexpr size_t smem_floats =
        (size_t)NP * WLD + (size_t)kS * XLD + (size_t)kS * NPL + (size_t)kS * LLD +
                  (size_t)kS * LLD + 2 * kS + 2 * kS;
};

template <int NP, int MM>
__global__ void __launch_bounds__(kThreads, 1) estep_plain_kernel(EStepArgs a) {
    using Sh = PlainShape<NP>;
    constexpr int NPL = Sh::NPL, Q = Sh::Q;
    extern __shared__ __align__(16) float sm[];
    float* Wt = sm;                                   // [NP][WLD]  Wt[k][i] = W[i0 + i][k]
    float* xs = Wt + NP * Sh::WLD;                   // [S][XLD]
    float* bs = xs + kS * Sh::XLD;                   // [S][NPL]   (W x)_i per sample
    float* gs = bs + kS * NPL;                        // [S][NPL] g; its region is [S][LLD]
    float* lse = gs + kS * Sh::LLD;                 // [S][LLD]   log-sum-exp over mixtures
    float* slot = lse + kS * Sh::LLD;                 // [2][S]     cluster-visible L_h(t)
    float* vS = slot + 2 * kS;                        // [S]        v_h(t) (0 if not used)

    cg::cluster_group cluster = cg::this_cluster();
    const int rank = (int)cluster.block_rank();
    const int h = rank / Q, cq = rank % Q;            // model, channel block
    const int i0c = cq * NPL;                         // first channel of this CTA
    const int cid = blockIdx.x / (a.M * Q);
    const int tid = threadIdx.x;
    const int n = a.n, M = a.M;
    if (a.m != MM || n > NP) {
        if (tid == 0) atomicOr(a.err, kErrShape);
    }

    // ---- resident per-CTA data: W_h^T and this thread's mixture constants
    {
        const float* Wh = a.Wf + ((size_t)h * NP + i0c) * NP;
        for (int e = tid; e < NPL * NP; e += kThreads) {
            int i = e / NP, k = e % NP;
            Wt[k * Sh::WLD + i] = Wh[e];
        }
    }
    const int ch = tid % NPL;           // density-phase channel (of this CTA)
    const int grp = tid / NPL;          // density-phase sample group
    const int gch = i0c + ch;           // the channel's index in the model
    const bool ch_ok = gch < n;
    // mixtures (0,1), (2,3) as float2 pairs, an odd last one as a scalar
    constexpr int NPR = MM / 2;
    constexpr bool kOdd = (MM & 1) != 0;
    constexpr int NPRA = NPR > 0 ? NPR : 1;
    float pr[MM];
    MixV<float2> P2[NPRA];
    MixV<float> P1;
#pragma unroll
    for (int j = 0; j < MM; j++) {
        const MixParam q = a.mp[((size_t)h * MM + j) * NP + gch];
        pr[j] = q.rho;
        if (j < 2 * NPR) {
            float2* f[5] = {&P2[j / 2].s, &P2[j / 2].npo, &P2[j / 2].pc, &P2[j / 2].pr, &P2[j / 2].sr};
            const float vals[5] = {q.s, -q.off, q.cl2, q.rho, q.s * q.rho};
#pragma unroll
            for (int e = 0; e < 5; e++) {
                if (j & 1) f[e]->y = vals[e];
                else f[e]->x = vals[e];
            }
        } else {
            P1.s = q.s; P1.npo = -q.off; P1.pc = q.cl2; P1.pr = q.rho; P1.sr = q.s * q.rho;
        }
    }
    const float wci = a.wc[(size_t)h * NP + gch];
    float ltc[kMaxModels];
#pragma unroll
    for (int q = 0; q < kMaxModels; q++) ltc[q] = (q < M) ? (float)(a.ltc64[q] - a.ltc64[0]) : 0.f;

    // FP64 running sums for this thread's channel: A0..A6 of dens_acc per mixture
    double dA[7][MM];
#pragma unroll
    for (int k = 0; k < 7; k++)
#pragma unroll
        for (int j = 0; j < MM; j++) dA[k][j] = 0.0;
    double dCn = 0.0, dS2 = 0.0, dGs = 0.0;
    double dLL = 0.0, dVs = 0.0;   // per-sample threads (tid < S)
    constexpr int PRI = Sh::RI, PRK = Sh::RK;
    float psi[PRI][PRK];
#pragma unroll
    for (int r = 0; r < PRI; r++)
#pragma unroll
        for (int c = 0; c < PRK; c++) psi[r][c] = 0.f;

    int par = 0;
    for (int tile = cid; tile < a.ntiles; tile += a.nclusters, par ^= 1) {
        const int64_t t0 = (int64_t)tile * kS;
        {
        // ---- stage the x tile (float4, coalesced; rows past T are zero)
        for (int e = tid; e < kS * (NP / 4); e += kThreads) {
            int t = e / (NP / 4), k4 = e % (NP / 4);
            float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
            if (t0 + t < a.T) v = reinterpret_cast<const float4*>(a.x + (t0 + t) * a.ldx)[k4];
            *reinterpret_cast<float4*>(xs + t * Sh::XLD + 4 * k4) = v;
        }
        __syncthreads();
        // ---- b = W_h x  (thread: channels 4*ti..+3, samples tt*CT..+CT-1)
        {
            const int ti = tid % Sh::NTI, tt = tid / Sh::NTI;
            float acc[Sh::CT][4];
#pragma unroll
            for (int c = 0; c < Sh::CT; c++)
#pragma unroll
                for (int q = 0; q < 4; q++) acc[c][q] = 0.f;
#pragma unroll 2
            for (int k = 0; k < NP; k += 4) {
                float4 w0 = *reinterpret_cast<const float4*>(Wt + (k + 0) * Sh::WLD + 4 * ti);
                float4 w1 = *reinterpret_cast<const float4*>(Wt + (k + 1) * Sh::WLD + 4 * ti);
                float4 w2 = *reinterpret_cast<const float4*>(Wt + (k + 2) * Sh::WLD + 4 * ti);
                float4 w3 = *reinterpret_cast<const float4*>(Wt + (k + 3) * Sh::WLD + 4 * ti);
#pragma unroll
                for (int c = 0; c < Sh::CT; c++) {
                    float4 xv = *reinterpret_cast<const float4*>(xs + (tt * Sh::CT + c) * Sh::XLD + k);
                    acc[c][0] = fmaf(w0.x, xv.x, acc[c][0]); acc[c][1] = fmaf(w0.y, xv.x, acc[c][1]);
                    acc[c][2] = fmaf(w0.z, xv.x, acc[c][2]); acc[c][3] = fmaf(w0.w, xv.x, acc[c][3]);
                    acc[c][0] = fmaf(w1.x, xv.y, acc[c][0]); acc[c][1] = fmaf(w1.y, xv.y, acc[c][1]);
                    acc[c][2] = fmaf(w1.z, xv.y, acc[c][2]); acc[c][3] = fmaf(w1.w, xv.y, acc[c][3]);
                    acc[c][0] = fmaf(w2.x, xv.z, acc[c][0]); acc[c][1] = fmaf(w2.y, xv.z, acc[c][1]);
                    acc[c][2] = fmaf(w2.z, xv.z, acc[c][2]); acc[c][3] = fmaf(w2.w, xv.z, acc[c][3]);
                    acc[c][0] = fmaf(w3.x, xv.w, acc[c][0]); acc[c][1] = fmaf(w3.y, xv.w, acc[c][1]);
                    acc[c][2] = fmaf(w3.z, xv.w, acc[c][2]); acc[c][3] = fmaf(w3.w, xv.w, acc[c][3]);
                }
            }
#pragma unroll
            for (int c = 0; c < Sh::CT; c++)
                *reinterpret_cast<float4*>(bs + (tt * Sh::CT + c) * NPL + 4 * ti) =
                    make_float4(acc[c][0], acc[c][1], acc[c][2], acc[c][3]);
        }
        }
        __syncthreads();
        // ---- phase 1: per (channel, sample) log-sum-exp over mixtures (log2 units)
#pragma unroll 4
        for (int r = 0; r < Sh::SUB; r++) {
            const int t = grp * Sh::SUB + r;
            const float bx = bs[t * NPL + ch];
            float q[MM];
#pragma unroll
            for (int qq = 0; qq < NPR; qq++) {
                float2 L2;
                const float2 q2 = dens_q(P2[qq], bx, L2);
                q[2 * qq] = q2.x; q[2 * qq + 1] = q2.y;
            }
            if constexpr (kOdd) {
                float L2;
                q[MM - 1] = dens_q(P1, bx, L2);
            }
            lse[t * Sh::LLD + ch] = ch_ok ? lse2<MM>(q) : 0.f;
        }
        __syncthreads();
        // ---- Lt_h(t): channel sum in fixed order, published for the cluster
        // (with Q > 1, this CTA's channels only; the blocks are added below)
        float* myslot = slot + par * kS;
        if (tid < kS) {
            float s = 0.f;
            if constexpr (Q == 1) {
                for (int i = 0; i < n; i++) s += lse[tid * Sh::LLD + i];
                myslot[tid] = ltc[h] + kLn2 * s;
            } else {
                for (int i = 0; i < NPL; i++) s += lse[tid * Sh::LLD + i];
                myslot[tid] = s;
            }
        }
        cluster.sync();
        // ---- P(t) and v_h(t) (identical arithmetic in every CTA of the cluster)
        if (tid < kS) {
            float L[kMaxModels];
            float lmax = -INFINITY;
#pragma unroll
            for (int q = 0; q < kMaxModels; q++) {
                if (q < M) {
                    if constexpr (Q == 1) {
                        const float* ps_q = cluster.map_shared_rank(myslot, q);
                        L[q] = ps_q[tid];
                    } else {
                        float s = 0.f;
#pragma unroll
                        for (int b = 0; b < Q; b++) s += cluster.map_shared_rank(myslot, q * Q + b)[tid];
                        L[q] = ltc[q] + kLn2 * s;
                    }
                    lmax = fmaxf(lmax, L[q]);
                }
            }
            float se = 0.f;
#pragma unroll
            for (int q = 0; q < kMaxModels; q++)
                if (q < M) se += ptx_ex2((L[q] - lmax) * kLog2e);
            const float P = lmax + kLn2 * ptx_lg2(se);
            const float vh = ptx_ex2((L[h] - P) * kLog2e);
            const int64_t tg = t0 + tid;
            const bool valid = tg < a.T && (a.keep == nullptr || a.keep[tg]);
            vS[tid] = valid ? vh : 0.f;
            if (valid && cq == 0) {
                dVs += (double)vh;
                if (h == 0) dLL += (double)P;
            }
            if (tg < a.T && cq == 0) {
                if (a.Lt_out) a.Lt_out[(size_t)h * a.T + tg] = L[h];
                if (a.P_out && h == 0) a.P_out[tg] = P;
            }
        }
        __syncthreads();
        // ---- phase 2: responsibilities, score function and sufficient statistics
        {
            float2 fP[NPRA][7];
            float fS1[7];
#pragma unroll
            for (int k = 0; k < 7; k++) {
#pragma unroll
                for (int qq = 0; qq < NPRA; qq++) fP[qq][k] = make_float2(0.f, 0.f);
                fS1[k] = 0.f;
            }
            float fCn = 0.f, fS2 = 0.f, fGs = 0.f;
            // the densities, responsibilities and sums of tile sample t; returns g
            auto sample = [&](int t) -> float {
                const float v = vS[t];
                // a sample whose model responsibility is exactly 0 adds exactly 0
                // to every sum and to g (v is the same in every lane of the warp)
                if (v == 0.f) return 0.f;
                const float bx = bs[t * NPL + ch];
                const float nl = -lse[t * Sh::LLD + ch];
                float2 g2 = make_float2(0.f, 0.f);
                float g1 = 0.f;
#pragma unroll
                for (int qq = 0; qq < NPR; qq++)
                    dens_acc<float2, false>(P2[qq], bx, make_float2(0.f, 0.f), nl, v, fP[qq], g2);
                if constexpr (kOdd) dens_acc<float, false>(P1, bx, 0.f, nl, v, fS1, g1);
                const float g = (g2.x + g2.y) + g1;
                const float bb = bx - wci;
                fCn = fmaf(v, bb, fCn);          // sum v b; cnew = A sum(v b) / vsum + c
                fS2 = fmaf(v * bb, bb, fS2);
                fGs += ch_ok ? g : 0.f;
                return g;
            };
            {
#pragma unroll 2
                for (int r = 0; r < Sh::SUB; r++) {
                    const int t = grp * Sh::SUB + r;
                    const float g = sample(t);
                    gs[t * NPL + ch] = ch_ok ? g : 0.f;
                }
            }
            if (ch_ok) {
#pragma unroll
                for (int k = 0; k < 7; k++) {
#pragma unroll
                    for (int qq = 0; qq < NPR; qq++) {
                        dA[k][2 * qq] += fP[qq][k].x;
                        dA[k][2 * qq + 1] += fP[qq][k].y;
                    }
                    if constexpr (kOdd) dA[k][MM - 1] += fS1[k];
                }
                dCn += fCn; dS2 += fS2; dGs += fGs;
            }
        }
        __syncthreads();
        // ---- Psi_h += g x^T over the tile (thread: RI x RK block)
        {
            const int pi = tid % 16, pk = tid / 16;
            const int i0 = pi * Sh::RI, k0 = pk * Sh::RK;
#pragma unroll 4
            for (int t = 0; t < kS; t++) {
                float gv[Sh::RI], xv[Sh::RK];
#pragma unroll
                for (int r = 0; r < Sh::RI; r++) gv[r] = gs[t * NPL + i0 + r];
#pragma unroll
                for (int c = 0; c < Sh::RK; c++) xv[c] = xs[t * Sh::XLD + k0 + c];
#pragma unroll
                for (int r = 0; r < Sh::RI; r++)
#pragma unroll
                    for (int c = 0; c < Sh::RK; c++) psi[r][c] = fmaf(gv[r], xv[c], psi[r][c]);
            }
        }
        __syncthreads();
    }

    // ---- write this CTA's partial sums (fixed-order combination of groups)
    PartLayout L{n, MM};
    // one slot per (cluster, channel block); entries of the other blocks stay zero
    double* out = a.partial + ((size_t)(cid * Q + cq) * M + h) * L.stride();
    double* red = reinterpret_cast<double*>(xs);   // [SPLIT][NPL] doubles, one statistic at a time
    constexpr int NACC = 7 * MM + 3;
    double vals[NACC];
#pragma unroll
    for (int j = 0; j < MM; j++) {
        mix_stats_from_sums(dA[0][j], dA[1][j], dA[2][j], dA[3][j], dA[4][j], dA[5][j], dA[6][j],
                            pr[j], a.grad_mode, a.update_rho, vals[kUs * MM + j], vals[kKn * MM + j],
                            vals[kLn * MM + j], vals[kMn * MM + j], vals[kMd * MM + j],
                            vals[kBd * MM + j], vals[kRn * MM + j]);
    }
    vals[7 * MM + 0] = dCn; vals[7 * MM + 1] = dS2; vals[7 * MM + 2] = dGs;
#pragma unroll
    for (int k = 0; k < NACC; k++) {
        red[grp * NPL + ch] = vals[k];
        __syncthreads();
        if (tid < NPL && i0c + tid < n) {
            double s = 0.0;
            for (int g2 = 0; g2 < Sh::SPLIT; g2++) s += red[g2 * NPL + tid];
            const int gi = i0c + tid;
            int dst;
            if (k < 7 * MM) dst = L.mix(k / MM) + (k % MM) * n + gi;
            else if (k == 7 * MM) dst = L.cn() + gi;
            else if (k == 7 * MM + 1) dst = L.s2() + gi;
            else dst = L.gs() + gi;
            out[dst] = s;
        }
        __syncthreads();
    }
    // LL numerator and vsum: per-sample threads, combined in fixed order
    double* red2 = red;
    if (tid < kS) { red2[tid] = dLL; red2[kS + tid] = dVs; }
    __syncthreads();
    if (tid == 0 && cq == 0) {
        double s0 = 0.0, s1 = 0.0;
        for (int t = 0; t < kS; t++) { s0 += red2[t]; s1 += red2[kS + t]; }
        out[0] = s0;
        out[1] = s1;
    }
    {
        const int pi = tid % 16, pk = tid / 16;
        const int i0 = pi * Sh::RI, k0 = pk * Sh::RK;
#pragma unroll
        for (int r = 0; r < Sh::RI; r++)
#pragma unroll
            for (int c = 0; c < Sh::RK; c++) {
                const int i = i0c + i0 + r, k = k0 + c;
                if (i < n && k < n) out[L.psi() + (size_t)k * n + i] = (double)psi[r][c];
            }
    }
    // peers may still read this CTA's slots: leave together
    cluster.sync();
}

template <int NP, int MM>
cudaError_t launch_plain(const EStepArgs& a, int nclusters, cudaStream_t st) {
    using Sh = PlainShape<NP>;
    const size_t smem = Sh::smem_floats * sizeof(float);
    auto kern = estep_plain_kernel<NP, MM>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    if (a.M * Sh::Q > 1) {
        e = cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
        if (e != cudaSuccess) return e;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(nclusters * a.M * Sh::Q);
    cfg.blockDim = dim3(kThreads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = a.M * Sh::Q;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kern, a);
}

}  // namespace

namespace amica {

int plain_tile_samples() { return kS; }

int plain_pad_channels(int n) {
    return n <= 32 ? 32 : (n <= 64 ? 64 : (n <= 128 ? 128 : (n <= 256 ? 256 : -1)));
}
// Partial-sum slots per cluster: one per channel block.
int plain_partial_groups(int n) { return plain_pad_channels(n) == 256 ? PlainShape<256>::Q : 1; }

// Largest cluster count whose clusters can all be resident at once (the grid
// is persistent: every cluster loops over its share of the tiles).
template <int NP, int MM>
int max_active_clusters(int M) {
    using Sh = PlainShape<NP>;
    const size_t smem = Sh::smem_floats * sizeof(float);
    auto kern = estep_plain_kernel<NP, MM>;
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return -1;
    const int csize = M * Sh::Q;
    if (csize > 8 &&
        cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess)
        return -1;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(csize * 64);
    cfg.blockDim = dim3(kThreads);
    cfg.dynamicSmemBytes = smem;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = csize;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int num = 0;
    if (cudaOccupancyMaxActiveClusters(&num, kern, &cfg) != cudaSuccess) {
        cudaGetLastError();
        return -1;
    }
    return num;
}

int plain_max_clusters(int n, int m, int M) {
    const int NP = plain_pad_channels(n);
    if (NP < 0 || m < 1 || m > 5 || M < 1 || M > kMaxModels) return -1;
#define AMICA_PLAIN_OCC(NPV, MMV) \
    if (NP == NPV && m == MMV) return max_active_clusters<NPV, MMV>(M);
#define AMICA_PLAIN_OCC_NP(NPV) \
    AMICA_PLAIN_OCC(NPV, 1) AMICA_PLAIN_OCC(NPV, 2) AMICA_PLAIN_OCC(NPV, 3) \
    AMICA_PLAIN_OCC(NPV, 4) AMICA_PLAIN_OCC(NPV, 5)
    AMICA_PLAIN_OCC_NP(32)
    AMICA_PLAIN_OCC_NP(64)
    AMICA_PLAIN_OCC_NP(128)
    AMICA_PLAIN_OCC_NP(256)
#undef AMICA_PLAIN_OCC_NP
#undef AMICA_PLAIN_OCC
    return -1;
}

cudaError_t launch_estep_plain(const EStepArgs& a, int NP, int nclusters, cudaStream_t st) {
#define AMICA_PLAIN_CASE(NPV, MMV) \
    if (NP == NPV && a.m == MMV) return launch_plain<NPV, MMV>(a, nclusters, st);
#define AMICA_PLAIN_NP(NPV) \
    AMICA_PLAIN_CASE(NPV, 1) AMICA_PLAIN_CASE(NPV, 2) AMICA_PLAIN_CASE(NPV, 3) \
    AMICA_PLAIN_CASE(NPV, 4) AMICA_PLAIN_CASE(NPV, 5)
    AMICA_PLAIN_NP(32)
    AMICA_PLAIN_NP(64)
    AMICA_PLAIN_NP(128)
    AMICA_PLAIN_NP(256)
#undef AMICA_PLAIN_NP
#undef AMICA_PLAIN_CASE
    return cudaErrorInvalidValue;
}

// the split mixed form (128 < n <= 256) runs its density-only kernel on the
// channels this form pads to 256
bool split_form_supported(int n) { return plain_pad_channels(n) == 256; }

}  // namespace amica

namespace {

// W_hi = tf32(W) (round to nearest, ties away: the low 13 bits zero, so the
// MMA's reading of it as TF32 keeps it exactly) and W_lo = W - W_hi.
__global__ void k_split_w(const float* __restrict__ Wf, float* __restrict__ whi, float* __restrict__ wlo,
                          int64_t len) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < len; e += (int64_t)gridDim.x * blockDim.x) {
        const float w = Wf[e];
        float hi = w;
        if (isfinite(w)) hi = __uint_as_float((__float_as_uint(w) + 0x1000u) & 0xffffe000u);
        whi[e] = hi;
        wlo[e] = w - hi;
    }
}

}  // namespace

namespace amica {

cudaError_t launch_split_w(const float* Wf, float* whi, float* wlo, int64_t len, cudaStream_t st) {
    k_split_w<<<(int)std::min<int64_t>((len + 255) / 256, 1184), 256, 0, st>>>(Wf, whi, wlo, len);
    return cudaGetLastError();
}

}  // namespace amica
