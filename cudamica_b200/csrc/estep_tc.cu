// Mixed-precision fused AMICA E-step on the 5th-generation tensor cores
// (tcgen05, TF32 operands, FP32 accumulation in tensor memory).
//
// Cluster of M CTAs, CTA rank h = model h; persistent over tiles of 48 rows of
// the data (a row is one sample, or R samples side by side when n <= 64: see
// "Lane packing" below).
//   warp 12 (control; warps 13-15 of its warpgroup idle, so that setmaxnreg
//     can move registers to the density warpgroups): TMA loads of the x tile
//     (128B-swizzled, two stages),
//     and the two contractions issued by one thread:
//       MMA1  b_h = W_hi x^T + W_lo x^T   M=128 (lanes) N=48 (rows) K=128
//             W_hi = tf32(W_h) K-major in smem, W_lo = tf32(W_h - W_hi) in TMEM,
//             B = x tile (K-major, TMA), D -> TMEM (2 buffers)
//       MMA2  phi_h += G B^T            M=128 N=128 K=48
//             A = G, B = the b tile, both K-major tiles written by the density
//             warps, D -> TMEM for the CTA's life
//   warps 0-11 (3 warpgroups x 4 warps): thread = (TMEM lane, warpgroup =
//     16-row slice).  Each reads its b values with tcgen05.ld, evaluates the
//     generalized-Gaussian mixture densities and the log-sum-exp over
//     mixtures (FP32, MUFU ex2/lg2), reduces over channels with warp shuffles,
//     exchanges the per-sample Lt_h(t) with the other models' CTAs through
//     distributed shared memory (st.async onto the peers' mbarriers), forms
//     P(t) and v_h(t), accumulates the sufficient statistics and writes
//     g = sum_j sqrt(beta) u f' and b = W (x - c) into the MMA2 operand tiles.
// (An MN-major TF32 operand needs the 32-byte-atom 128B swizzle, which the
// x tile cannot have while it is also MMA1's K-major operand; so the second
// contraction is phi = g b^T from two thread-written K-major tiles.)
// The work of src/kernels.cu:227-827 and both cuBLAS Dgemm of the reference's
// block loop (src/amica.cu:1054-1069, :1535-1550) happens in this one kernel.
//
// Every mbarrier wait is bounded (~1 s); on expiry the kernel records
// kErrWaitTimeout, stops waiting, frees its tensor memory and exits.
#include <cooperative_groups.h>
#include <cuda.h>
#include <cstdint>

#include "common.cuh"
#include "density.cuh"
#include "tc_ptx.cuh"

namespace cg = cooperative_groups;
using namespace amica;

namespace {

template <int V>
struct IntC {
    static constexpr int value = V;
};

constexpr int kS = 48;                  // samples per tile (MMA1 N)
constexpr int kWG = 3;                  // density warpgroups
constexpr int kDensWarps = 4 * kWG;     // 12
constexpr int kThreads = (kDensWarps + 4) * 32;   // + one control warpgroup
// Register split (setmaxnreg, per warpgroup): launched at 128 per thread
// (512 x 128 = 65536), the control warpgroup drops to 96 (its unrolled MMA
// issue needs about 80) and the three density warpgroups rise to 136:
// 3 x 128 x 136 + 128 x 96 = 64512.  Measured at n=128, T=1M, M=3, m=3:
// 136 beats 128 (no split, 3.37 ms), 144, 152 and 160 (3.18 against 3.24-3.41 ms).
constexpr int kCtlRegs = 96;
constexpr int kDensRegs = 136;
static_assert(3 * 128 * kDensRegs + 128 * kCtlRegs <= kThreads * 128, "register split");
constexpr int kSub = kS / kWG;          // 16 samples per thread per tile
constexpr int kBcol = 64;               // TMEM column stride of the two b buffers
constexpr int kPsiCol = 128;            // TMEM column of phi (N = NP columns)
constexpr int kWloCol = 256;            // TMEM columns of W_lo, the A operand of the low MMA1 half
// tiles between FP32 -> FP64 flushes: 16 tiles, 256 samples per thread (128
// per half of each FP32x2 sum); 2.72 ms per E-step at n=128, T=1M, M=3, m=3
// against 2.77 ms with 8
constexpr int kFlush = 16;

// Tensor-memory column of chunk c (kSub columns) of the log2|y| cache: the
// 16-column gaps after the two b buffers when a chunk fits there, then the 128
// columns after W_lo.
constexpr int kL2Gap = kSub <= 16 ? 2 : 0;
constexpr int kL2Chunks = kL2Gap + 128 / kSub;
__device__ __forceinline__ uint32_t l2_chunk_col(int c) {
    if (kL2Gap && c < kL2Gap) return c == 0 ? 48u : 112u;
    return 384u + (uint32_t)(kSub * (c - kL2Gap));
}

// SPLIT: the form with the split correction of phi (one x stage; the G and b
// tiles twice as wide, their low parts in columns [kS, 2 kS)).
template <int NP, bool SPLIT = false>
struct TcShape {
    static constexpr int KB = NP / 32;                       // 128-B column blocks of x / W
    static constexpr int NSTAGE = SPLIT ? 1 : 2;             // x stages
    static constexpr int TCOLS = SPLIT ? 2 * kS : kS;        // columns of the G / b tiles
    static constexpr uint32_t W_BYTES = 128u * NP * 4u;      // 128 rows x NP
    static constexpr uint32_t X_BYTES = (uint32_t)kS * NP * 4u;
    static constexpr uint32_t G_BYTES = 128u * 128u * ((TCOLS + 31) / 32);   // 128 rows x 32-column blocks
    static constexpr uint32_t OFF_W = 0;
    static constexpr uint32_t OFF_X0 = OFF_W + W_BYTES;
    static constexpr uint32_t OFF_G = OFF_X0 + NSTAGE * X_BYTES;
    static constexpr uint32_t OFF_BT = OFF_G + G_BYTES;                  // b tile, same layout as G
    // per-warp channel sums of Lt from every model's CTA: [2][8 models][4 warps][kS] f32
    static constexpr uint32_t OFF_SLOT = OFF_BT + G_BYTES;
    static constexpr uint32_t OFF_LSE = OFF_SLOT + 2 * kMaxModels * 4 * kS * 4;  // [WG][kSub][128] f32
    static constexpr uint32_t OFF_V = OFF_LSE + kWG * kSub * 128 * 4;       // [warp][kSub] f32
    static constexpr uint32_t OFF_BAR = OFF_V + kDensWarps * kSub * 4;
    static constexpr uint32_t NBAR = 32;
    static constexpr uint32_t OFF_MISC = OFF_BAR + NBAR * 8;
    // per density warp: the models' log-likelihood offsets ltc_q - ltc_0 (FP32)
    static constexpr uint32_t OFF_LC = OFF_MISC + 64;
    static constexpr uint32_t BYTES = OFF_LC + kDensWarps * kMaxModels * 4;
    static constexpr uint32_t TMEM_COLS = 512;   // b: [0,48) [64,112); phi: [128,128+NP); W_lo: [256,256+NP);
                                                 // log2|y| cache: [48,64) [112,128) [384,512)
    static_assert(BYTES + 1024 <= 232448, "shared memory");
};

enum { BAR_FULL0 = 0, BAR_FULL1, BAR_EMPTY0, BAR_EMPTY1, BAR_BFULL0, BAR_BFULL1, BAR_BEMPTY0,
       BAR_BEMPTY1, BAR_GFULL, BAR_GEMPTY, BAR_PSI, BAR_DRAIN,
       BAR_LT0 /* 2 parities x kWG warpgroups: BAR_LT0 + par * kWG + wg */ };

// Lane packing: with npc (n padded to 32, 64 or 128) channels, the 128 TMEM
// lanes hold R = 128 / npc sample sets side by side.  The sphered data
// (T x npc floats, sample-major) is read as a (T / R) x 128 matrix whose row p
// holds samples pR .. pR + R - 1; W_h enters as the block-diagonal
// diag(W_h, ..., W_h), so lane r*npc + i of MMA1 yields b_i of sample pR + r.
// Lanes of set r sum over their own channels; the statistics of set r go to
// their own partial slots (folded with every other slot by the fixed-order
// reduction), and phi_h is the sum of the R diagonal blocks of g b^T.
struct TcArgs {
    EStepArgs e;
    int ngroups;   // partial slots per cluster: kWG per sample set, set-major
};

template <int NP, int MM, int R, bool SPLIT>
__global__ void __launch_bounds__(kThreads, 1)
    estep_tc_kernel(const __grid_constant__ CUtensorMap xmap, TcArgs ta) {
    using Sh = TcShape<NP, SPLIT>;
    const EStepArgs& a = ta.e;
    // Both forms are launched when the split correction can switch on during a
    // fit (the switch is a device-side flag, so that the iteration's graph does
    // not change); the one that does not match the flag leaves at once.
    if ((a.split_phi != nullptr && *a.split_phi != 0) != SPLIT) return;
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    // 1024-byte alignment for the swizzled operand tiles (pointer arithmetic on
    // the shared array, so that every pointer derived from it stays a shared
    // memory pointer and its accesses compile to shared loads and stores)
    uint8_t* sm = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
    float* Wsm = (float*)(sm + Sh::OFF_W);
    float* slot = (float*)(sm + Sh::OFF_SLOT);
    uint64_t* bar = (uint64_t*)(sm + Sh::OFF_BAR);
    uint32_t* tmem_holder = (uint32_t*)(sm + Sh::OFF_MISC);
    volatile int* abort_flag = (volatile int*)(sm + Sh::OFF_MISC + 8);

    cg::cluster_group cluster = cg::this_cluster();
    const int h = (int)cluster.block_rank();
    const int M = a.M, n = a.n;
    const int cid = blockIdx.x / M;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int ntile_local = (a.ntiles > cid) ? (a.ntiles - cid + a.nclusters - 1) / a.nclusters : 0;

    // ---- setup: barriers, W_h into the swizzled A tile, tensor memory
    if (tid == 0) {
        mbar_init(&bar[BAR_FULL0], 1);
        mbar_init(&bar[BAR_FULL1], 1);
        mbar_init(&bar[BAR_EMPTY0], 1);
        mbar_init(&bar[BAR_EMPTY1], 1);
        mbar_init(&bar[BAR_BFULL0], 1);
        mbar_init(&bar[BAR_BFULL1], 1);
        mbar_init(&bar[BAR_BEMPTY0], kDensWarps);
        mbar_init(&bar[BAR_BEMPTY1], kDensWarps);
        mbar_init(&bar[BAR_GFULL], kDensWarps);
        mbar_init(&bar[BAR_GEMPTY], 1);
        // one local arrival (with the expected bytes) per tile; the data comes by st.async
        for (int r = 0; r < 2 * kWG; r++) mbar_init(&bar[BAR_LT0 + r], 1);
        mbar_init(&bar[BAR_PSI], 1);
        mbar_init(&bar[BAR_DRAIN], 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    {
        // block-diagonal diag(W_h, ..., W_h) of R blocks of npc x npc; W[i][k]
        // row-major with stride npc, rows i >= n zero
        constexpr int npc = NP / R;
        const float* Wh = a.Wf + (size_t)h * npc * npc;
        for (int e4 = tid; e4 < 128 * (NP / 4); e4 += kThreads) {
            const int i = e4 / (NP / 4), k = (e4 % (NP / 4)) * 4;
            const int si = i / npc, sk = k / npc;
            float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
            if (si == sk)
                v = *reinterpret_cast<const float4*>(Wh + (size_t)(i - si * npc) * npc + (k - sk * npc));
            v.x = tf32_rna(v.x); v.y = tf32_rna(v.y); v.z = tf32_rna(v.z); v.w = tf32_rna(v.w);
            *reinterpret_cast<float4*>((uint8_t*)Wsm + sw128_off(i, k, 128)) = v;
        }
    }
    if (warp == kDensWarps) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     ::"r"(smem_u32(tmem_holder)), "r"(Sh::TMEM_COLS) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    fence_proxy_async();                 // W tile written by generic stores -> async proxy
    tc_fence_before();
    cluster.sync();                      // barriers of every CTA initialised before remote use
    tc_fence_after();
    const uint32_t tmem = *tmem_holder;
    const uint32_t tmem_b0 = tmem, tmem_psi = tmem + kPsiCol;
    // W_lo = W - tf32(W) into tensor memory (row i -> lane i): the A operand of the
    // second half of MMA1, so that b = W_hi x + W_lo x keeps W to ~2^-22
    if (warp < 4) {
        const int i = warp * 32 + lane;
        constexpr int npc = NP / R;
        const int si = i / npc;
        const float* Wrow = a.Wf + ((size_t)h * npc + (i - si * npc)) * npc;
#pragma unroll 1
        for (int k0 = 0; k0 < NP; k0 += 16) {
            float lo[16];
            const bool blk = (k0 / npc) == si;   // 16 columns never straddle a block
#pragma unroll
            for (int q = 0; q < 16; q++) {
                const float w = blk ? Wrow[k0 - si * npc + q] : 0.f;
                lo[q] = tf32_rna(w - tf32_rna(w));
            }
            tmem_st16(tmem + kWloCol + ((uint32_t)(warp * 32) << 16) + (uint32_t)k0, lo);
        }
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();

    if (warp >= kDensWarps) {
        // =========================== control warpgroup: TMA + MMA ================
        asm volatile("setmaxnreg.dec.sync.aligned.u32 %0;" ::"n"(kCtlRegs));
        if (warp == kDensWarps && lane == 0 && ntile_local > 0) {
            const CUtensorMap* item_map = &xmap;
            const int64_t item_tile0 = cid, item_stride = a.nclusters;
#include "tc_control_item.inc"
        }
        __syncwarp();
    } else {
        // =========================== density warps =================================
        asm volatile("setmaxnreg.inc.sync.aligned.u32 %0;" ::"n"(kDensRegs));
        const int64_t item_tile0 = cid, item_stride = a.nclusters;
        const int item_slot = cid, item_ngroups = ta.ngroups;
#include "tc_density_item.inc"
    }
    tc_fence_before();
    cluster.sync();
    if (warp == kDensWarps) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;"
                     ::"r"(tmem), "r"(Sh::TMEM_COLS) : "memory");
    }
}

// ---------------------------------------------------------------- cohort
// One persistent launch over the sample tiles of many single-model fits of the
// same m (a cohort of subjects with their own channel counts and lengths).  A
// work item is a run of consecutive tiles of one subject; CTA c (a cluster of
// one) processes items item_off[c] .. item_off[c + 1] - 1 in order.  Per item
// the control warpgroup re-arms the barriers and loads the subject's W
// (block-diagonal for its lane packing) while the density warps wait; the item
// body is the single-fit kernel's (tc_control_item.inc, tc_density_item.inc),
// and each item's statistics go to its own partial-slot group of the subject.
__device__ __forceinline__ void named_bar(int id, int nthreads) {
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
}

// the barriers of one item; `reinit` invalidates those of the previous item
// (every wait on them has completed by then)
__device__ __forceinline__ void tc_item_barriers(uint64_t* bar, bool reinit) {
    if (reinit)
        for (int r = 0; r < BAR_LT0 + 2 * kWG; r++)
            asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_u32(&bar[r])) : "memory");
    mbar_init(&bar[BAR_FULL0], 1);
    mbar_init(&bar[BAR_FULL1], 1);
    mbar_init(&bar[BAR_EMPTY0], 1);
    mbar_init(&bar[BAR_EMPTY1], 1);
    mbar_init(&bar[BAR_BFULL0], 1);
    mbar_init(&bar[BAR_BFULL1], 1);
    mbar_init(&bar[BAR_BEMPTY0], kDensWarps);
    mbar_init(&bar[BAR_BEMPTY1], kDensWarps);
    mbar_init(&bar[BAR_GFULL], kDensWarps);
    mbar_init(&bar[BAR_GEMPTY], 1);
    for (int r = 0; r < 2 * kWG; r++) mbar_init(&bar[BAR_LT0 + r], 1);
    mbar_init(&bar[BAR_PSI], 1);
    mbar_init(&bar[BAR_DRAIN], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

template <int MM, int R>
__device__ __forceinline__ void tc_cohort_density(uint8_t* sm, uint64_t* bar, volatile int* abort_flag,
                                                  const EStepArgs& a, const TcCohortItem& itm,
                                                  uint32_t tmem, int warp, int lane) {
    constexpr int NP = 128;
    constexpr bool SPLIT = false;
    using Sh = TcShape<NP>;
    float* slot = (float*)(sm + Sh::OFF_SLOT);
    const int h = 0, M = a.M, n = a.n;
    const int ntile_local = itm.ntiles;
    const uint32_t tmem_b0 = tmem, tmem_psi = tmem + kPsiCol;
    const int64_t item_tile0 = itm.tile0, item_stride = 1;
    const int item_slot = itm.slot, item_ngroups = kWG * R;
#include "tc_density_item.inc"
}

template <int MM>
__global__ void __launch_bounds__(kThreads, 1)
    estep_tc_cohort_kernel(const TcCohortSub* __restrict__ subs, const CUtensorMap* __restrict__ maps,
                           const TcCohortItem* __restrict__ items, const int* __restrict__ item_off) {
    constexpr int NP = 128;
    constexpr bool SPLIT = false;
    using Sh = TcShape<NP>;
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t* sm = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
    uint64_t* bar = (uint64_t*)(sm + Sh::OFF_BAR);
    uint32_t* tmem_holder = (uint32_t*)(sm + Sh::OFF_MISC);
    volatile int* abort_flag = (volatile int*)(sm + Sh::OFF_MISC + 8);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int i0 = item_off[blockIdx.x], i1 = item_off[blockIdx.x + 1];
    if (warp == kDensWarps) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     ::"r"(smem_u32(tmem_holder)), "r"(Sh::TMEM_COLS) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) *abort_flag = 0;
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_holder;
    const uint32_t tmem_b0 = tmem, tmem_psi = tmem + kPsiCol;
    if (warp >= kDensWarps) {
        // =========================== control warpgroup ==========================
        asm volatile("setmaxnreg.dec.sync.aligned.u32 %0;" ::"n"(kCtlRegs));
        const int ct = tid - kDensWarps * 32;         // 0 .. 127
        for (int ii = i0; ii < i1; ii++) {
            const TcCohortItem itm = items[ii];
            const EStepArgs& a = subs[itm.sub].a;
            const int npc = 128 / subs[itm.sub].R;
            if (ct == 0) tc_item_barriers(bar, ii > i0);
            // W_hi: the subject's block-diagonal W into the swizzled A tile
            {
                float* Wsm = (float*)(sm + Sh::OFF_W);
                for (int e4 = ct; e4 < 128 * (NP / 4); e4 += 128) {
                    const int i = e4 / (NP / 4), k = (e4 % (NP / 4)) * 4;
                    const int si = i / npc, sk = k / npc;
                    float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
                    if (si == sk)
                        v = *reinterpret_cast<const float4*>(a.Wf + (size_t)(i - si * npc) * npc + (k - sk * npc));
                    v.x = tf32_rna(v.x); v.y = tf32_rna(v.y); v.z = tf32_rna(v.z); v.w = tf32_rna(v.w);
                    *reinterpret_cast<float4*>((uint8_t*)Wsm + sw128_off(i, k, 128)) = v;
                }
            }
            // W_lo into tensor memory: warp 12 + q writes lanes 32 q .. 32 q + 31
            {
                const int q = warp & 3, i = q * 32 + lane, si = i / npc;
                const float* Wrow = a.Wf + (size_t)(i - si * npc) * npc;
#pragma unroll 1
                for (int k0 = 0; k0 < NP; k0 += 16) {
                    float lo[16];
                    const bool blk = (k0 / npc) == si;
#pragma unroll
                    for (int qq = 0; qq < 16; qq++) {
                        const float w = blk ? Wrow[k0 - si * npc + qq] : 0.f;
                        lo[qq] = tf32_rna(w - tf32_rna(w));
                    }
                    tmem_st16(tmem + kWloCol + ((uint32_t)(q * 32) << 16) + (uint32_t)k0, lo);
                }
            }
            fence_proxy_async();
            tc_fence_before();
            named_bar(1, kThreads);                   // item set up
            tc_fence_after();
            if (warp == kDensWarps && lane == 0 && itm.ntiles > 0) {
                const int ntile_local = itm.ntiles;
                const CUtensorMap* item_map = maps + itm.sub;
                const int64_t item_tile0 = itm.tile0, item_stride = 1;
#include "tc_control_item.inc"
            }
            __syncwarp();
            tc_fence_before();
            named_bar(2, kThreads);                   // item done
            tc_fence_after();
        }
    } else {
        // =========================== density warps ==============================
        asm volatile("setmaxnreg.inc.sync.aligned.u32 %0;" ::"n"(kDensRegs));
        for (int ii = i0; ii < i1; ii++) {
            named_bar(1, kThreads);
            tc_fence_after();
            const TcCohortItem itm = items[ii];
            const TcCohortSub& S = subs[itm.sub];
            if (S.R == 4) tc_cohort_density<MM, 4>(sm, bar, abort_flag, S.a, itm, tmem, warp, lane);
            else if (S.R == 2) tc_cohort_density<MM, 2>(sm, bar, abort_flag, S.a, itm, tmem, warp, lane);
            else tc_cohort_density<MM, 1>(sm, bar, abort_flag, S.a, itm, tmem, warp, lane);
            tc_fence_before();
            named_bar(2, kThreads);
            tc_fence_after();
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == kDensWarps) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;"
                     ::"r"(tmem), "r"(Sh::TMEM_COLS) : "memory");
    }
}

// ---------------------------------------------------------------- self-test
// One CTA runs a single contraction D[128][N] = A[128][K] . B[N][K]^T with the
// layouts, descriptors and TMEM access of the E-step kernel (B K-major in
// shared memory, as the x tile in MMA1 and the b tile in MMA2):
//   mode 0: A = tf32(A) K-major in shared memory (W_hi, G)
//   mode 1: A = tf32(A) in tensor memory (the A-from-TMEM form of W_lo)
//   mode 2: A = hi + lo split, hi in shared memory, lo in tensor memory (MMA1)
// K is a multiple of 16 (<= 64); N a multiple of 16 (<= 128).
__global__ void __launch_bounds__(128, 1) umma_selftest_kernel(const float* __restrict__ A,
                                                               const float* __restrict__ B,
                                                               float* __restrict__ D, int mode,
                                                               int N, int K, int* err) {
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t* sm = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
    uint8_t* As = sm;                      // K-major, 128 rows, ceil(K/32) blocks of 16 KB
    uint8_t* Bs = sm + 2 * 16384;          // K-major, N rows
    uint64_t* bar = (uint64_t*)(sm + 2 * 16384 + 2 * 16384);
    uint32_t* holder = (uint32_t*)(bar + 2);
    volatile int* abort_flag = (volatile int*)(bar + 3);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    for (int e = tid; e < 128 * K; e += 128) {
        const int r = e / K, c = e % K;
        *(float*)(As + sw128_off(r, c, 128)) = tf32_rna(A[e]);
    }
    for (int e = tid; e < N * K; e += 128) {
        const int r = e / K, c = e % K;
        *(float*)(Bs + sw128_off(r, c, N)) = tf32_rna(B[e]);
    }
    if (tid == 0) {
        mbar_init(&bar[0], 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     ::"r"(smem_u32(holder)), "r"(128u) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    fence_proxy_async();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *holder;                     // D: columns [0, N); A in TMEM: [N, N+K)
    if (mode >= 1) {
        const int r = warp * 32 + lane;
        for (int k0 = 0; k0 < K; k0 += 16) {
            float v[16];
            for (int q = 0; q < 16; q++) {
                const float w = A[(size_t)r * K + k0 + q];
                v[q] = mode == 1 ? tf32_rna(w) : tf32_rna(w - tf32_rna(w));
            }
            tmem_st16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(N + k0), v);
        }
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (tid == 0) {
        const uint32_t abase = smem_u32(As), bbase = smem_u32(Bs);
        const uint32_t id = idesc_tf32(128, N, 0, 0);
        for (int kk = 0; kk < K / 8; kk++) {
            const uint64_t bd = sdesc(bbase + (kk >> 2) * N * 128 + (kk & 3) * 32, 16, 1024);
            if (mode == 0 || mode == 2) {
                const uint64_t ad = sdesc(abase + (kk >> 2) * 128 * 128 + (kk & 3) * 32, 16, 1024);
                tc_mma_tf32(tmem, ad, bd, id, kk > 0 ? 1u : 0u);
            }
            if (mode >= 1)
                tc_mma_tf32_ta(tmem, tmem + (uint32_t)(N + kk * 8), bd, id,
                               (mode == 2 || kk > 0) ? 1u : 0u);
        }
        tc_commit(&bar[0]);
    }
    __syncwarp();
    const bool ok = mbar_wait(&bar[0], 0u, abort_flag, err);
    tc_fence_after();
    if (ok) {
        for (int c0 = 0; c0 < N; c0 += 16) {
            float v[16];
            tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
            for (int q = 0; q < 16; q++) D[(size_t)(warp * 32 + lane) * N + c0 + q] = v[q];
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(128u)
                     : "memory");
    }
}

// ---------------------------------------------------------------- host side
// Channels per packed sample set and sets per 128 lanes.
int tc_np(int n) { return n <= 32 ? 32 : (n <= 64 ? 64 : 128); }
int tc_pack(int n) { return 128 / tc_np(n); }

// a.x holds at least ceil(T / R) * R samples of a.ldx = npc floats (samples at
// and beyond T zero); it is read as ceil(T / R) rows of 128 floats.
template <int NP, int MM, int R, bool SPLIT>
cudaError_t launch_tc(const EStepArgs& a, int nclusters, cudaStream_t st) {
    using Sh = TcShape<NP, SPLIT>;
    PFN_encodeTiled enc = get_encode();
    if (!enc) return cudaErrorNotSupported;
    if (a.ldx * R != NP) return cudaErrorInvalidValue;
    const int64_t rows = (a.T + R - 1) / R;
    if (a.ntiles != (int)((rows + kS - 1) / kS)) return cudaErrorInvalidValue;
    CUtensorMap map;
    cuuint64_t dims[2] = {(cuuint64_t)NP, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)NP * 4};
    cuuint32_t box[2] = {32, (cuuint32_t)kS};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = enc(&map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, (void*)a.x, dims, strides, box, estr,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                     CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return cudaErrorInvalidValue;
    const size_t smem = Sh::BYTES + 1024;
    auto kern = estep_tc_kernel<NP, MM, R, SPLIT>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    TcArgs ta;
    ta.e = a;
    ta.ngroups = kWG * R;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(nclusters * a.M);
    cfg.blockDim = dim3(kThreads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = a.M;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kern, map, ta);
}

template <int NP, int MM, int R>
int tc_active_clusters(int M) {
    using Sh = TcShape<NP>;
    const size_t smem = Sh::BYTES + 1024;
    auto kern = estep_tc_kernel<NP, MM, R, false>;
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return -1;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(M * 64);
    cfg.blockDim = dim3(kThreads);
    cfg.dynamicSmemBytes = smem;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = M;
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

template <int MM>
cudaError_t launch_cohort(const TcCohortSub* subs, const CUtensorMap* maps, const TcCohortItem* items,
                          const int* item_off, int nctas, cudaStream_t st) {
    using Sh = TcShape<128>;
    const size_t smem = Sh::BYTES + 1024;
    auto kern = estep_tc_cohort_kernel<MM>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(nctas);
    cfg.blockDim = dim3(kThreads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = 1;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kern, subs, maps, items, item_off);
}

}  // namespace

namespace amica {

int tc_selftest(int mode, int N, int K, const float* hA, const float* hB, float* hD, int* derr) {
    if (mode < 0 || mode > 2 || N % 16 || N < 16 || N > 64 || K % 16 || K < 16 || K > 64)
        return -3;
    float *dA, *dB, *dD;
    int* err;
    if (cudaMalloc(&dA, sizeof(float) * 128 * K) != cudaSuccess) return -1;
    cudaMalloc(&dB, sizeof(float) * N * K);
    cudaMalloc(&dD, sizeof(float) * 128 * N);
    cudaMalloc(&err, sizeof(int));
    cudaMemset(err, 0, sizeof(int));
    cudaMemcpy(dA, hA, sizeof(float) * 128 * K, cudaMemcpyHostToDevice);
    cudaMemcpy(dB, hB, sizeof(float) * N * K, cudaMemcpyHostToDevice);
    const int smem = 4 * 16384 + 1024 + 64;
    cudaFuncSetAttribute(umma_selftest_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    umma_selftest_kernel<<<1, 128, smem>>>(dA, dB, dD, mode, N, K, err);
    cudaError_t e = cudaDeviceSynchronize();
    if (e == cudaSuccess) {
        cudaMemcpy(hD, dD, sizeof(float) * 128 * N, cudaMemcpyDeviceToHost);
        cudaMemcpy(derr, err, sizeof(int), cudaMemcpyDeviceToHost);
    }
    cudaFree(dA); cudaFree(dB); cudaFree(dD); cudaFree(err);
    return e == cudaSuccess ? 0 : -20;
}

// Samples per tile: kS packed rows of R samples each.
int tc_tile_samples(int n) { return kS * tc_pack(n); }
// Partial slots per cluster, and the stride between the slots that carry phi.
int tc_partial_groups(int n) { return kWG * tc_pack(n); }
int tc_psi_step() { return kWG; }

int tc_supported(int n, int m, int M) {
    return n >= 2 && n <= 128 && m >= 1 && m <= 5 && M >= 1 && M <= kMaxModels;
}

// Every channel count runs the 128-lane kernel (packed below 65 channels).
int tc_max_clusters(int n, int m, int M) {
    if (!tc_supported(n, m, M)) return -1;
    const int R = tc_pack(n);
#define AMICA_TC_OCC(MMV) \
    if (m == MMV) return R == 1 ? tc_active_clusters<128, MMV, 1>(M) \
                                : (R == 2 ? tc_active_clusters<128, MMV, 2>(M) \
                                          : tc_active_clusters<128, MMV, 4>(M));
    AMICA_TC_OCC(1) AMICA_TC_OCC(2) AMICA_TC_OCC(3) AMICA_TC_OCC(4) AMICA_TC_OCC(5)
#undef AMICA_TC_OCC
    return -1;
}

// The x tensor map of one subject for the cohort kernel (a.x read as rows of
// 128 floats, R samples each); `map` receives a CUtensorMap (128 bytes).
int tc_cohort_encode_map(const EStepArgs& a, void* map) {
    PFN_encodeTiled enc = get_encode();
    if (!enc) return -1;
    const int R = tc_pack(a.n);
    if (a.ldx * R != 128) return -1;
    const int64_t rows = (a.T + R - 1) / R;
    cuuint64_t dims[2] = {(cuuint64_t)128, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)128 * 4};
    cuuint32_t box[2] = {32, (cuuint32_t)kS};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = enc((CUtensorMap*)map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, (void*)a.x, dims, strides, box,
                     estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                     CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? 0 : -1;
}

// CTAs of the cohort launch: one per SM.
int tc_cohort_ctas() {
    int dev = 0, nsm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    return nsm;
}

cudaError_t launch_estep_tc_cohort(const TcCohortSub* subs, const void* maps, const TcCohortItem* items,
                                   const int* item_off, int nctas, int m, cudaStream_t st) {
    const CUtensorMap* mp = (const CUtensorMap*)maps;
    switch (m) {
        case 1: return launch_cohort<1>(subs, mp, items, item_off, nctas, st);
        case 2: return launch_cohort<2>(subs, mp, items, item_off, nctas, st);
        case 3: return launch_cohort<3>(subs, mp, items, item_off, nctas, st);
        case 4: return launch_cohort<4>(subs, mp, items, item_off, nctas, st);
        case 5: return launch_cohort<5>(subs, mp, items, item_off, nctas, st);
        default: return cudaErrorInvalidValue;
    }
}

// split: 0 the plain instantiation only, 1 the split-correction one only, 2
// both (each leaves at once unless the device flag a.split_phi selects it).
template <bool SPLIT>
cudaError_t launch_tc_form(const EStepArgs& a, int nclusters, cudaStream_t st) {
    const int R = tc_pack(a.n);
#define AMICA_TC_CASE(MMV) \
    if (a.m == MMV) return R == 1 ? launch_tc<128, MMV, 1, SPLIT>(a, nclusters, st) \
                                  : (R == 2 ? launch_tc<128, MMV, 2, SPLIT>(a, nclusters, st) \
                                            : launch_tc<128, MMV, 4, SPLIT>(a, nclusters, st));
    AMICA_TC_CASE(1) AMICA_TC_CASE(2) AMICA_TC_CASE(3) AMICA_TC_CASE(4) AMICA_TC_CASE(5)
#undef AMICA_TC_CASE
    return cudaErrorInvalidValue;
}

cudaError_t launch_estep_tc(const EStepArgs& a, int NP, int nclusters, cudaStream_t st, int split) {
    if (NP != tc_np(a.n) || a.ldx != NP) return cudaErrorInvalidValue;
    if (split != 1) {
        const cudaError_t e = launch_tc_form<false>(a, nclusters, st);
        if (e != cudaSuccess) return e;
    }
    if (split != 0) return launch_tc_form<true>(a, nclusters, st);
    return cudaSuccess;
}

}  // namespace amica
