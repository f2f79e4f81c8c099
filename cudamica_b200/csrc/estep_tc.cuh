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
//
// This header holds the kernel template and its launchers; estep_tc.cu
// instantiates the 3-warpgroup shape (and the cohort kernel, the self-test and
// the host interface), estep_tc_wg2.cu the 2-warpgroup shapes, so that the two
// compile in parallel.
#pragma once
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


// Tile shapes: WG density warpgroups of 4 warps, each handling kSub = 16
// samples of a tile, so kS = 16 WG samples (rows) per tile (MMA1 N, MMA2 K);
// NST x stages for the plain form (the split-correction form has one).
// Register split (setmaxnreg, per warpgroup): every thread is launched with
// kLaunchRegs registers; the control warpgroup drops to kCtlRegs (its rolled
// MMA issue needs about 80) and the density warpgroups rise to kDensRegs.
// Measured at n=128, T=1M, M=3, m=3 with 3 warpgroups: 136 beats 128 (no
// split), 144, 152 and 160.
template <int WG, int NST>
struct TcCfg {
    static constexpr int kWG = WG;
    static constexpr int kNST = NST;
    static constexpr int kSub = 16;
    static constexpr int kS = kSub * WG;
    static constexpr int kDensWarps = 4 * WG;
    static constexpr int kThreads = (kDensWarps + 4) * 32;
    static constexpr int kLaunchRegs = (65536 / kThreads) & ~7;
    static constexpr int kCtlRegs = 96;
    static constexpr int kDensRegs = WG == 3 ? 136 : 200;
    static_assert(WG * 128 * kDensRegs + 128 * kCtlRegs <= kThreads * kLaunchRegs, "register split");
    static_assert(kS < 64, "a tile and its log2|y| chunks share each 64-column b buffer");
    // log2|y| cache: chunks of kSub tensor-memory columns, first in the spare
    // columns [kS, 64) after each of the two b buffers, then in [384, 512)
    static constexpr int kGapChunks = (64 - kS) / kSub;
    static constexpr int kL2Chunks = 2 * kGapChunks + 128 / kSub;
    __host__ __device__ static constexpr uint32_t l2col(int c) {
        return c < 2 * kGapChunks ? (uint32_t)(64 * (c / kGapChunks) + kS + kSub * (c % kGapChunks))
                                  : 384u + (uint32_t)(kSub * (c - 2 * kGapChunks));
    }
};
using TcDef = TcCfg<3, 2>;               // the default shape (and the cohort kernel's)
constexpr int kS = TcDef::kS;            // samples per tile (MMA1 N)
constexpr int kWG = TcDef::kWG;          // density warpgroups
constexpr int kDensWarps = TcDef::kDensWarps;
constexpr int kThreads = TcDef::kThreads;
constexpr int kCtlRegs = TcDef::kCtlRegs;
constexpr int kDensRegs = TcDef::kDensRegs;
constexpr int kSub = TcDef::kSub;
constexpr int kBcol = 64;               // TMEM column stride of the two b buffers
constexpr int kPsiCol = 128;            // TMEM column of phi (N = NP columns)
constexpr int kWloCol = 256;            // TMEM columns of W_lo, the A operand of the low MMA1 half
// tiles between FP32 -> FP64 flushes: 16 tiles, 256 samples per thread (128
// per half of each FP32x2 sum); 2.72 ms per E-step at n=128, T=1M, M=3, m=3
// against 2.77 ms with 8
constexpr int kFlush = 16;
// x stages: up to kMaxStages, each with a FULL (TMA landed) and an EMPTY
// (MMAs done reading it) barrier
constexpr int kMaxStages = 3;

constexpr int kL2Chunks = TcDef::kL2Chunks;
__device__ __forceinline__ uint32_t l2_chunk_col(int c) { return TcDef::l2col(c); }

// SPLIT: the form with the split correction of phi (one x stage; the G and b
// tiles twice as wide, their low parts in columns [kS, 2 kS)).
template <int NP, bool SPLIT = false, class Cf = TcDef>
struct TcShape {
    static constexpr int kS = Cf::kS, kWG = Cf::kWG, kSub = Cf::kSub, kDensWarps = Cf::kDensWarps;
    static constexpr int KB = NP / 32;                       // 128-B column blocks of x / W
    static constexpr int NSTAGE = SPLIT ? 1 : Cf::kNST;      // x stages
    static_assert(NSTAGE >= 1 && NSTAGE <= kMaxStages, "x stages");
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
    // b: [0, kS) and [64, 64 + kS); phi: [128, 128 + NP); W_lo: [256, 256 + NP);
    // the log2|y| cache in the rest (TcCfg::l2col)
    static constexpr uint32_t TMEM_COLS = 512;
    static_assert(BYTES + 1024 <= 232448, "shared memory");
};

enum { BAR_FULL0 = 0, BAR_EMPTY0 = kMaxStages, BAR_BFULL0 = 2 * kMaxStages, BAR_BFULL1, BAR_BEMPTY0,
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
template <int NP, int MM, int R, bool SPLIT, int WG, int NST>
__global__ void __launch_bounds__(TcCfg<WG, NST>::kThreads, 1)
    estep_tc_kernel(const __grid_constant__ CUtensorMap xmap, TcArgs ta) {
    // this shape's constants, under the names the included bodies use
    using Cf = TcCfg<WG, NST>;
    constexpr int kS = Cf::kS, kWG = Cf::kWG, kSub = Cf::kSub, kDensWarps = Cf::kDensWarps;
    constexpr int kThreads = Cf::kThreads, kCtlRegs = Cf::kCtlRegs, kDensRegs = Cf::kDensRegs;
    constexpr int kL2Chunks = Cf::kL2Chunks;
    auto l2_chunk_col = [](int c) -> uint32_t { return Cf::l2col(c); };
    using Sh = TcShape<NP, SPLIT, Cf>;
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
        for (int q = 0; q < kMaxStages; q++) {
            mbar_init(&bar[BAR_FULL0 + q], 1);
            mbar_init(&bar[BAR_EMPTY0 + q], 1);
        }
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

// ---------------------------------------------------------------- host side
// Channels per packed sample set and sets per 128 lanes.
inline int tc_np(int n) { return n <= 32 ? 32 : (n <= 64 ? 64 : 128); }
inline int tc_pack(int n) { return 128 / tc_np(n); }

// a.x holds at least ceil(T / R) * R samples of a.ldx = npc floats (samples at
// and beyond T zero); it is read as ceil(T / R) rows of 128 floats.
template <int NP, int MM, int R, bool SPLIT, int WG, int NST>
cudaError_t launch_tc(const EStepArgs& a, int nclusters, cudaStream_t st) {
    using Cf = TcCfg<WG, NST>;
    constexpr int kS = Cf::kS, kWG = Cf::kWG, kThreads = Cf::kThreads;
    using Sh = TcShape<NP, SPLIT, Cf>;
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
    auto kern = estep_tc_kernel<NP, MM, R, SPLIT, WG, NST>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    // setmaxnreg draws on the registers the block is launched with: refuse a
    // build whose launch count cannot cover the split (the raise would wait)
    cudaFuncAttributes fa;
    e = cudaFuncGetAttributes(&fa, kern);
    if (e != cudaSuccess) return e;
    if (fa.numRegs * kThreads < WG * 128 * Cf::kDensRegs + 128 * Cf::kCtlRegs) return cudaErrorInvalidConfiguration;
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
template <int NP, int MM, int R, int WG, int NST>
int tc_active_clusters(int M) {
    using Cf = TcCfg<WG, NST>;
    constexpr int kThreads = Cf::kThreads;
    using Sh = TcShape<NP, false, Cf>;
    const size_t smem = Sh::BYTES + 1024;
    auto kern = estep_tc_kernel<NP, MM, R, false, WG, NST>;
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

// One tile shape's E-step for the context's n and m.  split: 0 the plain
// instantiation only, 1 the split-correction one only, 2 both (each leaves at
// once unless the device flag a.split_phi selects it); the split-correction
// form has one x stage whatever NST.
template <bool SPLIT, int WG, int NST>
cudaError_t launch_tc_form(const EStepArgs& a, int nclusters, cudaStream_t st) {
    const int R = tc_pack(a.n);
#define AMICA_TC_CASE(MMV) \
    if (a.m == MMV) return R == 1 ? launch_tc<128, MMV, 1, SPLIT, WG, NST>(a, nclusters, st) \
                                  : (R == 2 ? launch_tc<128, MMV, 2, SPLIT, WG, NST>(a, nclusters, st) \
                                            : launch_tc<128, MMV, 4, SPLIT, WG, NST>(a, nclusters, st));
    AMICA_TC_CASE(1) AMICA_TC_CASE(2) AMICA_TC_CASE(3) AMICA_TC_CASE(4) AMICA_TC_CASE(5)
#undef AMICA_TC_CASE
    return cudaErrorInvalidValue;
}

template <int WG, int NST>
cudaError_t launch_tc_shape(const EStepArgs& a, int nclusters, cudaStream_t st, int split) {
    if (split != 1) {
        const cudaError_t e = launch_tc_form<false, WG, NST>(a, nclusters, st);
        if (e != cudaSuccess) return e;
    }
    if (split != 0) return launch_tc_form<true, WG, 2>(a, nclusters, st);
    return cudaSuccess;
}

template <int WG, int NST>
int tc_max_clusters_shape(int n, int m, int M) {
    const int R = tc_pack(n);
#define AMICA_TC_OCC(MMV) \
    if (m == MMV) return R == 1 ? tc_active_clusters<128, MMV, 1, WG, NST>(M) \
                                : (R == 2 ? tc_active_clusters<128, MMV, 2, WG, NST>(M) \
                                          : tc_active_clusters<128, MMV, 4, WG, NST>(M));
    AMICA_TC_OCC(1) AMICA_TC_OCC(2) AMICA_TC_OCC(3) AMICA_TC_OCC(4) AMICA_TC_OCC(5)
#undef AMICA_TC_OCC
    return -1;
}

}  // namespace
