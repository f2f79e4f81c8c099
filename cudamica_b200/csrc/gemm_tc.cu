// The two contractions of the split mixed form (128 < n <= 256 channels) on the
// 5th-generation tensor cores (tcgen05, kind::tf32, FP32 accumulation in tensor
// memory), around the density-only E-step kernel (estep_plain.cu, EXT form):
//
//   k_wx_tc  b_h(t) = W_hi,h x(t) + W_lo,h x(t) for every model h and sample t
//            (src/amica.cu:1054-1069, the Dgemm of b = W x).  CTA = (model h,
//            channel half c, sample chunk): W_hi rows [128c, 128c + 128) stay in
//            shared memory (K-major, 128-byte swizzle, 128 KB), W_lo of the same
//            rows in tensor memory (the A operand of the low half, 256 columns);
//            64-sample x tiles arrive by TMA in 64-column chunks (6 stages) and
//            are the B operand; the W_hi and W_lo products accumulate in two
//            tensor-memory accumulators [128 channels x 64 samples] (each
//            double-buffered), and 4 epilogue warps add them (thread = channel)
//            and write b[t][h][i] rows, 128 contiguous bytes per warp and sample.
//   k_gx_tc  Psi_h = sum_t g_h(t) x(t)^T (src/amica.cu:1535-1550, the Dgemm of
//            phi = g b^T, taken as Psi = g x^T and finished in the M-step's
//            finalize as phi = (Psi - gsum c^T) W^T).  CTA = (model h, half c,
//            sample chunk); per 32-sample block one thread copies the g^T block
//            (128 x 32, written in this layout by the density kernel) and the
//            x^T block (256 x 32, made once per data set by k_xt_image) into a
//            stage with two plain bulk copies and issues MMA M=128 N=256 K=32
//            into one of two 256-column tensor-memory accumulators; 4 flush
//            warps add each accumulator into the chunk's FP64 partial slot
//            every 256 blocks (8192 samples), so that no FP32 sum covers more
//            than 8192 samples.  Each FP64 address has one writer and the
//            slots are summed in a fixed order: the result is deterministic.
//
// The data x is T + 3 rows of 256 floats (TF32 values); g and the images hold
// TF32 values too, so the MMA's reading of its operands is exact.
// Every wait is bounded (tc_ptx.cuh) and a timed-out wait sets the error flag.
#include <cuda.h>
#include <cstdint>

#include "common.cuh"
#include "tc_ptx.cuh"

using namespace amica;

namespace {

constexpr int kNP = 256;                 // padded channels of the split form

// ------------------------------------------------------------------ b = W x
constexpr int kWxN = 64;                 // samples per tile (MMA N)
constexpr int kWxKC = 64;                // K columns per x stage (two 128-byte column blocks)
constexpr int kWxChunks = kNP / kWxKC;   // stages per tile
constexpr int kWxStages = 6;             // x stages
constexpr int kWxThreads = 5 * 32;       // 4 epilogue warps + the control warp
// tensor memory: W_lo [0, 256); D_hi buffers [256, 320) [320, 384); D_lo [384, 448) [448, 512)
constexpr uint32_t kWxDhi = 256, kWxDlo = 384;
struct WxShape {
    static constexpr uint32_t W_BYTES = 128u * kNP * 4u;             // 128 rows x 256 K
    static constexpr uint32_t X_BYTES = (uint32_t)kWxN * kWxKC * 4u;  // 64 rows x 64 K
    static constexpr uint32_t OFF_W = 0;
    static constexpr uint32_t OFF_X = OFF_W + W_BYTES;
    static constexpr uint32_t OFF_BAR = OFF_X + kWxStages * X_BYTES;
    static constexpr uint32_t NBAR = 24;
    static constexpr uint32_t OFF_MISC = OFF_BAR + NBAR * 8;
    static constexpr uint32_t BYTES = OFF_MISC + 64;
    static_assert(BYTES + 1024 <= 232448, "shared memory");
};
enum {
    WX_FULL0 = 0,
    WX_EMPTY0 = kWxStages,
    WX_DFULL0 = 2 * kWxStages,
    WX_DEMPTY0 = 2 * kWxStages + 2,
    WX_DRAIN = 2 * kWxStages + 4
};

struct WxArgs {
    const float* Whi;   // M x 256 x 256, W[h][i][k] rounded to TF32
    const float* Wlo;   // M x 256 x 256, W - W_hi
    float* B;           // T x (M * 256): B[t][h * 256 + i]
    int64_t T;
    int64_t ntiles;     // ceil(T / kWxN)
    int M;
    int nchunks;        // sample chunks: CTAs per (model, half)
    int* err;
};

// b = W_hi x + W_lo x with the two halves in separate accumulators, added in
// FP32 by the epilogue: the W_lo products (2^-11 of the W_hi ones) are summed
// among themselves and not into the large W_hi sum MMA by MMA.
__global__ void __launch_bounds__(kWxThreads, 1)
    k_wx_tc(const __grid_constant__ CUtensorMap xmap, WxArgs a) {
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t* sm = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
    uint64_t* bar = (uint64_t*)(sm + WxShape::OFF_BAR);
    uint32_t* tmem_holder = (uint32_t*)(sm + WxShape::OFF_MISC);
    volatile int* abort_flag = (volatile int*)(sm + WxShape::OFF_MISC + 8);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int slices = 2 * a.M;
    const int slice = blockIdx.x % slices, chunk = blockIdx.x / slices;
    const int h = slice >> 1, half = slice & 1;
    const int64_t kt0 = a.ntiles * chunk / a.nchunks, kt1 = a.ntiles * (chunk + 1) / a.nchunks;
    const int ntl = (int)(kt1 - kt0);

    if (tid == 0) {
        for (int s = 0; s < kWxStages; s++) {
            mbar_init(&bar[WX_FULL0 + s], 1);
            mbar_init(&bar[WX_EMPTY0 + s], 1);
        }
        for (int d = 0; d < 2; d++) {
            mbar_init(&bar[WX_DFULL0 + d], 1);
            mbar_init(&bar[WX_DEMPTY0 + d], 4);
        }
        mbar_init(&bar[WX_DRAIN], 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    // W_hi rows [128 half, 128 half + 128) of model h: the K-major A tile
    {
        const float* Wh = a.Whi + ((size_t)h * kNP + half * 128) * kNP;
        for (int e4 = tid; e4 < 128 * (kNP / 4); e4 += kWxThreads) {
            const int i = e4 / (kNP / 4), k = (e4 % (kNP / 4)) * 4;
            const float4 v = *reinterpret_cast<const float4*>(Wh + (size_t)i * kNP + k);
            *reinterpret_cast<float4*>(sm + WxShape::OFF_W + sw128_off(i, k, 128)) = v;
        }
    }
    if (warp == 4) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     ::"r"(smem_u32(tmem_holder)), "r"(512) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    fence_proxy_async();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_holder;
    // W_lo of the same rows into tensor memory (row -> lane), RNA-rounded to TF32
    if (warp < 4) {
        const int r = warp * 32 + lane;
        const float* wl = a.Wlo + ((size_t)h * kNP + half * 128 + r) * kNP;
#pragma unroll 1
        for (int k0 = 0; k0 < kNP; k0 += 16) {
            float lo[16];
#pragma unroll
            for (int q = 0; q < 16; q++) lo[q] = tf32_rna(wl[k0 + q]);
            tmem_st16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)k0, lo);
        }
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();

    if (warp == 4) {
        // ---- control: TMA loads of x chunks (tile kt, K columns [64 kc, 64 kc + 64)
        // = chunk u = 4 kt + kc), MMA issue from one thread
        if (lane == 0 && ntl > 0) {
            const uint32_t sbase = smem_u32(sm);
            const int nu = ntl * kWxChunks;
            auto issue = [&](int u) {
                const int s = u % kWxStages, kt = u / kWxChunks, kc = u % kWxChunks;
                const uint32_t xo = sbase + WxShape::OFF_X + (uint32_t)s * WxShape::X_BYTES;
                mbar_expect_tx(&bar[WX_FULL0 + s], WxShape::X_BYTES);
#pragma unroll
                for (int cb = 0; cb < kWxKC / 32; cb++)
                    tma_load_2d(xo + (uint32_t)(cb * kWxN * 128), &xmap, (kc * (kWxKC / 32) + cb) * 32,
                                (int)((kt0 + kt) * kWxN), &bar[WX_FULL0 + s]);
            };
            constexpr uint32_t ID = idesc_tf32(128, kWxN, 0, 0);
            int issued = 0, consumed = 0;
            while (issued < kWxStages && issued < nu) issue(issued++);
            bool ok = true;
            for (int u = 0; u < nu && ok; u++) {
                const int s = u % kWxStages, kt = u / kWxChunks, kc = u % kWxChunks, d = kt & 1;
                ok = mbar_wait(&bar[WX_FULL0 + s], (uint32_t)((u / kWxStages) & 1), abort_flag, a.err);
                if (ok) consumed = u + 1;
                if (ok && kc == 0 && kt >= 2)
                    ok = mbar_wait(&bar[WX_DEMPTY0 + d], (uint32_t)(((kt >> 1) - 1) & 1), abort_flag, a.err);
                if (!ok) break;
                tc_fence_after();
                const uint32_t xb = sbase + WxShape::OFF_X + (uint32_t)s * WxShape::X_BYTES;
                const uint32_t dhi = tmem + kWxDhi + (uint32_t)(d * kWxN);
                const uint32_t dlo = tmem + kWxDlo + (uint32_t)(d * kWxN);
                // descriptors of this chunk's first K step; the others differ by
                // constant address offsets (the address field is addr >> 4)
                const uint64_t ad0 =
                    sdesc(sbase + WxShape::OFF_W + (uint32_t)(kc * (kWxKC / 32) * 128 * 128), 16, 1024);
                const uint64_t bd0 = sdesc(xb, 16, 1024);
#pragma unroll
                for (int kk = 0; kk < kWxKC / 8; kk++) {
                    const uint32_t koff = (uint32_t)((kk & 3) * 32);
                    const uint64_t ad = ad0 + (((uint32_t)((kk >> 2) * 128 * 128) + koff) >> 4);
                    const uint64_t bd = bd0 + (((uint32_t)((kk >> 2) * kWxN * 128) + koff) >> 4);
                    const uint32_t acc = (kc > 0 || kk > 0) ? 1u : 0u;
                    tc_mma_tf32(dhi, ad, bd, ID, acc);
                    tc_mma_tf32_ta(dlo, tmem + (uint32_t)(kc * kWxKC + kk * 8), bd, ID, acc);
                }
                tc_commit(&bar[WX_EMPTY0 + s]);
                if (kc == kWxChunks - 1) tc_commit(&bar[WX_DFULL0 + d]);
                // the stage of the chunk before the previous one is refilled: its
                // MMAs have finished by now, so issuing does not wait on the
                // tensor pipe while it still has this chunk's work queued
                if (u >= 2 && u - 2 + kWxStages < nu) {
                    const int sp = (u - 2) % kWxStages;
                    ok = mbar_wait(&bar[WX_EMPTY0 + sp], (uint32_t)(((u - 2) / kWxStages) & 1), abort_flag,
                                   a.err);
                    if (!ok) break;
                    issue(u - 2 + kWxStages);
                    issued = u - 1 + kWxStages;
                }
            }
            // drain: every load issued has landed and every MMA has completed
            // before the CTA frees its tensor memory (bounded)
            for (int t = consumed; t < issued; t++)
                mbar_wait(&bar[WX_FULL0 + (t % kWxStages)], (uint32_t)((t / kWxStages) & 1), abort_flag, a.err,
                          false, false);
            tc_commit(&bar[WX_DRAIN]);
            mbar_wait(&bar[WX_DRAIN], 0u, abort_flag, a.err, false, false);
        }
        __syncwarp();
    } else {
        // ---- epilogue: thread = channel; b = D_hi + D_lo for the tile's 64 samples
        const int r = warp * 32 + lane;
        const size_t ldb = (size_t)a.M * kNP;
        float* Bout = a.B + (size_t)h * kNP + half * 128 + r;
        const uint32_t lane_addr = (uint32_t)(warp * 32) << 16;
        bool ok = true;
        for (int kt = 0; kt < ntl && ok; kt++) {
            const int d = kt & 1;
            ok = mbar_wait(&bar[WX_DFULL0 + d], (uint32_t)((kt >> 1) & 1), abort_flag, a.err);
            if (!ok) break;
            tc_fence_after();
            const int64_t t0 = (kt0 + kt) * kWxN;
#pragma unroll 1
            for (int c0 = 0; c0 < kWxN; c0 += 16) {
                float vh[16], vl[16];
                tmem_ld16(tmem + lane_addr + kWxDhi + (uint32_t)(d * kWxN + c0), vh);
                tmem_ld16(tmem + lane_addr + kWxDlo + (uint32_t)(d * kWxN + c0), vl);
#pragma unroll
                for (int s = 0; s < 16; s++)
                    if (t0 + c0 + s < a.T) Bout[(size_t)(t0 + c0 + s) * ldb] = vh[s] + vl[s];
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&bar[WX_DEMPTY0 + d]);
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 4) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512) : "memory");
    }
}

// ------------------------------------------------------------ Psi = g x^T
// Both operands come as ready-made images of K-major 128-byte-swizzled tiles,
// one per 32-sample block: g^T (128 channel rows x 32 samples, 16 KB, written
// by the density kernel) and x^T (256 rows x 32 samples, 32 KB, made once per
// data set by k_xt_image), so that each stage is two plain bulk copies.
constexpr int kGxT = 32;                 // samples per block (MMA K)
constexpr int kGxStages = 4;
constexpr int kGxThreads = 5 * 32;       // 4 flush warps + the control warp
constexpr int kGxFlushTiles = 256;       // blocks per FP32 accumulation period
struct GxShape {
    static constexpr uint32_t A_BYTES = 128u * 128u;   // 128 rows x 32 samples
    static constexpr uint32_t B_BYTES = 256u * 128u;   // 256 rows x 32 samples
    static constexpr uint32_t STAGE = A_BYTES + B_BYTES;
    static constexpr uint32_t OFF_BAR = kGxStages * STAGE;
    static constexpr uint32_t NBAR = 16;
    static constexpr uint32_t OFF_MISC = OFF_BAR + NBAR * 8;
    static constexpr uint32_t BYTES = OFF_MISC + 64;
    static_assert(BYTES + 1024 <= 232448, "shared memory");
};
enum {
    GX_FULL0 = 0,
    GX_EMPTY0 = kGxStages,
    GX_DFULL0 = 2 * kGxStages,
    GX_DEMPTY0 = 2 * kGxStages + 2,
    GX_DRAIN = 2 * kGxStages + 4
};

struct GxArgs {
    const float* gimg;  // [block][model][half][4096]
    const float* ximg;  // [block][8192]
    double* partial;    // partial slots; chunk q adds into slot q's Psi block
    int64_t nblocks;    // ceil(T / 32)
    int64_t pstride;    // doubles per model in a slot (PartLayout::stride)
    int psi_off;        // PartLayout::psi
    int M, n;
    int nchunks;
    int* err;
};

__global__ void __launch_bounds__(kGxThreads, 1) k_gx_tc(GxArgs a) {
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t* sm = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
    uint64_t* bar = (uint64_t*)(sm + GxShape::OFF_BAR);
    uint32_t* tmem_holder = (uint32_t*)(sm + GxShape::OFF_MISC);
    volatile int* abort_flag = (volatile int*)(sm + GxShape::OFF_MISC + 8);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int slices = 2 * a.M;
    const int slice = blockIdx.x % slices, chunk = blockIdx.x / slices;
    const int h = slice >> 1, half = slice & 1;
    const int64_t kt0 = a.nblocks * chunk / a.nchunks, kt1 = a.nblocks * (chunk + 1) / a.nchunks;
    const int ntl = (int)(kt1 - kt0);
    const int nper = (ntl + kGxFlushTiles - 1) / kGxFlushTiles;

    if (tid == 0) {
        for (int s = 0; s < kGxStages; s++) {
            mbar_init(&bar[GX_FULL0 + s], 1);
            mbar_init(&bar[GX_EMPTY0 + s], 1);
        }
        for (int d = 0; d < 2; d++) {
            mbar_init(&bar[GX_DFULL0 + d], 1);
            mbar_init(&bar[GX_DEMPTY0 + d], 4);
        }
        mbar_init(&bar[GX_DRAIN], 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 4) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     ::"r"(smem_u32(tmem_holder)), "r"(512) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_holder;

    if (warp < 4) {
        // ---- flush warps: thread = row i of this half; each period's FP32
        // accumulator is added into the chunk's FP64 slot
        const int r = warp * 32 + lane, i = half * 128 + r;
        const uint32_t lane_addr = (uint32_t)(warp * 32) << 16;
        double* out = a.partial + ((size_t)chunk * a.M + h) * a.pstride + a.psi_off;
        bool ok = true;
        for (int p = 0; p < nper && ok; p++) {
            const int db = p & 1;
            ok = mbar_wait(&bar[GX_DFULL0 + db], (uint32_t)((p >> 1) & 1), abort_flag, a.err);
            if (!ok) break;
            tc_fence_after();
#pragma unroll 1
            for (int k0 = 0; k0 < kNP; k0 += 16) {
                float v[16];
                tmem_ld16(tmem + lane_addr + (uint32_t)(db * kNP + k0), v);
                if (i < a.n) {
#pragma unroll
                    for (int q = 0; q < 16; q++)
                        if (k0 + q < a.n) red_add_f64(out + (size_t)(k0 + q) * a.n + i, (double)v[q]);
                }
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&bar[GX_DEMPTY0 + db]);
        }
    } else {
        // ---- control: bulk copies of the two operand blocks, MMA issue
        if (lane == 0 && ntl > 0) {
            const uint32_t sbase = smem_u32(sm);
            auto issue = [&](int kt) {
                const int s = kt % kGxStages;
                const int64_t blk = kt0 + kt;
                const uint32_t ab = sbase + (uint32_t)s * GxShape::STAGE;
                mbar_expect_tx(&bar[GX_FULL0 + s], GxShape::STAGE);
                bulk_load(ab, a.gimg + ((size_t)(blk * a.M + h) * 2 + half) * 4096, GxShape::A_BYTES,
                          &bar[GX_FULL0 + s]);
                bulk_load(ab + GxShape::A_BYTES, a.ximg + (size_t)blk * 8192, GxShape::B_BYTES,
                          &bar[GX_FULL0 + s]);
            };
            constexpr uint32_t ID = idesc_tf32(128, kNP, 0, 0);
            int issued = 0, consumed = 0;
            while (issued < kGxStages && issued < ntl) issue(issued++);
            bool ok = true;
            for (int kt = 0; kt < ntl && ok; kt++) {
                const int s = kt % kGxStages, p = kt / kGxFlushTiles, db = p & 1;
                const bool first = (kt % kGxFlushTiles) == 0;
                ok = mbar_wait(&bar[GX_FULL0 + s], (uint32_t)((kt / kGxStages) & 1), abort_flag, a.err);
                if (ok) consumed = kt + 1;
                if (ok && first && p >= 2)
                    ok = mbar_wait(&bar[GX_DEMPTY0 + db], (uint32_t)(((p >> 1) - 1) & 1), abort_flag, a.err);
                if (!ok) break;
                tc_fence_after();
                const uint32_t ab = sbase + (uint32_t)s * GxShape::STAGE, bb = ab + GxShape::A_BYTES;
#pragma unroll
                for (int kk = 0; kk < kGxT / 8; kk++)
                    tc_mma_tf32(tmem + (uint32_t)(db * kNP), sdesc(ab + (uint32_t)(kk * 32), 16, 1024),
                                sdesc(bb + (uint32_t)(kk * 32), 16, 1024), ID, (first && kk == 0) ? 0u : 1u);
                tc_commit(&bar[GX_EMPTY0 + s]);
                if ((kt % kGxFlushTiles) == kGxFlushTiles - 1 || kt == ntl - 1) tc_commit(&bar[GX_DFULL0 + db]);
                if (kt >= 1 && kt - 1 + kGxStages < ntl) {
                    const int sp = (kt - 1) % kGxStages;
                    ok = mbar_wait(&bar[GX_EMPTY0 + sp], (uint32_t)(((kt - 1) / kGxStages) & 1), abort_flag,
                                   a.err);
                    if (!ok) break;
                    issue(kt - 1 + kGxStages);
                    issued = kt + kGxStages;
                }
            }
            // drain: every copy issued has landed and every MMA has completed
            // before tensor memory is freed (bounded)
            for (int t = consumed; t < issued; t++)
                mbar_wait(&bar[GX_FULL0 + (t % kGxStages)], (uint32_t)((t / kGxStages) & 1), abort_flag, a.err,
                          false, false);
            tc_commit(&bar[GX_DRAIN]);
            mbar_wait(&bar[GX_DRAIN], 0u, abort_flag, a.err, false, false);
        }
        __syncwarp();
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 4) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512) : "memory");
    }
}

// The x^T operand image: block q holds samples [32 q, 32 q + 32) as a 256 x 32
// K-major swizzled tile (row = channel); samples past T are zero.
__global__ void __launch_bounds__(256) k_xt_image(const float* __restrict__ x, int64_t T, int64_t nblocks,
                                                  float* __restrict__ ximg) {
    const int k = threadIdx.x;
    for (int64_t q = blockIdx.x; q < nblocks; q += gridDim.x) {
#pragma unroll 2
        for (int c4 = 0; c4 < 8; c4++) {
            float v[4];
#pragma unroll
            for (int e = 0; e < 4; e++) {
                const int64_t t = q * 32 + c4 * 4 + e;
                v[e] = t < T ? x[(size_t)t * kNP + k] : 0.f;
            }
            *reinterpret_cast<float4*>(ximg + (size_t)q * 8192 + sw128_off(k, c4 * 4, 256) / 4) =
                make_float4(v[0], v[1], v[2], v[3]);
        }
    }
}

int sm_count_cur() {
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    return nsm;
}

}  // namespace

namespace amica {

// b = W_hi x + W_lo x for all models: x (T + 3) x 256 floats, W_hi / W_lo
// M x 256 x 256, B T x (M * 256).
cudaError_t launch_wx_tc(const float* x, int64_t T, const float* Whi, const float* Wlo, float* B, int M,
                         int* err, cudaStream_t st) {
    if (T < 1 || M < 1 || M > kMaxModels) return cudaErrorInvalidValue;
    PFN_encodeTiled enc = get_encode();
    if (!enc) return cudaErrorNotSupported;
    CUtensorMap map;
    cuuint64_t dims[2] = {(cuuint64_t)kNP, (cuuint64_t)(T + 3)};
    cuuint64_t strides[1] = {(cuuint64_t)kNP * 4};
    cuuint32_t box[2] = {32, (cuuint32_t)kWxN};   // one 128-byte column block of a tile
    cuuint32_t estr[2] = {1, 1};
    if (enc(&map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, (void*)x, dims, strides, box, estr,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return cudaErrorInvalidValue;
    WxArgs a{};
    a.Whi = Whi; a.Wlo = Wlo; a.B = B; a.T = T; a.M = M; a.err = err;
    a.ntiles = (T + kWxN - 1) / kWxN;
    const int slices = 2 * M;
    int nch = sm_count_cur() / slices;
    if (nch < 1) nch = 1;
    if (nch > a.ntiles) nch = (int)a.ntiles;
    a.nchunks = nch;
    const size_t smem = WxShape::BYTES + 1024;
    cudaError_t e = cudaFuncSetAttribute(k_wx_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    k_wx_tc<<<slices * nch, kWxThreads, smem, st>>>(map, a);
    return cudaGetLastError();
}

// Psi_h = sum_t g_h(t) x(t)^T from the two operand images, added into the
// Psi block of partial slots 0 .. nchunks-1 (nchunks <= nslots), which the
// density kernel has zeroed.
cudaError_t launch_gx_tc(const float* gimg, const float* ximg, int64_t T, int n, int m, int M, double* partial,
                         int nslots, int* err, cudaStream_t st) {
    if (T < 1 || M < 1 || M > kMaxModels || n < 1 || n > kNP || nslots < 1) return cudaErrorInvalidValue;
    PartLayout L{n, m};
    GxArgs a{};
    a.gimg = gimg; a.ximg = ximg; a.partial = partial; a.M = M; a.n = n; a.err = err;
    a.nblocks = (T + kGxT - 1) / kGxT;
    a.pstride = L.stride();
    a.psi_off = L.psi();
    const int slices = 2 * M;
    int nch = sm_count_cur() / slices;
    if (nch < 1) nch = 1;
    if (nch > nslots) nch = nslots;
    if (nch > a.nblocks) nch = (int)a.nblocks;
    a.nchunks = nch;
    const size_t smem = GxShape::BYTES + 1024;
    cudaError_t e = cudaFuncSetAttribute(k_gx_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    k_gx_tc<<<slices * nch, kGxThreads, smem, st>>>(a);
    return cudaGetLastError();
}

// The x^T image of the sphered data (ceil(T / 32) blocks of 8192 floats).
cudaError_t launch_xt_image(const float* x, int64_t T, float* ximg, cudaStream_t st) {
    if (T < 1) return cudaErrorInvalidValue;
    const int64_t nb = (T + kGxT - 1) / kGxT;
    const int grid = (int)(nb < 4 * 148 ? nb : 4 * 148);
    k_xt_image<<<grid, 256, 0, st>>>(x, T, nb, ximg);
    return cudaGetLastError();
}

}  // namespace amica
