// The mixed-precision fused E-step (estep_tc.cuh) in its default shape of 3
// density warpgroups, the persistent cohort kernel over many single-model fits,
// the tensor-core self-test and the host interface that picks a shape.
#include "estep_tc.cuh"

namespace {

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

// Tile shapes the context can run (TcCfg): 0 = 3 density warpgroups,
// 48-sample tiles, 2 x stages (the default); 1 = 2 warpgroups, 32-sample tiles,
// 2 stages; 2 = 2 warpgroups, 3 stages.
int tc_wg2_max_clusters(int n, int m, int M, int nst);
cudaError_t tc_wg2_launch(const EStepArgs& a, int nclusters, cudaStream_t st, int split, int nst);

int tc_num_shapes() { return 3; }
static int shape_wg(int shape) { return shape == 0 ? 3 : 2; }
// Samples per tile: 16 rows per warpgroup, R samples per row.
int tc_tile_samples(int n, int shape) { return 16 * shape_wg(shape) * tc_pack(n); }
// Partial slots per cluster, and the stride between the slots that carry phi.
int tc_partial_groups(int n, int shape) { return shape_wg(shape) * tc_pack(n); }
int tc_psi_step(int shape) { return shape_wg(shape); }

int tc_supported(int n, int m, int M) {
    return n >= 2 && n <= 128 && m >= 1 && m <= 5 && M >= 1 && M <= kMaxModels;
}

// Every channel count runs the 128-lane kernel (packed below 65 channels).
int tc_max_clusters(int n, int m, int M, int shape) {
    if (!tc_supported(n, m, M) || shape < 0 || shape >= tc_num_shapes()) return -1;
    if (shape == 0) return tc_max_clusters_shape<3, 2>(n, m, M);
    return tc_wg2_max_clusters(n, m, M, shape == 1 ? 2 : 3);
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

cudaError_t launch_estep_tc(const EStepArgs& a, int NP, int nclusters, cudaStream_t st, int split, int shape) {
    if (NP != tc_np(a.n) || a.ldx != NP) return cudaErrorInvalidValue;
    if (shape == 0) return launch_tc_shape<3, 2>(a, nclusters, st, split);
    if (shape == 1 || shape == 2) return tc_wg2_launch(a, nclusters, st, split, shape == 1 ? 2 : 3);
    return cudaErrorInvalidValue;
}

}  // namespace amica
