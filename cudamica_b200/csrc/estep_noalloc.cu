// E-step statistics without any allocation, for callers that cannot call
// cudaMalloc: code that runs inside another framework's memory pool or a host
// process that forbids allocations after start-up (real-time acquisition
// loops, plugins whose host owns the device memory budget).  Such a caller
// passes its own device buffers for the data, the parameters and the result;
// everything the computation needs in between lives in the fixed array below.
//
// The array is part of the module: every GPU that loads this library holds
// kNoAllocScratchBytes (5 MiB) of device memory for it until the process exits.
// Every call on a device uses the same array, and calls whose work overlaps on
// the GPU (two streams, two host threads) race on it: serialise them.
#include <cstdint>
#include <cstring>

#include "amica_b200.h"
#include "common.cuh"

namespace amica {
int plain_pad_channels(int n);
int plain_partial_groups(int n);
int plain_max_clusters(int n, int m, int M);
int plain_tile_samples();
cudaError_t launch_estep_plain(const EStepArgs& a, int NP, int nclusters, cudaStream_t st);
cudaError_t launch_prep(const MStepBuffers& b, const MStepCfgHost& h, cudaStream_t st);
cudaError_t launch_reduce_finalize(const MStepBuffers& b, const MStepCfgHost& h, int nclusters,
                                   cudaStream_t st);
}  // namespace amica

using namespace amica;

namespace {

constexpr size_t kNoAllocScratchBytes = 5u << 20;     // 5 MiB per device
constexpr int kNoAllocMaxClusters = 8;                // largest E-step grid in this mode

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// Device address of the scratch array in the CUDA context current on the
// calling thread.  The host-side symbol is only a handle, never a device
// address.  The lookup is repeated on every call (it is a table lookup once
// the module is loaded) rather than cached, so that an address never outlives
// its context: a device reset, or a caller that makes its own (non-primary)
// context current, gets the address that is valid in that context.
int scratch_in_current_context(unsigned char** out) {
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0) return AMICA_ERR_NODEVICE;
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || p == nullptr) return AMICA_ERR_CUDA;
    *out = (unsigned char*)p;
    return AMICA_OK;
}

__global__ void k_noalloc_ctrl(Ctrl* ctrl, int64_t nkeep) {
    Ctrl c;
    memset(&c, 0, sizeof(c));
    c.nkeep = nkeep;
    *ctrl = c;
}

// carve the scratch array; returns the bytes needed (0 on overflow of size_t)
size_t carve(unsigned char* base, int n, int M, int m, int NP, int nslots, MStepBuffers* b) {
    PartLayout PL{n, m};
    size_t off = 0;
    auto take = [&](size_t bytes) -> unsigned char* {
        unsigned char* p = base ? base + off : nullptr;
        off += (bytes + 255) & ~(size_t)255;
        return p;
    };
    memset(b, 0, sizeof(*b));
    b->W = (double*)take(sizeof(double) * M * n * n);
    b->ldet = (double*)take(sizeof(double) * M);
    b->ltc64 = (double*)take(sizeof(double) * M);
    b->Wf = (float*)take(sizeof(float) * M * NP * NP);
    b->wcf = (float*)take(sizeof(float) * M * NP);
    b->mp = (MixParam*)take(sizeof(MixParam) * M * m * NP);
    b->partial = (double*)take(sizeof(double) * (size_t)nslots * M * PL.stride());
    b->raw = (double*)take(sizeof(double) * (size_t)M * PL.stride());
    b->ctrl = (Ctrl*)take(sizeof(Ctrl));
    b->err = (int*)take(sizeof(int));
    if (n > 128) b->gj = (double*)take(sizeof(double) * ((size_t)M * n * n + (size_t)M * n));
    return off;
}

}  // namespace

extern "C" int amica_estep_stats_noalloc(const float* x, int64_t ldx, int64_t n, int64_t T,
                                         int64_t M, int64_t m, const double* A, const double* c,
                                         const double* alpha, const double* mu, const double* beta,
                                         const double* rho, const double* gm, double ldetS,
                                         const uint8_t* keep, int64_t nkeep, int64_t update_rho,
                                         double* stats, void* stream) {
    if (!x || !A || !c || !alpha || !mu || !beta || !rho || !gm || !stats) return AMICA_ERR_INVALIDPARAM;
    if (n < 2 || T < 2 || M < 1 || M > kMaxModels || m < 1 || m > 5) return AMICA_ERR_INVALIDPARAM;
    const int NP = plain_pad_channels((int)n);
    if (NP < 0 || ldx != NP) return AMICA_ERR_INVALIDPARAM;
    if (nkeep < 1 || nkeep > T) return AMICA_ERR_INVALIDPARAM;
    if (keep == nullptr && nkeep != T) return AMICA_ERR_INVALIDPARAM;   // every sample counts
    const int ntiles = (int)((T + plain_tile_samples() - 1) / plain_tile_samples());
    int ncl = plain_max_clusters((int)n, (int)m, (int)M);
    if (ncl <= 0) return AMICA_ERR_UNSUPPORTED;
    if (ncl > kNoAllocMaxClusters) ncl = kNoAllocMaxClusters;
    if (ncl > ntiles) ncl = ntiles;
    // above 128 channels each cluster has one slot per channel block
    const int groups = plain_partial_groups((int)n);
    // every cluster writes its own partial slots: use fewer clusters (down to
    // one, which runs every tile) until the layout fits the fixed array
    MStepBuffers b;
    while (ncl > 1 && carve(nullptr, (int)n, (int)M, (int)m, NP, ncl * groups, &b) > kNoAllocScratchBytes)
        ncl--;
    if (carve(nullptr, (int)n, (int)M, (int)m, NP, ncl * groups, &b) > kNoAllocScratchBytes)
        return AMICA_ERR_UNSUPPORTED;   // beyond the fixed 5 MiB even with one cluster
    unsigned char* base = nullptr;
    int rc = scratch_in_current_context(&base);
    if (rc != AMICA_OK) return rc;
    carve(base, (int)n, (int)M, (int)m, NP, ncl * groups, &b);
    b.A = const_cast<double*>(A);
    b.c = const_cast<double*>(c);
    b.alpha = const_cast<double*>(alpha);
    b.mu = const_cast<double*>(mu);
    b.beta = const_cast<double*>(beta);
    b.rho = const_cast<double*>(rho);
    b.gm = const_cast<double*>(gm);
    b.stats = stats;

    MStepCfgHost h;
    memset(&h, 0, sizeof(h));
    h.n = (int)n; h.m = (int)m; h.M = (int)M; h.NP = NP;
    h.ldetS = ldetS;
    h.psi_is_phi = 0;
    h.psi_step = 1;
    cudaStream_t st = (cudaStream_t)stream;

    // the only state that must start from zero each call: the error flag
    if (cudaMemsetAsync(b.err, 0, sizeof(int), st) != cudaSuccess) return AMICA_ERR_CUDA;
    // with channel blocks a slot leaves the other blocks' entries unwritten
    if (groups > 1) {
        PartLayout PL{(int)n, (int)m};
        const size_t pbytes = sizeof(double) * (size_t)ncl * groups * M * PL.stride();
        if (cudaMemsetAsync(b.partial, 0, pbytes, st) != cudaSuccess) return AMICA_ERR_CUDA;
    }
    k_noalloc_ctrl<<<1, 1, 0, st>>>(b.ctrl, nkeep);
    if (launch_prep(b, h, st) != cudaSuccess) return AMICA_ERR_CUDA;
    EStepArgs a;
    memset(&a, 0, sizeof(a));
    a.x = x; a.Wf = b.Wf; a.wc = b.wcf; a.mp = b.mp; a.ltc64 = b.ltc64;
    a.keep = keep; a.Lt_out = nullptr; a.P_out = nullptr; a.partial = b.partial; a.err = b.err;
    a.T = T; a.ldx = (int)ldx; a.n = (int)n; a.M = (int)M; a.m = (int)m;
    a.ntiles = ntiles; a.nclusters = ncl; a.update_rho = (int)update_rho; a.grad_mode = 0;
    if (launch_estep_plain(a, NP, ncl, st) != cudaSuccess) return AMICA_ERR_CUDA;
    if (launch_reduce_finalize(b, h, ncl * groups, st) != cudaSuccess) return AMICA_ERR_CUDA;
    int herr = 0;
    if (cudaMemcpyAsync(&herr, b.err, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess)
        return AMICA_ERR_CUDA;
    if (cudaStreamSynchronize(st) != cudaSuccess) return AMICA_ERR_CUDA;
    if (herr & kErrSingular) return AMICA_ERR_SINGULAR;
    if (herr & kErrShape) return AMICA_ERR_UNSUPPORTED;
    if (herr) return AMICA_ERR_CUDA;
    return AMICA_OK;
}
