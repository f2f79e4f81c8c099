// Host side of the AMICA EM engine: context, device buffers, the iteration
// pipeline and the C ABI declared in include/amica_b200.h.
//
// One iteration is a fixed sequence of kernels on the context's stream:
//   k_inverse_derive (FP64 inverse, log-det, E-step constants)
//   -> fused E-step (plain FP32 or tcgen05 TF32; above 128 channels the
//      mixed form is the split one: b = W x as TF32 tensor-core GEMMs, the
//      density-only E-step, then Psi = sum g x^T as TF32 GEMMs)
//   -> k_reduce + k_finalize (deterministic FP64 reduction of per-CTA sums)
//   -> k_mstep_params -> k_ctrl -> k_gemm64 (A update) -> k_reparm
//   (-> k_reject on schedule)
// with no host synchronisation, so amica_run() replays one captured CUDA graph
// per iteration.  This replaces runamica()'s iteration body
// (src/amica.cu:820-2541), which synchronised with the host ~T/block_size
// times per iteration.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>
#include <string>
#include <vector>


#include "amica_b200.h"
#include "common.cuh"

namespace amica {
// estep_plain.cu
int plain_pad_channels(int n);
int plain_partial_groups(int n);
int plain_max_clusters(int n, int m, int M);
int plain_tile_samples();
cudaError_t launch_estep_plain(const EStepArgs& a, int NP, int nclusters, cudaStream_t st);
bool split_form_supported(int n);
int dens_max_clusters(int m, int M);
cudaError_t launch_estep_dens(const EStepArgs& a, int nclusters, cudaStream_t st);
cudaError_t launch_split_w(const float* Wf, float* whi, float* wlo, int64_t len, cudaStream_t st);
// gemm_tc.cu
cudaError_t launch_wx_tc(const float* x, int64_t T, const float* Whi, const float* Wlo, float* B, int M,
                         int* err, cudaStream_t st);
cudaError_t launch_gx_tc(const float* gimg, const float* ximg, int64_t T, int n, int m, int M, double* partial,
                         int nslots, int* err, cudaStream_t st);
cudaError_t launch_xt_image(const float* x, int64_t T, float* ximg, cudaStream_t st);
// estep_tc.cu
int tc_supported(int n, int m, int M);
int tc_max_clusters(int n, int m, int M, int shape);
int tc_tile_samples(int n, int shape);
int tc_partial_groups(int n, int shape);
int tc_psi_step(int shape);
int tc_num_shapes();
int tc_cohort_encode_map(const EStepArgs& a, void* map);
int tc_cohort_ctas();
cudaError_t launch_estep_tc_cohort(const TcCohortSub* subs, const void* maps, const TcCohortItem* items,
                                   const int* item_off, int nctas, int m, cudaStream_t st);
int tc_selftest(int mode, int N, int K, const float* hA, const float* hB, float* hD, int* derr);
cudaError_t launch_estep_tc(const EStepArgs& a, int NP, int nclusters, cudaStream_t st, int split, int shape);
// preprocess.cu
cudaError_t launch_preprocess(const float* raw, int64_t T, int n, int do_sphere, double* means,
                              double* cov, double* sphere, double* evwork, double* ldetS_dev,
                              float* x, int ldx, int tf32, int* err, cudaStream_t st,
                              long long fault_wait_cycles);
cudaError_t launch_convert_sphered(const double* xs, int64_t T, int n, float* x, int ldx, int tf32,
                                   cudaStream_t st);
cudaError_t launch_shard_colsum(const float* raw, int64_t T, int n, double* sums, cudaStream_t st);
cudaError_t launch_shard_scatter(const float* raw, int64_t T, int n, const double* sums, int64_t T_total,
                                 double* means, double* scatter, cudaStream_t st);
cudaError_t launch_shard_finish(const float* raw, int64_t T, int n, int do_sphere, const double* means,
                                const double* scatter, int64_t T_total, double* cov, double* sphere,
                                double* evwork, double* ldetS_dev, float* x, int ldx, int tf32, int* err,
                                cudaStream_t st);
// adjoint.cu
cudaError_t launch_adjoint(const EStepArgs& a, int NP, double* grad_partial, int nclusters,
                           cudaStream_t st, bool use_tc, int tc_shape);
cudaError_t launch_adjoint_finalize(const double* grad_partial, double* raw, int nclusters, int n,
                                    int m, int M, const double* A, const double* c,
                                    const double* beta, const double* rho, double* out,
                                    int psi_is_phi, cudaStream_t st);

cudaError_t launch_prep(const MStepBuffers& b, const MStepCfgHost& h, cudaStream_t st);
cudaError_t launch_reduce_finalize(const MStepBuffers& b, const MStepCfgHost& h, int nclusters,
                                   cudaStream_t st);
cudaError_t launch_mstep(const MStepBuffers& b, const MStepCfgHost& h, const float* P_rel,
                         uint8_t* keep, int64_t T, cudaStream_t st);
cudaError_t launch_reject_now(const MStepBuffers& b, const MStepCfgHost& h, const float* P_rel,
                              uint8_t* keep, int64_t T, cudaStream_t st);
}  // namespace amica

using namespace amica;

struct amica_ctx {
    amica_cfg cfg{};
    int dev = 0;
    cudaStream_t st = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    int n = 0, M = 0, m = 0, NP = 0, S = 0;
    int64_t T = 0;
    bool use_tc = false;
    // split mixed form (128 < n <= 256): tcgen05 TF32 contractions around the
    // density-only E-step
    bool use_split = false;
    float *d_B = nullptr, *d_G = nullptr;         // b = W x per sample (T x M x NP); g as the Psi operand image
    float *d_Whi = nullptr, *d_Wlo = nullptr;     // M x NP x NP TF32 split of W
    float* d_xT = nullptr;                        // x^T operand image of the Psi contraction
    int adj_nclusters = 0;                        // grid of the plain gradient kernel (split form)
    int nclusters = 0, ntiles = 0, nslots = 0;   // nslots: partial-sum slots per model
    int tc_shape = 0;                             // tile shape of the fused E-step
    int nclusters_cap = 0;                        // grid the partial-sum buffer was sized for
    bool have_data = false, have_x = false, have_init = false, have_estep = false;
    bool have_shard_mean = false;   // amica_shard_scatter has set the mean of all shards

    float* d_rawx = nullptr;     // T x n raw input (float)
    float* d_x = nullptr;        // T x NP sphered (float)
    double *d_means = nullptr, *d_sphere = nullptr, *d_cov = nullptr, *d_evwork = nullptr,
           *d_ldetS = nullptr;
    double ldetS = 0.0;
    std::vector<double> h_means, h_sphere;

    MStepBuffers b{};
    MStepCfgHost hc{};
    uint8_t* d_keep = nullptr;
    float *d_Lt = nullptr, *d_P = nullptr;
    double* d_backup = nullptr;   // parameter snapshot for NaN rollback
    size_t backup_len = 0;
    double* d_gradp = nullptr;    // adjoint partials
    double* d_grad = nullptr;

    Ctrl* h_ctrl = nullptr;       // pinned
    long long fault_wait_cycles = 0;   // amica_test_arm_wait_fault: armed for the next preprocess
    int* h_err = nullptr;         // pinned
    std::vector<IterRec> hist;    // host copy of the iteration history

    cudaGraphExec_t graph = nullptr;
    int64_t pending = -1;         // iterations enqueued by amica_run_async, -1 if none
    int64_t pending_it0 = 0;
};

struct amica_cohort {
    std::vector<amica_ctx*> subs;
    int dev = 0, m = 0, nctas = 0, nitems = 0;
    cudaStream_t st = nullptr;                    // the cohort E-step's stream
    cudaEvent_t fork = nullptr, mid = nullptr, ev0 = nullptr, ev1 = nullptr;
    std::vector<cudaEvent_t> evs;                 // per subject: prep done, M-step done
    std::vector<int> nslots;                      // per subject: partial slots its items fill
    TcCohortSub* d_subs = nullptr;
    unsigned char* d_maps = nullptr;              // one CUtensorMap (128 bytes) per subject
    TcCohortItem* d_items = nullptr;
    int* d_off = nullptr;                         // items of CTA c: [d_off[c], d_off[c + 1])
    cudaGraphExec_t graph = nullptr;
};

namespace {

int g_last_cuda_error = 0;

#define CK(x)                                                                       \
    do {                                                                            \
        cudaError_t e_ = (x);                                                       \
        if (e_ != cudaSuccess) {                                                    \
            g_last_cuda_error = (int)e_;                                            \
            if (getenv("AMICA_DEBUG"))                                              \
                fprintf(stderr, "amica: %s -> %s (%s:%d)\n", #x, cudaGetErrorString(e_), \
                        __FILE__, __LINE__);                                        \
            return e_ == cudaErrorMemoryAllocation ? AMICA_ERR_NODEVICEMEM : AMICA_ERR_CUDA; \
        }                                                                           \
    } while (0)

template <class T>
int dalloc(T** p, size_t count) {
    CK(cudaMalloc((void**)p, sizeof(T) * (count > 0 ? count : 1)));
    CK(cudaMemset(*p, 0, sizeof(T) * (count > 0 ? count : 1)));
    return AMICA_OK;
}

#define TRY(x)                    \
    do {                          \
        int r_ = (x);             \
        if (r_ != AMICA_OK) return r_; \
    } while (0)

int64_t param_len(const amica_ctx* c) {
    const int64_t n = c->n, M = c->M, m = c->m;
    return M * n * n + M * n + 4 * M * m * n + M;
}

int snapshot_params(amica_ctx* c, bool restore) {
    const int64_t n = c->n, M = c->M, m = c->m;
    double* p = c->d_backup;
    struct Seg { double* d; int64_t len; } segs[] = {
        {c->b.A, M * n * n}, {c->b.c, M * n}, {c->b.alpha, M * m * n}, {c->b.mu, M * m * n},
        {c->b.beta, M * m * n}, {c->b.rho, M * m * n}, {c->b.gm, M}};
    for (auto& s : segs) {
        if (restore) CK(cudaMemcpyAsync(s.d, p, sizeof(double) * s.len, cudaMemcpyDeviceToDevice, c->st));
        else CK(cudaMemcpyAsync(p, s.d, sizeof(double) * s.len, cudaMemcpyDeviceToDevice, c->st));
        p += s.len;
    }
    Ctrl* cb = reinterpret_cast<Ctrl*>(p);
    if (restore) CK(cudaMemcpyAsync(c->b.ctrl, cb, sizeof(Ctrl), cudaMemcpyDeviceToDevice, c->st));
    else CK(cudaMemcpyAsync(cb, c->b.ctrl, sizeof(Ctrl), cudaMemcpyDeviceToDevice, c->st));
    return AMICA_OK;
}

EStepArgs estep_args(amica_ctx* c) {
    EStepArgs a{};
    a.x = c->d_x;
    a.Wf = c->b.Wf;
    a.wc = c->b.wcf;
    a.mp = c->b.mp;
    a.ltc64 = c->b.ltc64;
    a.keep = c->d_keep;
    a.Lt_out = c->d_Lt;
    a.P_out = c->d_P;
    a.partial = c->b.partial;
    a.err = c->b.err;
    a.split_phi = c->use_tc ? &c->b.ctrl->phi_split : nullptr;
    a.T = c->T;
    a.ldx = c->NP;
    a.n = c->n;
    a.M = c->M;
    a.m = c->m;
    a.ntiles = c->ntiles;
    a.nclusters = c->nclusters;
    a.update_rho = (int)c->cfg.update_rho;
    if (c->use_split) {
        a.bext = c->d_B;
        a.gout = c->d_G;
        a.ldb = c->M * c->NP;
    }
    return a;
}

// The split form's E-step: W -> (W_hi, W_lo), b = W_hi x + W_lo x (tensor-core
// kernel), the density-only kernel, Psi = sum g x^T (tensor-core kernel, FP32
// accumulation over at most 8192 samples, added into the partial slots in
// FP64).  W_hi has no bits below TF32 and x and g are stored rounded to TF32,
// so only W_lo is rounded by the MMA.
int enqueue_split_estep(amica_ctx* c, const EStepArgs& a) {
    const int M = c->M, NP = c->NP;
    CK(launch_split_w(c->b.Wf, c->d_Whi, c->d_Wlo, (int64_t)M * NP * NP, c->st));
    CK(launch_wx_tc(c->d_x, c->T, c->d_Whi, c->d_Wlo, c->d_B, M, c->b.err, c->st));
    CK(launch_estep_dens(a, c->nclusters, c->st));
    CK(launch_gx_tc(c->d_G, c->d_xT, c->T, c->n, c->m, M, c->b.partial, c->nslots, c->b.err, c->st));
    return AMICA_OK;
}

// The sphered data is in place: the split form also needs its x^T image.
int x_ready(amica_ctx* c) {
    if (c->use_split) {
        CK(launch_xt_image(c->d_x, c->T, c->d_xT, c->st));
        CK(cudaStreamSynchronize(c->st));
    }
    c->have_x = true;
    return AMICA_OK;
}

int enqueue_estep(amica_ctx* c) {
    CK(launch_prep(c->b, c->hc, c->st));
    EStepArgs a = estep_args(c);
    if (c->use_split) TRY(enqueue_split_estep(c, a));
    else if (c->use_tc) CK(launch_estep_tc(a, c->NP, c->nclusters, c->st, c->hc.phi_split, c->tc_shape));
    else CK(launch_estep_plain(a, c->NP, c->nclusters, c->st));
    CK(launch_reduce_finalize(c->b, c->hc, c->nslots, c->st));
    return AMICA_OK;
}

// Kernels one iteration launches: inverse/derive, E-step, reduce, finalize
// (+ phi from Psi in the plain form), params, ctrl, A update (when A is
// updated), reparametrisation, the finiteness check (+ rejection when enabled).
int launches_per_iteration(const amica_ctx* c) {
    // the split form adds the W split and its two tensor-core contractions
    const int split = c->use_split ? 3 : 0;
    return 8 + split + (c->hc.psi_is_phi ? 0 : 1) + (c->hc.update_A ? 1 : 0) + (c->hc.do_reject ? 1 : 0);
}

int enqueue_iteration(amica_ctx* c) {
    TRY(enqueue_estep(c));
    CK(launch_mstep(c->b, c->hc, c->d_P, c->d_keep, c->T, c->st));
    return AMICA_OK;
}

int check_device_error(amica_ctx* c) {
    CK(cudaMemcpyAsync(c->h_err, c->b.err, sizeof(int), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    int e = *c->h_err;
    if (e) {
        CK(cudaMemsetAsync(c->b.err, 0, sizeof(int), c->st));
        if (e & kErrWaitTimeout) return AMICA_ERR_TIMEOUT;
        if (e & kErrSingular) return AMICA_ERR_SINGULAR;
        if (e & kErrShape) return AMICA_ERR_UNSUPPORTED;
        if (e & kErrNonFinite) return AMICA_ERR_NUMERIC;
        return AMICA_ERR_CUDA;
    }
    return AMICA_OK;
}

void fill_out(const IterRec& r, const Ctrl& c, double ms, amica_iter_out* out) {
    if (!out) return;
    out->iter = r.iter;
    out->ll = r.ll;
    out->lrate = r.lrate;
    out->ll_decreased = r.ll_decreased;
    out->newton = r.newton;
    out->nkeep = c.nkeep;
    out->nrejected = r.nrejected;
    out->device_ms = ms;
    out->phi_split = r.phi_split;
}

void print_iter(const amica_ctx* c, const IterRec& r) {
    if (!c->cfg.verbose) return;
    // the reference's stdout lines, src/amica.cu:1983-1986 and :2322-2324
    fprintf(stdout, "Iteration %ld: lrate %.16f LL %.16f \n", (long)r.iter, r.lrate, r.ll);
    if (r.ll_decreased) fprintf(stdout, "Likelihood decreasing!\n");
    if (r.nrejected) fprintf(stdout, "Rejected %ld samples\n", (long)r.nrejected);
}

}  // namespace

extern "C" {

int amica_default_cfg(amica_cfg* c) {
    if (!c) return AMICA_ERR_INVALIDPARAM;
    memset(c, 0, sizeof(*c));
    c->nmmodels = 1;          // include/config.h:46-83
    c->nsdm = 3;
    c->maxiter = 200;
    c->do_sphere = 1;
    c->block_size = 5000;
    c->fix_init = 1;
    c->do_newton = 1;
    c->update_rho = 1;
    c->rho_start_iter = 1;
    c->newt_start_iter = 50;
    c->maxdec = 3;
    c->update_gm = c->update_alpha = c->update_A = c->update_mu = c->update_beta = 1;
    c->do_reparm = 1;
    c->do_reject = 0;
    c->rejstart = 10;
    c->rejint = 10;
    c->maxrej = 100;
    c->precision = AMICA_PREC_MIXED;
    c->device = 0;
    c->seed = 1234;
    c->verbose = 0;
    c->phi_split = 2;
    c->tc_shape = 0;
    c->phi_split_rel = kPhiSplitRel;
    c->lrate0 = 0.1;
    c->lratemax = 1.0;
    c->lnatrate = 0.1;
    c->lratefact = 0.5;
    c->rho0 = 1.5;
    c->rholrate = 0.1;
    c->rhomin = 1.0;
    c->rhomax = 2.0;
    c->rejsig = 3.0;
    return AMICA_OK;
}

int64_t amica_stats_len(int64_t n, int64_t M, int64_t m) {
    return 1 + M * (1 + 2 * n + n * n + 7 * m * n);
}

const char* amica_status_string(int s) {
    switch (s) {
        case AMICA_OK: return "Success!";
        case AMICA_ERR_NODEVICEMEM: return "No device memory";
        case AMICA_ERR_NOPARAM: return "No parameter";
        case AMICA_ERR_INVALIDPARAM: return "Invalid parameter";
        case AMICA_ERR_INVALIDCONFIG: return "Invalid config";
        case AMICA_ERR_NOFILE: return "No file";
        case AMICA_ERR_IO: return "Input/Output error";
        case AMICA_ERR_NOMEM: return "No more memory on host";
        case AMICA_ERR_CUDA: return "CUDA runtime error";
        case AMICA_ERR_STATE: return "Call out of order";
        case AMICA_ERR_SINGULAR: return "Mixing matrix is singular";
        case AMICA_ERR_NUMERIC: return "Non-finite log-likelihood or parameters (state rolled back)";
        case AMICA_ERR_TIMEOUT: return "A bounded device-side wait expired";
        case AMICA_ERR_UNSUPPORTED: return "Shape not supported by the compiled kernels";
        case AMICA_ERR_NODEVICE: return "No usable CUDA device";
        default: return "Unknown error";
    }
}

int amica_create(const amica_cfg* cfg, amica_ctx** out) {
    if (!cfg || !out) return AMICA_ERR_INVALIDPARAM;
    *out = nullptr;
    const int64_t n = cfg->nchannels, T = cfg->nsamples, M = cfg->nmmodels, m = cfg->nsdm;
    if (n < 2 || T < 2 || M < 1 || m < 1) return AMICA_ERR_INVALIDPARAM;
    if (M > kMaxModels || m > 5) return AMICA_ERR_UNSUPPORTED;
    if (cfg->precision != AMICA_PREC_FP32 && cfg->precision != AMICA_PREC_MIXED)
        return AMICA_ERR_INVALIDPARAM;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return AMICA_ERR_NODEVICE;
    if (cfg->device < 0 || cfg->device >= ndev) return AMICA_ERR_INVALIDPARAM;
    const int NP = plain_pad_channels((int)n);
    if (NP < 0) return AMICA_ERR_UNSUPPORTED;

    amica_ctx* c = new amica_ctx();
    c->cfg = *cfg;
    c->dev = (int)cfg->device;
    c->n = (int)n; c->T = T; c->M = (int)M; c->m = (int)m; c->NP = NP;
    CK(cudaSetDevice(c->dev));
    CK(cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking));
    CK(cudaEventCreate(&c->ev0));
    CK(cudaEventCreate(&c->ev1));

    c->use_tc = (cfg->precision == AMICA_PREC_MIXED) && tc_supported((int)n, (int)m, (int)M);
    c->use_split = (cfg->precision == AMICA_PREC_MIXED) && !c->use_tc && split_form_supported((int)n) &&
                   T <= 0x7fffffff;
    if (cfg->tc_shape < 0 || cfg->tc_shape >= tc_num_shapes()) { amica_destroy(c); return AMICA_ERR_INVALIDPARAM; }
    c->tc_shape = c->use_tc ? (int)cfg->tc_shape : 0;
    c->S = c->use_tc ? tc_tile_samples((int)n, c->tc_shape) : plain_tile_samples();
    c->ntiles = (int)((T + c->S - 1) / c->S);
    int maxcl = c->use_tc      ? tc_max_clusters((int)n, (int)m, (int)M, c->tc_shape)
                : c->use_split ? dens_max_clusters((int)m, (int)M)
                               : plain_max_clusters((int)n, (int)m, (int)M);
    if (maxcl <= 0) { amica_destroy(c); return AMICA_ERR_UNSUPPORTED; }
    // partial-sum slots are sized for the full grid (and, in the fused form,
    // every tile shape) so that amica_set_grid and amica_set_tile_shape can
    // move between them later
    c->nclusters_cap = maxcl < c->ntiles ? maxcl : c->ntiles;
    if (c->use_tc)
        for (int sh = 0; sh < tc_num_shapes(); sh++) {
            const int mc = tc_max_clusters((int)n, (int)m, (int)M, sh);
            const int nt = (int)((T + tc_tile_samples((int)n, sh) - 1) / tc_tile_samples((int)n, sh));
            const int cap = mc < nt ? mc : nt;
            if (cap > c->nclusters_cap) c->nclusters_cap = cap;
        }
    if (cfg->max_clusters > 0 && cfg->max_clusters < maxcl) maxcl = (int)cfg->max_clusters;
    c->nclusters = maxcl < c->ntiles ? maxcl : c->ntiles;

    MStepCfgHost& h = c->hc;
    h.n = (int)n; h.m = (int)m; h.M = (int)M; h.NP = NP;
    h.do_newton = (int)cfg->do_newton; h.update_rho = (int)cfg->update_rho;
    h.rho_start_iter = (int)cfg->rho_start_iter; h.newt_start_iter = (int)cfg->newt_start_iter;
    h.maxdec = (int)cfg->maxdec; h.update_gm = (int)cfg->update_gm;
    h.update_alpha = (int)cfg->update_alpha; h.update_A = (int)cfg->update_A;
    h.update_mu = (int)cfg->update_mu; h.update_beta = (int)cfg->update_beta;
    h.do_reparm = (int)cfg->do_reparm; h.do_reject = (int)cfg->do_reject;
    h.rejstart = (int)cfg->rejstart; h.rejint = (int)cfg->rejint; h.maxrej = (int)cfg->maxrej;
    h.lratemax = cfg->lratemax; h.lnatrate = cfg->lnatrate; h.lratefact = cfg->lratefact;
    h.rholrate = cfg->rholrate; h.rhomin = cfg->rhomin; h.rhomax = cfg->rhomax;
    h.rejsig = cfg->rejsig; h.ldetS = 0.0;
    h.psi_is_phi = c->use_tc ? 1 : 0;
    h.psi_step = c->use_tc ? tc_psi_step(c->tc_shape) : 1;
    h.phi_split = c->use_tc ? (int)cfg->phi_split : 0;
    h.phi_split_rel = cfg->phi_split_rel;

    MStepBuffers& b = c->b;
    const size_t nn = (size_t)n * n, mn = (size_t)m * n;
    int r = AMICA_OK;
#define AL(p, cnt) if ((r = dalloc(&(p), (cnt))) != AMICA_OK) { amica_destroy(c); return r; }
    AL(b.A, M * nn); AL(b.Anew, M * nn); AL(b.c, M * n); AL(b.alpha, M * mn); AL(b.mu, M * mn);
    AL(b.beta, M * mn); AL(b.rho, M * mn); AL(b.gm, M); AL(b.W, M * nn); AL(b.ldet, M);
    AL(b.ltc64, M);
    PartLayout PL{(int)n, (int)m};
    const int groups = c->use_tc ? tc_partial_groups((int)n, c->tc_shape) : c->use_split ? 1 : plain_partial_groups((int)n);
    c->nslots = c->nclusters * groups;
    int gmax = groups;
    if (c->use_tc)
        for (int sh = 0; sh < tc_num_shapes(); sh++) gmax = std::max(gmax, tc_partial_groups((int)n, sh));
    size_t pslots = (size_t)c->nclusters_cap * gmax;
    if (c->use_split) {
        // its adjoint runs the plain gradient kernel (channel-split clusters)
        const int pcl = plain_max_clusters((int)n, (int)m, (int)M);
        if (pcl <= 0) { amica_destroy(c); return AMICA_ERR_UNSUPPORTED; }
        c->adj_nclusters = pcl < c->ntiles ? pcl : c->ntiles;
        pslots = std::max(pslots, (size_t)c->adj_nclusters * plain_partial_groups((int)n));
    }
    AL(b.partial, pslots * M * PL.stride());
    AL(b.raw, M * (size_t)PL.stride());
    AL(b.stats, (size_t)amica_stats_len(n, M, m));
    AL(b.work, M * 4 * n);
    const int64_t nch = (T + 4095) / 4096;
    AL(b.chunk, 2 * nch + 2);
    if (n > 128) AL(b.gj, (size_t)M * nn + (size_t)M * n);
    AL(b.bflag, M); AL(b.use_newton, M);
    AL(b.Wf, (size_t)M * NP * NP); AL(b.wcf, (size_t)M * NP); AL(b.mp, (size_t)M * m * NP);
    AL(b.ctrl, 1);
    b.hist_cap = cfg->maxiter > 0 ? cfg->maxiter : 200;
    if (b.hist_cap < 1000) b.hist_cap = 1000;
    AL(b.hist, b.hist_cap);
    AL(b.err, 1);
    AL(c->d_keep, T); AL(c->d_Lt, M * T); AL(c->d_P, T);
    // 3 zero samples past T: the tensor-core form reads the data as rows of up
    // to 4 samples
    AL(c->d_x, (size_t)(T + 3) * NP);
    AL(c->d_means, n); AL(c->d_sphere, nn); AL(c->d_cov, nn); AL(c->d_evwork, 4 * nn + 4 * n);
    AL(c->d_ldetS, 1);
    c->backup_len = param_len(c) + (sizeof(Ctrl) + 7) / 8;
    AL(c->d_backup, c->backup_len);
    if (c->use_split) {
        // g is written per 64-sample tile as the Psi operand image
        AL(c->d_B, (size_t)T * M * NP); AL(c->d_G, (size_t)((T + 63) / 64) * 64 * M * NP);
        AL(c->d_xT, (size_t)((T + 31) / 32) * 32 * NP);
        AL(c->d_Whi, (size_t)M * NP * NP); AL(c->d_Wlo, (size_t)M * NP * NP);
    }
#undef AL
    CK(cudaMemsetAsync(c->d_keep, 1, T, c->st));
    CK(cudaMallocHost(&c->h_ctrl, sizeof(Ctrl)));
    CK(cudaMallocHost(&c->h_err, sizeof(int)));
    CK(cudaStreamSynchronize(c->st));
    *out = c;
    return AMICA_OK;
}

int amica_destroy(amica_ctx* c) {
    if (!c) return AMICA_OK;
    cudaSetDevice(c->dev);
    if (c->st) cudaStreamSynchronize(c->st);
    if (c->graph) cudaGraphExecDestroy(c->graph);
    void* ptrs[] = {c->b.A, c->b.Anew, c->b.c, c->b.alpha, c->b.mu, c->b.beta, c->b.rho, c->b.gm,
                    c->b.W, c->b.ldet, c->b.ltc64, c->b.partial, c->b.raw, c->b.stats,
                    c->b.work, c->b.chunk, c->b.gj, c->b.bflag, c->b.use_newton, c->b.Wf, c->b.wcf,
                    c->b.mp, c->b.ctrl, c->b.hist, c->b.err, c->d_keep, c->d_Lt, c->d_P, c->d_x,
                    c->d_rawx, c->d_means, c->d_sphere, c->d_cov, c->d_evwork, c->d_ldetS,
                    c->d_backup, c->d_gradp, c->d_grad, c->d_B, c->d_G, c->d_Whi, c->d_Wlo, c->d_xT};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    if (c->h_ctrl) cudaFreeHost(c->h_ctrl);
    if (c->h_err) cudaFreeHost(c->h_err);
    if (c->ev0) cudaEventDestroy(c->ev0);
    if (c->ev1) cudaEventDestroy(c->ev1);
    if (c->st) cudaStreamDestroy(c->st);
    delete c;
    return AMICA_OK;
}

const char* amica_kernel_name(amica_ctx* c) {
    if (!c) return "";
    return c->use_tc ? "tc_tf32" : c->use_split ? "split_tf32" : "plain_fp32";
}

static int load_raw(amica_ctx* c, const float* x, int64_t n, int64_t T, cudaMemcpyKind kind) {
    if (!c || !x) return AMICA_ERR_INVALIDPARAM;
    if (n != c->n || T != c->T) return AMICA_ERR_INVALIDPARAM;
    CK(cudaSetDevice(c->dev));
    if (!c->d_rawx) CK(cudaMalloc(&c->d_rawx, sizeof(float) * (size_t)T * n));
    CK(cudaMemcpyAsync(c->d_rawx, x, sizeof(float) * (size_t)T * n, kind, c->st));
    c->have_data = true;
    c->have_x = false;
    return AMICA_OK;
}

int amica_load_data(amica_ctx* c, const float* x, int64_t n, int64_t T) {
    return load_raw(c, x, n, T, cudaMemcpyHostToDevice);
}

int amica_load_data_device(amica_ctx* c, const float* dx, int64_t n, int64_t T) {
    return load_raw(c, dx, n, T, cudaMemcpyDeviceToDevice);
}

int amica_preprocess(amica_ctx* c) {
    if (!c) return AMICA_ERR_INVALIDPARAM;
    if (!c->have_data) return AMICA_ERR_STATE;
    CK(cudaSetDevice(c->dev));
    const long long fault = c->fault_wait_cycles;
    c->fault_wait_cycles = 0;                      // the hook arms one launch
    CK(launch_preprocess(c->d_rawx, c->T, c->n, (int)c->cfg.do_sphere, c->d_means, c->d_cov,
                         c->d_sphere, c->d_evwork, c->d_ldetS, c->d_x, c->NP, (c->use_tc || c->use_split) ? 1 : 0,
                         c->b.err, c->st, fault));
    double ld = 0.0;
    CK(cudaMemcpyAsync(&ld, c->d_ldetS, sizeof(double), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    TRY(check_device_error(c));
    c->ldetS = ld;
    c->hc.ldetS = ld;
    TRY(x_ready(c));
    return AMICA_OK;
}

int amica_set_sphered(amica_ctx* c, const double* xs, const double* means, const double* sphere,
                      double ldetS) {
    if (!c || !xs) return AMICA_ERR_INVALIDPARAM;
    CK(cudaSetDevice(c->dev));
    double* tmp = nullptr;
    const size_t bytes = sizeof(double) * (size_t)c->T * c->n;
    CK(cudaMalloc(&tmp, bytes));
    CK(cudaMemcpyAsync(tmp, xs, bytes, cudaMemcpyHostToDevice, c->st));
    CK(launch_convert_sphered(tmp, c->T, c->n, c->d_x, c->NP, (c->use_tc || c->use_split) ? 1 : 0, c->st));
    if (means) CK(cudaMemcpyAsync(c->d_means, means, sizeof(double) * c->n, cudaMemcpyHostToDevice, c->st));
    if (sphere) CK(cudaMemcpyAsync(c->d_sphere, sphere, sizeof(double) * c->n * c->n, cudaMemcpyHostToDevice, c->st));
    CK(cudaStreamSynchronize(c->st));
    CK(cudaFree(tmp));
    c->ldetS = ldetS;
    c->hc.ldetS = ldetS;
    TRY(x_ready(c));
    return AMICA_OK;
}

int amica_init(amica_ctx* c, const double* A0, const double* c0) {
    if (!c) return AMICA_ERR_INVALIDPARAM;
    CK(cudaSetDevice(c->dev));
    const int n = c->n, M = c->M, m = c->m;
    std::vector<double> A((size_t)M * n * n), cc((size_t)M * n), alpha((size_t)M * m * n),
        mu((size_t)M * m * n), beta((size_t)M * m * n), rho((size_t)M * m * n), gm(M);
    std::mt19937_64 rng((uint64_t)c->cfg.seed);
    std::uniform_real_distribution<double> U(0.0, 1.0);
    std::normal_distribution<double> N01(0.0, 1.0);
    if (A0) {
        memcpy(A.data(), A0, sizeof(double) * A.size());
        if (c0) memcpy(cc.data(), c0, sizeof(double) * cc.size());
    } else {
        // A = I + 0.05 (U - 0.5), unit columns; c ~ N(0, 1) (src/amica.cu:272-312)
        for (int h = 0; h < M; h++) {
            double* Ah = A.data() + (size_t)h * n * n;
            for (int e = 0; e < n * n; e++) Ah[e] = (U(rng) - 0.5) * 0.05 + ((e % n) == (e / n) ? 1.0 : 0.0);
            for (int col = 0; col < n; col++) {
                double s = 0.0;
                for (int r = 0; r < n; r++) s += Ah[col * n + r] * Ah[col * n + r];
                s = sqrt(s);
                for (int r = 0; r < n; r++) Ah[col * n + r] /= s;
            }
            for (int i = 0; i < n; i++) cc[(size_t)h * n + i] = c0 ? c0[(size_t)h * n + i] : N01(rng);
        }
    }
    for (int h = 0; h < M; h++) {
        gm[h] = 1.0 / M;                               // src/amica.cu:337
        for (int j = 0; j < m; j++)
            for (int i = 0; i < n; i++) {
                const size_t idx = ((size_t)h * m + j) * n + i;
                alpha[idx] = 1.0 / m;                  // :339-345
                if (c->cfg.fix_init) {                 // :347-362
                    mu[idx] = (double)j - (m - 1.0) / 2.0;
                    beta[idx] = 1.0;
                } else {                               // :363-387
                    mu[idx] = (m > 1) ? 0.1 * N01(rng) : 0.0;
                    beta[idx] = 1.0 + 0.1 * N01(rng);
                }
                rho[idx] = c->cfg.rho0;                // :389-394
            }
    }
    CK(cudaMemcpyAsync(c->b.A, A.data(), sizeof(double) * A.size(), cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync(c->b.c, cc.data(), sizeof(double) * cc.size(), cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync(c->b.alpha, alpha.data(), sizeof(double) * alpha.size(), cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync(c->b.mu, mu.data(), sizeof(double) * mu.size(), cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync(c->b.beta, beta.data(), sizeof(double) * beta.size(), cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync(c->b.rho, rho.data(), sizeof(double) * rho.size(), cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync(c->b.gm, gm.data(), sizeof(double) * gm.size(), cudaMemcpyHostToDevice, c->st));
    Ctrl ctl{};
    ctl.lrate = c->cfg.lrate0;
    ctl.lratemax = c->cfg.lratemax;
    ctl.iter = 0;
    ctl.nkeep = c->T;
    ctl.phi_split = c->hc.phi_split == 1 ? 1 : 0;   // 2: off until the M-step switches it on
    *c->h_ctrl = ctl;
    CK(cudaMemcpyAsync(c->b.ctrl, c->h_ctrl, sizeof(Ctrl), cudaMemcpyHostToDevice, c->st));
    CK(cudaMemsetAsync(c->d_keep, 1, c->T, c->st));
    CK(cudaStreamSynchronize(c->st));
    c->hist.clear();
    c->have_init = true;
    if (c->graph) { cudaGraphExecDestroy(c->graph); c->graph = nullptr; }
    return AMICA_OK;
}

int amica_em_step(amica_ctx* c, amica_iter_out* out) {
    if (!c) return AMICA_ERR_INVALIDPARAM;
    if (!c->have_x || !c->have_init) return AMICA_ERR_STATE;
    CK(cudaSetDevice(c->dev));
    TRY(snapshot_params(c, false));
    CK(cudaEventRecord(c->ev0, c->st));
    TRY(enqueue_iteration(c));
    CK(cudaEventRecord(c->ev1, c->st));
    CK(cudaMemcpyAsync(c->h_ctrl, c->b.ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    c->have_estep = true;
    int e = check_device_error(c);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, c->ev0, c->ev1);
    const Ctrl ctl = *c->h_ctrl;
    if (e == AMICA_OK && !std::isfinite(ctl.ll)) e = AMICA_ERR_NUMERIC;
    if (e != AMICA_OK) {
        snapshot_params(c, true);
        cudaStreamSynchronize(c->st);
        return e;
    }
    IterRec r{};
    CK(cudaMemcpy(&r, c->b.hist + (ctl.iter - 1), sizeof(IterRec), cudaMemcpyDeviceToHost));
    c->hist.push_back(r);
    print_iter(c, r);
    fill_out(r, ctl, ms, out);
    return AMICA_OK;
}

int amica_run_async(amica_ctx* c, int64_t maxiter) {
    if (!c) return AMICA_ERR_INVALIDPARAM;
    if (!c->have_x || !c->have_init) return AMICA_ERR_STATE;
    if (maxiter < 0) return AMICA_ERR_INVALIDPARAM;
    if (c->pending >= 0) return AMICA_ERR_STATE;      // a batch is still outstanding
    CK(cudaSetDevice(c->dev));
    if (!c->graph) {
        cudaGraph_t g;
        CK(cudaStreamBeginCapture(c->st, cudaStreamCaptureModeThreadLocal));
        int r = enqueue_iteration(c);
        cudaError_t ce = cudaStreamEndCapture(c->st, &g);
        if (r != AMICA_OK) return r;
        CK(ce);
        CK(cudaGraphInstantiate(&c->graph, g, 0));
        CK(cudaGraphDestroy(g));
    }
    CK(cudaMemcpyAsync(c->h_ctrl, c->b.ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    const int64_t it0 = c->h_ctrl->iter;
    if (it0 + maxiter > c->b.hist_cap) return AMICA_ERR_INVALIDPARAM;
    TRY(snapshot_params(c, false));
    CK(cudaEventRecord(c->ev0, c->st));
    for (int64_t k = 0; k < maxiter; k++) CK(cudaGraphLaunch(c->graph, c->st));
    CK(cudaEventRecord(c->ev1, c->st));
    CK(cudaMemcpyAsync(c->h_ctrl, c->b.ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, c->st));
    c->pending = maxiter;
    c->pending_it0 = it0;
    return AMICA_OK;
}

int amica_run_wait(amica_ctx* c, amica_iter_out* hist) {
    if (!c) return AMICA_ERR_INVALIDPARAM;
    if (c->pending < 0) return AMICA_ERR_STATE;
    CK(cudaSetDevice(c->dev));
    const int64_t maxiter = c->pending, it0 = c->pending_it0;
    c->pending = -1;
    CK(cudaStreamSynchronize(c->st));
    c->have_estep = maxiter > 0 || c->have_estep;
    int e = check_device_error(c);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, c->ev0, c->ev1);
    std::vector<IterRec> recs(maxiter);
    if (maxiter > 0)
        CK(cudaMemcpy(recs.data(), c->b.hist + it0, sizeof(IterRec) * maxiter, cudaMemcpyDeviceToHost));
    for (int64_t k = 0; k < maxiter; k++) {
        if (e == AMICA_OK && !std::isfinite(recs[k].ll)) e = AMICA_ERR_NUMERIC;
        c->hist.push_back(recs[k]);
        print_iter(c, recs[k]);
        if (hist) fill_out(recs[k], *c->h_ctrl, maxiter ? ms / maxiter : 0.0, &hist[k]);
    }
    if (e == AMICA_ERR_NUMERIC) {
        snapshot_params(c, true);
        cudaStreamSynchronize(c->st);
    }
    return e;
}

int amica_set_grid(amica_ctx* c, int64_t max_clusters, int64_t* nclusters) {
    if (!c || max_clusters < 0) return AMICA_ERR_INVALIDPARAM;
    if (c->pending >= 0) return AMICA_ERR_STATE;
    CK(cudaSetDevice(c->dev));
    int maxcl = c->use_tc      ? tc_max_clusters(c->n, c->m, c->M, c->tc_shape)
                : c->use_split ? dens_max_clusters(c->m, c->M)
                               : plain_max_clusters(c->n, c->m, c->M);
    if (maxcl <= 0) return AMICA_ERR_UNSUPPORTED;
    if (max_clusters > 0 && max_clusters < maxcl) maxcl = (int)max_clusters;
    const int ncl = maxcl < c->ntiles ? maxcl : c->ntiles;
    // the partial-sum slots were sized for the largest grid at creation
    if (ncl > c->nclusters_cap) return AMICA_ERR_INVALIDPARAM;
    c->nclusters = ncl;
    c->nslots = ncl * (c->use_tc ? tc_partial_groups(c->n, c->tc_shape) : c->use_split ? 1 : plain_partial_groups(c->n));
    if (c->graph) {
        CK(cudaStreamSynchronize(c->st));
        cudaGraphExecDestroy(c->graph);
        c->graph = nullptr;
    }
    if (nclusters) *nclusters = ncl;
    return AMICA_OK;
}

int amica_set_tile_shape(amica_ctx* c, int64_t shape) {
    if (!c || shape < 0 || shape >= tc_num_shapes()) return AMICA_ERR_INVALIDPARAM;
    if (!c->use_tc) return AMICA_ERR_UNSUPPORTED;
    if (c->pending >= 0) return AMICA_ERR_STATE;
    CK(cudaSetDevice(c->dev));
    const int S = tc_tile_samples(c->n, (int)shape);
    const int ntiles = (int)((c->T + S - 1) / S);
    const int mc = tc_max_clusters(c->n, c->m, c->M, (int)shape);
    if (mc <= 0) return AMICA_ERR_UNSUPPORTED;
    const int ncl = mc < ntiles ? mc : ntiles;
    if (ncl > c->nclusters_cap) return AMICA_ERR_UNSUPPORTED;
    if (c->graph) {
        CK(cudaStreamSynchronize(c->st));
        cudaGraphExecDestroy(c->graph);
        c->graph = nullptr;
    }
    c->tc_shape = (int)shape;
    c->S = S;
    c->ntiles = ntiles;
    c->nclusters = ncl;
    c->nslots = ncl * tc_partial_groups(c->n, c->tc_shape);
    c->hc.psi_step = tc_psi_step(c->tc_shape);
    return AMICA_OK;
}

int amica_run(amica_ctx* c, int64_t maxiter, amica_iter_out* hist) {
    TRY(amica_run_async(c, maxiter));
    return amica_run_wait(c, hist);
}

int amica_get_params(amica_ctx* c, double* A, double* W, double* cc, double* gm, double* alpha,
                     double* mu, double* beta, double* rho) {
    if (!c) return AMICA_ERR_INVALIDPARAM;
    CK(cudaSetDevice(c->dev));
    const size_t nn = (size_t)c->n * c->n * c->M, mn = (size_t)c->m * c->n * c->M;
    if (A) CK(cudaMemcpyAsync(A, c->b.A, sizeof(double) * nn, cudaMemcpyDeviceToHost, c->st));
    if (W) CK(cudaMemcpyAsync(W, c->b.W, sizeof(double) * nn, cudaMemcpyDeviceToHost, c->st));
    if (cc) CK(cudaMemcpyAsync(cc, c->b.c, sizeof(double) * c->n * c->M, cudaMemcpyDeviceToHost, c->st));
    if (gm) CK(cudaMemcpyAsync(gm, c->b.gm, sizeof(double) * c->M, cudaMemcpyDeviceToHost, c->st));
    if (alpha) CK(cudaMemcpyAsync(alpha, c->b.alpha, sizeof(double) * mn, cudaMemcpyDeviceToHost, c->st));
    if (mu) CK(cudaMemcpyAsync(mu, c->b.mu, sizeof(double) * mn, cudaMemcpyDeviceToHost, c->st));
    if (beta) CK(cudaMemcpyAsync(beta, c->b.beta, sizeof(double) * mn, cudaMemcpyDeviceToHost, c->st));
    if (rho) CK(cudaMemcpyAsync(rho, c->b.rho, sizeof(double) * mn, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    return AMICA_OK;
}

int amica_set_params(amica_ctx* c, const double* A, const double* cc, const double* gm,
                     const double* alpha, const double* mu, const double* beta, const double* rho) {
    if (!c) return AMICA_ERR_INVALIDPARAM;
    CK(cudaSetDevice(c->dev));
    const size_t nn = (size_t)c->n * c->n * c->M, mn = (size_t)c->m * c->n * c->M;
    if (A) CK(cudaMemcpyAsync(c->b.A, A, sizeof(double) * nn, cudaMemcpyHostToDevice, c->st));
    if (cc) CK(cudaMemcpyAsync(c->b.c, cc, sizeof(double) * c->n * c->M, cudaMemcpyHostToDevice, c->st));
    if (gm) CK(cudaMemcpyAsync(c->b.gm, gm, sizeof(double) * c->M, cudaMemcpyHostToDevice, c->st));
    if (alpha) CK(cudaMemcpyAsync(c->b.alpha, alpha, sizeof(double) * mn, cudaMemcpyHostToDevice, c->st));
    if (mu) CK(cudaMemcpyAsync(c->b.mu, mu, sizeof(double) * mn, cudaMemcpyHostToDevice, c->st));
    if (beta) CK(cudaMemcpyAsync(c->b.beta, beta, sizeof(double) * mn, cudaMemcpyHostToDevice, c->st));
    if (rho) CK(cudaMemcpyAsync(c->b.rho, rho, sizeof(double) * mn, cudaMemcpyHostToDevice, c->st));
    CK(cudaStreamSynchronize(c->st));
    return AMICA_OK;
}

int amica_estep_stats(amica_ctx* c, double* stats) {
    if (!c) return AMICA_ERR_INVALIDPARAM;
    if (!c->have_x || !c->have_init) return AMICA_ERR_STATE;
    CK(cudaSetDevice(c->dev));
    TRY(enqueue_estep(c));
    c->have_estep = true;
    TRY(check_device_error(c));
    if (stats)
        CK(cudaMemcpy(stats, c->b.stats, sizeof(double) * amica_stats_len(c->n, c->M, c->m),
                      cudaMemcpyDeviceToHost));
    return AMICA_OK;
}

int amica_get_loglik(amica_ctx* c, double* Lt, double* P, uint8_t* keep) {
    if (!c) return AMICA_ERR_INVALIDPARAM;
    if (!c->have_estep) return AMICA_ERR_STATE;
    CK(cudaSetDevice(c->dev));
    CK(cudaStreamSynchronize(c->st));
    double ltc0 = 0.0;
    CK(cudaMemcpy(&ltc0, c->b.ltc64, sizeof(double), cudaMemcpyDeviceToHost));
    if (Lt || P) {
        const int64_t len = (Lt ? (int64_t)c->M : 0) * c->T;
        std::vector<float> tmp(len > c->T ? len : c->T);
        if (Lt) {
            CK(cudaMemcpy(tmp.data(), c->d_Lt, sizeof(float) * c->M * c->T, cudaMemcpyDeviceToHost));
            for (int64_t e = 0; e < (int64_t)c->M * c->T; e++) Lt[e] = (double)tmp[e] + ltc0;
        }
        if (P) {
            CK(cudaMemcpy(tmp.data(), c->d_P, sizeof(float) * c->T, cudaMemcpyDeviceToHost));
            for (int64_t t = 0; t < c->T; t++) P[t] = (double)tmp[t] + ltc0;
        }
    }
    if (keep) CK(cudaMemcpy(keep, c->d_keep, c->T, cudaMemcpyDeviceToHost));
    return AMICA_OK;
}

// Relative per-sample P as the kernels store it (float), for bit-exact checks.
int amica_get_p_relative(amica_ctx* c, float* P) {
    if (!c || !P) return AMICA_ERR_INVALIDPARAM;
    CK(cudaSetDevice(c->dev));
    CK(cudaStreamSynchronize(c->st));
    CK(cudaMemcpy(P, c->d_P, sizeof(float) * c->T, cudaMemcpyDeviceToHost));
    return AMICA_OK;
}

int amica_reject_now(amica_ctx* c, int64_t* nrej) {
    if (!c) return AMICA_ERR_INVALIDPARAM;
    if (!c->have_estep) return AMICA_ERR_STATE;
    CK(cudaSetDevice(c->dev));
    CK(launch_reject_now(c->b, c->hc, c->d_P, c->d_keep, c->T, c->st));
    CK(cudaMemcpyAsync(c->h_ctrl, c->b.ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    if (nrej) *nrej = c->h_ctrl->last_rejected;
    return AMICA_OK;
}

int amica_loglik_adjoint(amica_ctx* c, double* ll, double* dW, double* dmu, double* dbeta,
                         double* drho) {
    if (!c) return AMICA_ERR_INVALIDPARAM;
    if (!c->have_x || !c->have_init) return AMICA_ERR_STATE;
    CK(cudaSetDevice(c->dev));
    const int n = c->n, M = c->M, m = c->m;
    const size_t glen = 1 + (size_t)M * n * n + 3 * (size_t)M * m * n;
    if (!c->d_grad) CK(cudaMalloc(&c->d_grad, sizeof(double) * glen));
    CK(launch_prep(c->b, c->hc, c->st));
    EStepArgs a = estep_args(c);
    int ncl = c->nclusters, nsl = c->nslots;
    if (c->use_split) {                           // the plain gradient kernel, on its own grid
        ncl = c->adj_nclusters;
        nsl = ncl * plain_partial_groups(n);
        a.nclusters = ncl;
        // its channel blocks each write only their own channels of a slot, and
        // the split form's E-step leaves whole slots of another layout in this
        // buffer: start from zero
        PartLayout PL{n, m};
        CK(cudaMemsetAsync(c->b.partial, 0, sizeof(double) * (size_t)nsl * M * PL.stride(), c->st));
    }
    CK(launch_adjoint(a, c->NP, c->b.partial, ncl, c->st, c->use_tc, c->tc_shape));
    CK(launch_adjoint_finalize(c->b.partial, c->b.raw, nsl, n, m, M, c->b.A, c->b.c,
                               c->b.beta, c->b.rho, c->d_grad, c->hc.psi_is_phi, c->st));
    TRY(check_device_error(c));
    std::vector<double> g(glen);
    CK(cudaMemcpy(g.data(), c->d_grad, sizeof(double) * glen, cudaMemcpyDeviceToHost));
    // L = sum_t P(t) / (n T_kept): add the constant part T_kept * ltc0
    double ltc0 = 0.0;
    CK(cudaMemcpy(&ltc0, c->b.ltc64, sizeof(double), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(c->h_ctrl, c->b.ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost));
    const double Tk = (double)c->h_ctrl->nkeep;
    const double norm = 1.0 / ((double)n * Tk);
    if (ll) *ll = (g[0] + Tk * ltc0) * norm;
    size_t off = 1;
    if (dW) for (size_t e = 0; e < (size_t)M * n * n; e++) dW[e] = g[off + e] * norm;
    off += (size_t)M * n * n;
    if (dmu) for (size_t e = 0; e < (size_t)M * m * n; e++) dmu[e] = g[off + e] * norm;
    off += (size_t)M * m * n;
    if (dbeta) for (size_t e = 0; e < (size_t)M * m * n; e++) dbeta[e] = g[off + e] * norm;
    off += (size_t)M * m * n;
    if (drho) for (size_t e = 0; e < (size_t)M * m * n; e++) drho[e] = g[off + e] * norm;
    return AMICA_OK;
}

static int write_doubles(const char* path, const double* v, size_t count) {
    FILE* f = fopen(path, "w");
    if (!f) return AMICA_ERR_NOFILE;
    const size_t w = fwrite(v, sizeof(double), count, f);
    fclose(f);
    return w == count ? AMICA_OK : AMICA_ERR_IO;
}

int amica_write_outputs(amica_ctx* c, const amica_paths* p) {
    if (!c || !p) return AMICA_ERR_INVALIDPARAM;
    if (!c->have_init) return AMICA_ERR_STATE;
    const int n = c->n, M = c->M, m = c->m;
    const size_t nn = (size_t)n * n;
    std::vector<double> A(M * nn), W(M * nn), cc(M * n), gm(M), alpha(M * m * n), mu(M * m * n),
        beta(M * m * n), rho(M * m * n), S(nn), means(n);
    TRY(amica_get_params(c, A.data(), W.data(), cc.data(), gm.data(), alpha.data(), mu.data(),
                         beta.data(), rho.data()));
    CK(cudaMemcpy(S.data(), c->d_sphere, sizeof(double) * nn, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(means.data(), c->d_means, sizeof(double) * n, cudaMemcpyDeviceToHost));
    // back-transform to the unsphered space as src/amica.cu:2564-2668 does:
    // c <- S^+ c + mean, A <- S^+ A with unit columns (mu/beta left as stored)
    std::vector<double> Sinv(nn);
    {
        // S^{-1} by Gauss-Jordan on the host (n x n output-stage algebra)
        std::vector<double> a(nn * 2);
        for (int r = 0; r < n; r++)
            for (int col = 0; col < 2 * n; col++)
                a[(size_t)r * 2 * n + col] = col < n ? S[(size_t)col * n + r] : (col - n == r ? 1.0 : 0.0);
        for (int k = 0; k < n; k++) {
            int pv = k;
            for (int r = k + 1; r < n; r++)
                if (fabs(a[(size_t)r * 2 * n + k]) > fabs(a[(size_t)pv * 2 * n + k])) pv = r;
            if (a[(size_t)pv * 2 * n + k] == 0.0) return AMICA_ERR_SINGULAR;
            if (pv != k)
                for (int col = 0; col < 2 * n; col++) std::swap(a[(size_t)k * 2 * n + col], a[(size_t)pv * 2 * n + col]);
            const double inv = 1.0 / a[(size_t)k * 2 * n + k];
            for (int col = 0; col < 2 * n; col++) a[(size_t)k * 2 * n + col] *= inv;
            for (int r = 0; r < n; r++) {
                if (r == k) continue;
                const double f = a[(size_t)r * 2 * n + k];
                if (f != 0.0)
                    for (int col = 0; col < 2 * n; col++) a[(size_t)r * 2 * n + col] -= f * a[(size_t)k * 2 * n + col];
            }
        }
        for (int r = 0; r < n; r++)
            for (int col = 0; col < n; col++) Sinv[(size_t)col * n + r] = a[(size_t)r * 2 * n + n + col];
    }
    std::vector<double> Aout(M * nn), cout_(M * n);
    for (int h = 0; h < M; h++) {
        for (int i = 0; i < n; i++) {
            double acc = means[i];
            for (int k = 0; k < n; k++) acc += Sinv[(size_t)k * n + i] * cc[(size_t)h * n + k];
            cout_[(size_t)h * n + i] = acc;
        }
        for (int col = 0; col < n; col++) {
            double s2 = 0.0;
            for (int r = 0; r < n; r++) {
                double acc = 0.0;
                for (int k = 0; k < n; k++) acc += Sinv[(size_t)k * n + r] * A[h * nn + (size_t)col * n + k];
                Aout[h * nn + (size_t)col * n + r] = acc;
                s2 += acc * acc;
            }
            const double nr = sqrt(s2);
            for (int r = 0; r < n; r++) Aout[h * nn + (size_t)col * n + r] /= nr;
        }
    }
    std::vector<double> ll;
    for (const auto& r : c->hist) ll.push_back(r.ll);
    if (p->weightsfile) TRY(write_doubles(p->weightsfile, W.data(), W.size()));
    if (p->afile) TRY(write_doubles(p->afile, Aout.data(), Aout.size()));
    if (p->cfile) TRY(write_doubles(p->cfile, cout_.data(), cout_.size()));
    if (p->gmfile) TRY(write_doubles(p->gmfile, gm.data(), gm.size()));
    if (p->alphafile) TRY(write_doubles(p->alphafile, alpha.data(), alpha.size()));
    if (p->betafile) TRY(write_doubles(p->betafile, beta.data(), beta.size()));
    if (p->mufile) TRY(write_doubles(p->mufile, mu.data(), mu.size()));
    if (p->rhofile) TRY(write_doubles(p->rhofile, rho.data(), rho.size()));
    if (p->llfile) TRY(write_doubles(p->llfile, ll.data(), ll.size()));
    if (p->spherefile) TRY(write_doubles(p->spherefile, S.data(), S.size()));
    if (p->ltallfile && c->have_estep) {
        std::vector<double> Lt((size_t)M * c->T);
        TRY(amica_get_loglik(c, Lt.data(), nullptr, nullptr));
        TRY(write_doubles(p->ltallfile, Lt.data(), Lt.size()));
    }
    return AMICA_OK;
}

int amica_last_cuda_error(void) { return g_last_cuda_error; }

// ---- sample-sharded fits: the E-step of one shard, then the M-step from the
// statistics of all shards (added by the caller, e.g. one all-reduce)
__global__ void k_set_nkeep(Ctrl* ctrl, int64_t nkeep) { ctrl->nkeep = nkeep; }

int amica_shard_estep(amica_ctx* c, double* d_stats) {
    if (!c || !d_stats) return AMICA_ERR_INVALIDPARAM;
    if (!c->have_x || !c->have_init) return AMICA_ERR_STATE;
    if (c->hc.do_reject) return AMICA_ERR_UNSUPPORTED;   // the rejection rule needs every sample's P
    CK(cudaSetDevice(c->dev));
    TRY(snapshot_params(c, false));
    CK(cudaEventRecord(c->ev0, c->st));
    TRY(enqueue_estep(c));
    CK(cudaMemcpyAsync(d_stats, c->b.stats, sizeof(double) * amica_stats_len(c->n, c->M, c->m),
                       cudaMemcpyDeviceToDevice, c->st));
    // stream-ordered: the all-reduce that follows is queued behind it on this
    // stream; a device error surfaces in amica_shard_mstep
    c->have_estep = true;
    return AMICA_OK;
}

int amica_get_stream(amica_ctx* c, void** stream) {
    if (!c || !stream) return AMICA_ERR_INVALIDPARAM;
    *stream = (void*)c->st;
    return AMICA_OK;
}

int amica_shard_mstep(amica_ctx* c, const double* d_stats, int64_t nkeep_total, amica_iter_out* out) {
    if (!c || !d_stats || nkeep_total < 1) return AMICA_ERR_INVALIDPARAM;
    if (!c->have_estep) return AMICA_ERR_STATE;
    CK(cudaSetDevice(c->dev));
    CK(cudaMemcpyAsync(c->b.stats, d_stats, sizeof(double) * amica_stats_len(c->n, c->M, c->m),
                       cudaMemcpyDeviceToDevice, c->st));
    // the M-step normalises by the samples of every shard (LL, gm); the next
    // E-step of this shard counts its own again
    k_set_nkeep<<<1, 1, 0, c->st>>>(c->b.ctrl, nkeep_total);
    CK(launch_mstep(c->b, c->hc, c->d_P, c->d_keep, c->T, c->st));
    k_set_nkeep<<<1, 1, 0, c->st>>>(c->b.ctrl, c->T);
    CK(cudaEventRecord(c->ev1, c->st));
    CK(cudaMemcpyAsync(c->h_ctrl, c->b.ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    int e = check_device_error(c);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, c->ev0, c->ev1);
    const Ctrl ctl = *c->h_ctrl;
    if (e == AMICA_OK && !std::isfinite(ctl.ll)) e = AMICA_ERR_NUMERIC;
    if (e != AMICA_OK) {
        snapshot_params(c, true);
        cudaStreamSynchronize(c->st);
        return e;
    }
    IterRec r{};
    CK(cudaMemcpy(&r, c->b.hist + (ctl.iter - 1), sizeof(IterRec), cudaMemcpyDeviceToHost));
    r.nkeep = nkeep_total;
    c->hist.push_back(r);
    print_iter(c, r);
    fill_out(r, ctl, ms, out);
    if (out) out->nkeep = nkeep_total;
    return AMICA_OK;
}

int amica_shard_colsum(amica_ctx* c, double* d_sums) {
    if (!c || !d_sums) return AMICA_ERR_INVALIDPARAM;
    if (!c->have_data) return AMICA_ERR_STATE;
    CK(cudaSetDevice(c->dev));
    CK(launch_shard_colsum(c->d_rawx, c->T, c->n, d_sums, c->st));
    CK(cudaStreamSynchronize(c->st));
    return check_device_error(c);
}

int amica_shard_scatter(amica_ctx* c, const double* d_sums_total, int64_t T_total, double* d_scatter) {
    if (!c || !d_sums_total || !d_scatter || T_total < c->T) return AMICA_ERR_INVALIDPARAM;
    if (!c->have_data) return AMICA_ERR_STATE;
    CK(cudaSetDevice(c->dev));
    CK(launch_shard_scatter(c->d_rawx, c->T, c->n, d_sums_total, T_total, c->d_means, d_scatter, c->st));
    CK(cudaStreamSynchronize(c->st));
    TRY(check_device_error(c));
    c->have_shard_mean = true;
    return AMICA_OK;
}

int amica_shard_sphere(amica_ctx* c, const double* d_scatter_total, int64_t T_total) {
    if (!c || !d_scatter_total || T_total < c->T || T_total < 2) return AMICA_ERR_INVALIDPARAM;
    if (!c->have_data || !c->have_shard_mean) return AMICA_ERR_STATE;
    CK(cudaSetDevice(c->dev));
    CK(launch_shard_finish(c->d_rawx, c->T, c->n, (int)c->cfg.do_sphere, c->d_means, d_scatter_total, T_total,
                           c->d_cov, c->d_sphere, c->d_evwork, c->d_ldetS, c->d_x, c->NP,
                           (c->use_tc || c->use_split) ? 1 : 0, c->b.err, c->st));
    double ld = 0.0;
    CK(cudaMemcpyAsync(&ld, c->d_ldetS, sizeof(double), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    TRY(check_device_error(c));
    c->ldetS = ld;
    c->hc.ldetS = ld;
    TRY(x_ready(c));
    c->have_shard_mean = false;
    return AMICA_OK;
}

int amica_test_arm_wait_fault(amica_ctx* c, int64_t wait_cycles) {
    if (!c || wait_cycles <= 0) return AMICA_ERR_INVALIDPARAM;
    // the cooperative eigensolver (and its grid barriers) runs above 128 channels
    if (c->n <= 128 || c->cfg.do_sphere != 1) return AMICA_ERR_UNSUPPORTED;
    c->fault_wait_cycles = (long long)wait_cycles;
    return AMICA_OK;
}

int64_t amica_launches_per_iteration(amica_ctx* c) { return c ? launches_per_iteration(c) : 0; }

int amica_selftest_umma(int mode, int N, int K, const float* A, const float* B, float* D,
                        int* device_err) {
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return AMICA_ERR_NODEVICE;
    if (!A || !B || !D || !device_err) return AMICA_ERR_INVALIDPARAM;
    return tc_selftest(mode, N, K, A, B, D, device_err);
}

int amica_set_iter_state(amica_ctx* c, int64_t iter, double lrate, double ll_prev) {
    if (!c || iter < 0 || !(lrate > 0.0)) return AMICA_ERR_INVALIDPARAM;
    if (!c->have_init) return AMICA_ERR_STATE;
    CK(cudaSetDevice(c->dev));
    CK(cudaMemcpyAsync(c->h_ctrl, c->b.ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    c->h_ctrl->iter = iter;
    c->h_ctrl->lrate = lrate;
    c->h_ctrl->ll_prev = ll_prev;
    CK(cudaMemcpyAsync(c->b.ctrl, c->h_ctrl, sizeof(Ctrl), cudaMemcpyHostToDevice, c->st));
    CK(cudaStreamSynchronize(c->st));
    return AMICA_OK;
}

int amica_time_estep(amica_ctx* c, int64_t reps, double* ms_per_launch, int64_t* launches) {
    if (!c || reps < 1 || !ms_per_launch) return AMICA_ERR_INVALIDPARAM;
    if (!c->have_x || !c->have_init) return AMICA_ERR_STATE;
    CK(cudaSetDevice(c->dev));
    CK(launch_prep(c->b, c->hc, c->st));
    EStepArgs a = estep_args(c);
    // one untimed launch, then reps timed back-to-back launches of the fused kernel
    // (the split form: its whole E-step, GEMMs included)
    if (c->use_split) TRY(enqueue_split_estep(c, a));
    else if (c->use_tc) CK(launch_estep_tc(a, c->NP, c->nclusters, c->st, c->hc.phi_split, c->tc_shape));
    else CK(launch_estep_plain(a, c->NP, c->nclusters, c->st));
    CK(cudaEventRecord(c->ev0, c->st));
    for (int64_t r = 0; r < reps; r++) {
        if (c->use_split) TRY(enqueue_split_estep(c, a));
        else if (c->use_tc) CK(launch_estep_tc(a, c->NP, c->nclusters, c->st, c->hc.phi_split, c->tc_shape));
        else CK(launch_estep_plain(a, c->NP, c->nclusters, c->st));
    }
    CK(cudaEventRecord(c->ev1, c->st));
    CK(cudaEventSynchronize(c->ev1));
    TRY(check_device_error(c));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
    *ms_per_launch = (double)ms / (double)reps;
    // the constants' kernels, then (reps + 1) E-steps: the split form's E-step
    // is the W split, b = W x, the density kernel and Psi = g x^T
    const int64_t per = c->use_split ? 4 : 1;
    if (launches) *launches = (reps + 1) * per + 1;
    return AMICA_OK;
}

// ---------------------------------------------------------------- cohort
// Several single-model fits (the same m) advanced together: per iteration, each
// subject's inverse/derive on its own stream, ONE persistent tensor-core E-step
// over all subjects' tiles (estep_tc_cohort_kernel), then each subject's
// reduction and M-step on its own stream -- captured as one CUDA graph.  The
// tiles of all subjects are dealt to the CTAs (one per SM) as contiguous
// ranges of the concatenated tile list, so every CTA gets the same number of
// tiles; a range that crosses subjects becomes one work item per subject.
int amica_cohort_create(amica_ctx* const* ctxs, int64_t nsub, amica_cohort** out) {
    if (!ctxs || nsub < 1 || !out) return AMICA_ERR_INVALIDPARAM;
    *out = nullptr;
    const amica_ctx* c0 = ctxs[0];
    if (!c0) return AMICA_ERR_INVALIDPARAM;
    for (int64_t s = 0; s < nsub; s++) {
        const amica_ctx* c = ctxs[s];
        if (!c || c->dev != c0->dev || c->m != c0->m) return AMICA_ERR_INVALIDPARAM;
        // the cohort kernel runs the default tile shape
        if (!c->use_tc || c->M != 1 || c->tc_shape != 0) return AMICA_ERR_UNSUPPORTED;
    }
    CK(cudaSetDevice(c0->dev));
    amica_cohort* co = new amica_cohort();
    co->subs.assign(ctxs, ctxs + nsub);
    co->dev = c0->dev;
    co->m = c0->m;
    co->nctas = tc_cohort_ctas();
    // deal the concatenated tiles to the CTAs
    std::vector<int64_t> first(nsub + 1, 0);
    for (int64_t s = 0; s < nsub; s++) first[s + 1] = first[s] + co->subs[s]->ntiles;
    const int64_t N = first[nsub];
    std::vector<TcCohortItem> items;
    std::vector<int> off(co->nctas + 1, 0), nitem(nsub, 0);
    for (int cta = 0; cta < co->nctas; cta++) {
        const int64_t a0 = N * cta / co->nctas, a1 = N * (cta + 1) / co->nctas;
        int64_t t = a0;
        int s = 0;
        while (s < nsub && first[s + 1] <= t) s++;
        while (t < a1 && s < nsub) {
            const int64_t e = std::min(a1, first[s + 1]);
            TcCohortItem it;
            it.sub = s;
            it.slot = nitem[s]++;
            it.tile0 = t - first[s];
            it.ntiles = (int)(e - t);
            items.push_back(it);
            t = e;
            s++;
        }
        off[cta + 1] = (int)items.size();
    }
    std::vector<TcCohortSub> subs(nsub);
    std::vector<unsigned char> maps((size_t)nsub * 128);
    for (int64_t s = 0; s < nsub; s++) {
        amica_ctx* c = co->subs[s];
        if (nitem[s] > c->nclusters_cap) { delete co; return AMICA_ERR_UNSUPPORTED; }
        subs[s].a = estep_args(c);
        subs[s].R = 128 / c->NP;
        if (tc_cohort_encode_map(subs[s].a, maps.data() + (size_t)s * 128) != 0) {
            delete co;
            return AMICA_ERR_CUDA;
        }
        co->nslots.push_back(nitem[s] * tc_partial_groups(c->n, 0));
    }
    co->nitems = (int)items.size();
    int r = AMICA_OK;
#define COAL(p, cnt) if ((r = dalloc(&(p), (cnt))) != AMICA_OK) { amica_cohort_destroy(co); return r; }
    COAL(co->d_subs, (size_t)nsub);
    COAL(co->d_maps, (size_t)nsub * 128);
    COAL(co->d_items, items.size() ? items.size() : 1);
    COAL(co->d_off, (size_t)co->nctas + 1);
#undef COAL
    CK(cudaMemcpy(co->d_subs, subs.data(), sizeof(TcCohortSub) * nsub, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(co->d_maps, maps.data(), maps.size(), cudaMemcpyHostToDevice));
    if (!items.empty())
        CK(cudaMemcpy(co->d_items, items.data(), sizeof(TcCohortItem) * items.size(), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(co->d_off, off.data(), sizeof(int) * off.size(), cudaMemcpyHostToDevice));
    CK(cudaStreamCreateWithFlags(&co->st, cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&co->fork, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&co->mid, cudaEventDisableTiming));
    CK(cudaEventCreate(&co->ev0));
    CK(cudaEventCreate(&co->ev1));
    co->evs.resize(2 * nsub);
    for (auto& e : co->evs) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    *out = co;
    return AMICA_OK;
}

int amica_cohort_destroy(amica_cohort* co) {
    if (!co) return AMICA_OK;
    cudaSetDevice(co->dev);
    if (co->st) cudaStreamSynchronize(co->st);
    if (co->graph) cudaGraphExecDestroy(co->graph);
    cudaFree(co->d_subs); cudaFree(co->d_maps); cudaFree(co->d_items); cudaFree(co->d_off);
    for (auto e : co->evs) if (e) cudaEventDestroy(e);
    for (auto e : {co->fork, co->mid, co->ev0, co->ev1}) if (e) cudaEventDestroy(e);
    if (co->st) cudaStreamDestroy(co->st);
    delete co;
    return AMICA_OK;
}

static int cohort_capture(amica_cohort* co) {
    const int ns = (int)co->subs.size();
    cudaGraph_t g;
    CK(cudaStreamBeginCapture(co->st, cudaStreamCaptureModeThreadLocal));
    auto step = [&]() -> int {
        CK(cudaEventRecord(co->fork, co->st));
        for (int s = 0; s < ns; s++) {
            amica_ctx* c = co->subs[s];
            CK(cudaStreamWaitEvent(c->st, co->fork, 0));
            CK(launch_prep(c->b, c->hc, c->st));
            CK(cudaEventRecord(co->evs[2 * s], c->st));
            CK(cudaStreamWaitEvent(co->st, co->evs[2 * s], 0));
        }
        CK(launch_estep_tc_cohort(co->d_subs, co->d_maps, co->d_items, co->d_off, co->nctas, co->m, co->st));
        CK(cudaEventRecord(co->mid, co->st));
        for (int s = 0; s < ns; s++) {
            amica_ctx* c = co->subs[s];
            CK(cudaStreamWaitEvent(c->st, co->mid, 0));
            CK(launch_reduce_finalize(c->b, c->hc, co->nslots[s], c->st));
            CK(launch_mstep(c->b, c->hc, c->d_P, c->d_keep, c->T, c->st));
            CK(cudaEventRecord(co->evs[2 * s + 1], c->st));
            CK(cudaStreamWaitEvent(co->st, co->evs[2 * s + 1], 0));
        }
        return AMICA_OK;
    };
    const int r = step();
    cudaError_t ce = cudaStreamEndCapture(co->st, &g);
    if (r != AMICA_OK) return r;
    CK(ce);
    CK(cudaGraphInstantiate(&co->graph, g, 0));
    CK(cudaGraphDestroy(g));
    return AMICA_OK;
}

int amica_cohort_run(amica_cohort* co, int64_t iters, amica_iter_out* hist, double* ms_per_iter) {
    if (!co || iters < 0) return AMICA_ERR_INVALIDPARAM;
    CK(cudaSetDevice(co->dev));
    const int ns = (int)co->subs.size();
    std::vector<int64_t> it0(ns);
    for (int s = 0; s < ns; s++) {
        amica_ctx* c = co->subs[s];
        if (!c->have_x || !c->have_init) return AMICA_ERR_STATE;
        if (c->pending >= 0) return AMICA_ERR_STATE;
        CK(cudaMemcpyAsync(c->h_ctrl, c->b.ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, c->st));
        CK(cudaStreamSynchronize(c->st));
        it0[s] = c->h_ctrl->iter;
        if (it0[s] + iters > c->b.hist_cap) return AMICA_ERR_INVALIDPARAM;
    }
    if (!co->graph) TRY(cohort_capture(co));
    for (int s = 0; s < ns; s++) {
        amica_ctx* c = co->subs[s];
        TRY(snapshot_params(c, false));
        CK(cudaEventRecord(co->evs[2 * s], c->st));
        CK(cudaStreamWaitEvent(co->st, co->evs[2 * s], 0));
    }
    CK(cudaEventRecord(co->ev0, co->st));
    for (int64_t k = 0; k < iters; k++) CK(cudaGraphLaunch(co->graph, co->st));
    CK(cudaEventRecord(co->ev1, co->st));
    CK(cudaStreamSynchronize(co->st));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, co->ev0, co->ev1));
    if (ms_per_iter) *ms_per_iter = iters ? (double)ms / (double)iters : 0.0;
    int first_err = AMICA_OK;
    for (int s = 0; s < ns; s++) {
        amica_ctx* c = co->subs[s];
        c->have_estep = c->have_estep || iters > 0;
        int e = check_device_error(c);
        CK(cudaMemcpy(c->h_ctrl, c->b.ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost));
        std::vector<IterRec> recs(iters);
        if (iters > 0)
            CK(cudaMemcpy(recs.data(), c->b.hist + it0[s], sizeof(IterRec) * iters, cudaMemcpyDeviceToHost));
        for (int64_t k = 0; k < iters; k++) {
            if (e == AMICA_OK && !std::isfinite(recs[k].ll)) e = AMICA_ERR_NUMERIC;
            c->hist.push_back(recs[k]);
            print_iter(c, recs[k]);
            if (hist) fill_out(recs[k], *c->h_ctrl, iters ? ms / iters : 0.0, &hist[(size_t)s * iters + k]);
        }
        if (e == AMICA_ERR_NUMERIC) {
            snapshot_params(c, true);
            cudaStreamSynchronize(c->st);
        }
        if (first_err == AMICA_OK) first_err = e;
    }
    return first_err;
}

int amica_get_sphere(amica_ctx* c, double* sphere, double* means, double* ldetS) {
    if (!c) return AMICA_ERR_INVALIDPARAM;
    if (!c->have_x) return AMICA_ERR_STATE;
    CK(cudaSetDevice(c->dev));
    CK(cudaStreamSynchronize(c->st));
    if (sphere) CK(cudaMemcpy(sphere, c->d_sphere, sizeof(double) * c->n * c->n, cudaMemcpyDeviceToHost));
    if (means) CK(cudaMemcpy(means, c->d_means, sizeof(double) * c->n, cudaMemcpyDeviceToHost));
    if (ldetS) *ldetS = c->ldetS;
    return AMICA_OK;
}

}  // extern "C"
