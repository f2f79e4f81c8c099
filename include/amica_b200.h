/*
 * amica_b200.h -- C ABI of the B200-native AMICA EM engine.
 *
 * This is the drop-in boundary for the reference's EM loop
 * (fraimondo/cudamica).  The reference exposes no library API: its EM loop
 * is `error runamica(void)` (include/amica.h:123), which reads the global
 * `currentConfig` (include/config.h:85-172) filled by `getConfig()`
 * (src/config.c:12-213) and global device/model arrays, and exit(1)s on any
 * failure.  Each entry point below names the piece of that loop it replaces.
 *
 * Conventions:
 *   - every call returns an int status: 0 on success, the reference's codes
 *     (include/error.h:111-118) for the same conditions, new negative codes
 *     below for conditions the reference handles by exit(1).  Nothing calls
 *     exit().
 *   - caller-owned host buffers, context-owned device buffers; one context per
 *     host thread, each on its own CUDA stream.
 *   - layouts follow the reference's files: data T x n sample-major float32;
 *     A and W column-major n x n per model; c n per model; alpha, mu, beta,
 *     rho as M x m x n (channel fastest).
 */
#ifndef AMICA_B200_H
#define AMICA_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes: the reference's (include/error.h:111-118) ... */
#define AMICA_OK                 0
#define AMICA_ERR_NODEVICEMEM   (-1)
#define AMICA_ERR_NOPARAM       (-2)
#define AMICA_ERR_INVALIDPARAM  (-3)
#define AMICA_ERR_INVALIDCONFIG (-4)
#define AMICA_ERR_NOFILE        (-5)
#define AMICA_ERR_IO            (-6)
#define AMICA_ERR_NOMEM         (-7)
/* ... and the engine's own */
#define AMICA_ERR_CUDA          (-20)  /* a CUDA runtime call failed */
#define AMICA_ERR_STATE         (-21)  /* call out of order (e.g. em_step before init) */
#define AMICA_ERR_SINGULAR      (-22)  /* A_h not invertible */
#define AMICA_ERR_NUMERIC       (-23)  /* NaN/Inf in LL or parameters; state rolled back */
#define AMICA_ERR_TIMEOUT       (-24)  /* a bounded device-side wait expired */
#define AMICA_ERR_UNSUPPORTED   (-25)  /* shape outside the compiled kernels */
#define AMICA_ERR_NODEVICE      (-26)  /* no CUDA device / extension unusable */

#define AMICA_PREC_FP32   0   /* plain FP32 form: SIMT FP32 contractions */
#define AMICA_PREC_MIXED  1   /* tcgen05 TF32 contractions, FP32 densities */

/* Replaces the reference's `config` struct (include/config.h:85-172) with the
 * defaults of include/config.h:46-83; the rejection and precision keys are
 * new.  All fields are 8 bytes wide. */
typedef struct amica_cfg {
    int64_t nchannels, nsamples, nmmodels, nsdm;
    int64_t maxiter, do_sphere, block_size, fix_init;
    int64_t do_newton, update_rho, rho_start_iter, newt_start_iter, maxdec;
    int64_t update_gm, update_alpha, update_A, update_mu, update_beta, do_reparm;
    int64_t do_reject, rejstart, rejint, maxrej;
    int64_t precision, device, seed, verbose;
    int64_t max_clusters;   /* cap on the E-step grid in clusters (0: as many as fit); lets
                               several contexts share the GPU's SMs concurrently (new key) */
    int64_t phi_split;      /* mixed form: form phi = sum g b^T from hi + lo TF32 parts of
                               both operands: 0 never, 1 always, 2 (default) from the
                               iteration after a Newton step changed every model's A by
                               less than phi_split_rel (relative, Frobenius) (new key) */
    int64_t tc_shape;       /* mixed form up to 128 channels: tile shape of the fused E-step,
                               0 (default) 3 density warpgroups and 48-sample tiles with 2 x
                               stages, 1 2 warpgroups and 32-sample tiles with 2 stages, 2 the
                               same with 3 stages (cudamica_b200.autotune picks one by
                               measurement) (new key) */
    double lrate0, lratemax, lnatrate, lratefact, rho0, rholrate, rhomin, rhomax, rejsig;
    double phi_split_rel;   /* the threshold of phi_split = 2 (default 1e-4) (new key) */
} amica_cfg;

/* What one iteration reports; the reference prints the same quantities
 * ("Iteration %lu: lrate %.16f LL %.16f", src/amica.cu:1983). */
typedef struct amica_iter_out {
    int64_t iter;          /* 1-based */
    double  ll;            /* log-likelihood per sample and channel */
    double  lrate;         /* learning rate in effect when LL was printed */
    int64_t ll_decreased;  /* the "Likelihood decreasing!" branch was taken */
    int64_t newton;        /* 1 if the A update used the Newton step */
    int64_t nkeep;         /* samples in the sums (T minus rejected) */
    int64_t nrejected;     /* samples dropped by this iteration's rejection pass */
    double  device_ms;     /* device time of the iteration (CUDA events) */
    int64_t phi_split;     /* 1 if this iteration's E-step formed phi with the split
                              (hi + lo) correction (mixed form) */
} amica_iter_out;

typedef struct amica_ctx amica_ctx;

/* Fill cfg with the reference's defaults (include/config.h:46-83). */
int amica_default_cfg(amica_cfg *cfg);

/* Create a context on cfg->device: replaces initializeDevs()
 * (src/device.cu:190-380) and the allocation half of initializeModels()
 * (src/amica.cu:135-556).  Shapes: 2 <= nchannels <= 256, 1 <= nmmodels <= 8,
 * 1 <= nsdm <= 5 (else AMICA_ERR_UNSUPPORTED).  AMICA_PREC_MIXED runs the
 * fused tensor-core E-step up to 128 channels and, above, the split form:
 * b = W x and Psi = sum g x^T as tcgen05 TF32 contraction kernels of this
 * library around a density-only E-step kernel.  amica_kernel_name() reports "tc_tf32",
 * "split_tf32" or "plain_fp32". */
int amica_create(const amica_cfg *cfg, amica_ctx **out);

/* Release every device and host resource: replaces finalizeModels() /
 * finalizeDevs() (src/amica.cu:562-622, src/device.cu:382-426). */
int amica_destroy(amica_ctx *ctx);

/* Raw (unsphered) data, T x n float32 sample-major, host memory: replaces
 * loadMatrix() + the H2D copy (src/amica.cu:671-705, src/helpers.cu:513-553). */
int amica_load_data(amica_ctx *ctx, const float *x, int64_t n, int64_t T);

/* Same, with x already in device memory (no host copy). */
int amica_load_data_device(amica_ctx *ctx, const float *dx, int64_t n, int64_t T);

/* Centring and sphering on the GPU in FP64: replaces center() and whiten()
 * (src/preprocess.cu:31-420); do_sphere 0/1/2 as in the reference. */
int amica_preprocess(amica_ctx *ctx);

/* Use caller-provided whitened data (T x n float64), means, sphere (n x n,
 * column-major) and ldetS instead of amica_preprocess(): the reference's
 * deterministic mode (-DNORAND, src/amica.cu:731-734). */
int amica_set_sphered(amica_ctx *ctx, const double *xs, const double *means,
                      const double *sphere, double ldetS);

/* Deterministic initial state: A0 (M x n x n) and c0 (M x n) as the
 * reference's -DNORAND files give them (src/amica.cu:314-322); gm, alpha, mu,
 * beta, rho follow fix_init (src/amica.cu:337-394).  A0 == NULL draws
 * A = I + 0.05*(U - 0.5) with unit columns and c ~ N(0,1) from cfg->seed. */
int amica_init(amica_ctx *ctx, const double *A0, const double *c0);

/* One EM iteration: replaces one pass of the iteration body of runamica()
 * (src/amica.cu:820-2541).  out may be NULL. */
int amica_em_step(amica_ctx *ctx, amica_iter_out *out);

/* maxiter iterations with no host synchronisation between them (one CUDA
 * graph per iteration); hist may be NULL or hold maxiter entries. */
int amica_run(amica_ctx *ctx, int64_t maxiter, amica_iter_out *hist);

/* Current parameters (any pointer may be NULL).  W is the inverse of A used
 * by the last E-step, as the reference's weightsfile (src/amica.cu:2546-2562). */
int amica_get_params(amica_ctx *ctx, double *A, double *W, double *c, double *gm,
                     double *alpha, double *mu, double *beta, double *rho);

/* Overwrite the parameters (any pointer may be NULL = keep). */
int amica_set_params(amica_ctx *ctx, const double *A, const double *c, const double *gm,
                     const double *alpha, const double *mu, const double *beta,
                     const double *rho);

/* E-step only, at the current parameters: the FP64 sufficient statistics in
 * the flat layout of amica_stats_len() (LL numerator, then per model vsum,
 * cnew, sigma2 numerator, phi = sum g b^T, and the usum / kappa / lambda /
 * mu / beta / rho sums of src/kernels.cu:495-827).  No parameter changes. */
int amica_estep_stats(amica_ctx *ctx, double *stats);
int64_t amica_stats_len(int64_t n, int64_t M, int64_t m);

/* Per-sample outputs of the last E-step: Lt (M x T, the reference's ltall,
 * src/amica.cu:1203-1209), P (T, per-sample log-likelihood) and the keep mask
 * (T bytes).  Any pointer may be NULL. */
int amica_get_loglik(amica_ctx *ctx, double *Lt, double *P, uint8_t *keep);

/* Log-likelihood L (sum over kept samples of P, per sample and channel as the
 * reference normalises it) and its gradient with respect to W (M x n x n,
 * column-major), mu, beta and rho (M x m x n), in one sweep that recomputes
 * the responsibilities per tile.  Any gradient pointer may be NULL. */
int amica_loglik_adjoint(amica_ctx *ctx, double *ll, double *dW, double *dmu,
                         double *dbeta, double *drho);

/* Rejection mask of the reference-free rule (mean - rejsig*std of P over kept
 * samples, FP64, fixed reduction order) applied to the last E-step's P. */
int amica_reject_now(amica_ctx *ctx, int64_t *nrejected);

/* Output stage: writes the reference's raw float64 files (any path may be
 * NULL): replaces src/amica.cu:2542-2816. */
typedef struct amica_paths {
    const char *weightsfile, *afile, *cfile, *ltallfile, *gmfile, *alphafile,
               *mufile, *betafile, *rhofile, *llfile, *spherefile;
} amica_paths;
int amica_write_outputs(amica_ctx *ctx, const amica_paths *paths);

/* P(t) minus log gm_0 + ldet_0 + ldetS, as float, exactly as the kernels
 * stored it (the input of the rejection rule). */
int amica_get_p_relative(amica_ctx *ctx, float *P);

/* Resume support: set the iteration counter, learning rate and previous LL
 * (the host-side loop state of src/amica.cu:800-806) after amica_init() +
 * amica_set_params(), so a fit can continue from saved parameters. */
int amica_set_iter_state(amica_ctx *ctx, int64_t iter, double lrate, double ll_prev);

/* Sphering matrix (n x n, column-major), channel means and ldetS in use. */
int amica_get_sphere(amica_ctx *ctx, double *sphere, double *means, double *ldetS);

/* Time the fused E-step kernel alone on the context's stream with CUDA
 * events: reps back-to-back launches after one warm launch.  *launches gets
 * the number of kernels launched (may be NULL). */
int amica_time_estep(amica_ctx *ctx, int64_t reps, double *ms_per_launch, int64_t *launches);

/* Number of kernels one EM iteration launches. */
int64_t amica_launches_per_iteration(amica_ctx *ctx);

/* Self-test of the tensor-core contraction forms used by the mixed-precision
 * E-step (one CTA, host buffers): D = A B^T with A (128 x K) and B (N x K),
 * B K-major in shared memory; mode 0: A in shared memory, mode 1: A in tensor
 * memory, mode 2: A split into TF32 hi (shared) + lo (tensor memory) halves.
 * K in {16, 32, 48, 64}, N a multiple of 16 up to 64.  D is 128 x N float. */
int amica_selftest_umma(int mode, int N, int K, const float *A, const float *B, float *D,
                        int *device_err);

/* Sample-sharded fits, one context per GPU, each over a contiguous range of
 * the samples (its own load_data / set_sphered of T_shard samples, the same
 * sphering and initial state on every shard).  Replaces the reference's
 * multi-device block loop and its per-device statistics reduction
 * (src/amica.cu:1618-1920, acumulate in src/kernels.cu:834-839).
 * amica_shard_estep: the E-step over this context's samples; d_stats (DEVICE
 * memory, amica_stats_len(n, M, m) doubles) receives its sufficient
 * statistics, which are sums over samples, so that adding the vectors of all
 * shards (one all-reduce) gives those of the whole data.  It returns without
 * waiting: the statistics are written in the order of the context's stream
 * (amica_get_stream), behind which the caller queues the all-reduce.
 * amica_shard_mstep: the M-step from the added statistics d_stats (DEVICE,
 * read in stream order), nkeep_total the samples of all shards; every shard
 * runs it on the same vector, so the parameters stay identical across shards.
 * It synchronises the stream, reports device errors of both calls and fills
 * `out`.  Rejection needs every sample's P and is not available here
 * (AMICA_ERR_UNSUPPORTED). */
int amica_shard_estep(amica_ctx *ctx, double *d_stats);
int amica_shard_mstep(amica_ctx *ctx, const double *d_stats, int64_t nkeep_total,
                      amica_iter_out *out);

/* The context's CUDA stream (a cudaStream_t), on which every call of this
 * context queues its work. */
int amica_get_stream(amica_ctx *ctx, void **stream);

/* Sharded preprocessing of raw data (after amica_load_data of this shard's
 * samples), the GPU form of the reference's centring and sphering
 * (src/preprocess.cu:31-230) over the samples of every shard, with two sums
 * added across shards between the calls (DEVICE memory throughout):
 * amica_shard_colsum: the column sums of this shard (n doubles);
 * amica_shard_scatter: with the added sums of all shards and their sample
 *   count T_total, sets the mean and writes this shard's scatter about it,
 *   sum_t (x_t - mean)(x_t - mean)^T (n x n doubles);
 * amica_shard_sphere: from the added scatter of all shards, the covariance,
 *   its eigendecomposition, S and ldetS (the same on every shard), applied to
 *   this shard's samples; the context is then ready for amica_init(). */
int amica_shard_colsum(amica_ctx *ctx, double *d_sums);
int amica_shard_scatter(amica_ctx *ctx, const double *d_sums_total, int64_t T_total,
                        double *d_scatter);
int amica_shard_sphere(amica_ctx *ctx, const double *d_scatter_total, int64_t T_total);

/* Switch the fused E-step's tile shape (amica_cfg.tc_shape) of a mixed-form
 * context of at most 128 channels; the grid goes back to as many clusters as
 * fit (the partial sums are sized for every shape).  AMICA_ERR_UNSUPPORTED for
 * other contexts. */
int amica_set_tile_shape(amica_ctx *ctx, int64_t shape);

/* Test hook for the failure path of the bounded device waits: arms the next
 * amica_preprocess() of this context so that one block of its cooperative
 * eigensolver (used above 128 channels with do_sphere = 1) skips its first
 * grid-barrier arrival and every barrier wait of that launch gives up after
 * wait_cycles clock cycles.  That amica_preprocess() then returns
 * AMICA_ERR_TIMEOUT, and the context stays usable (the next one succeeds).
 * No counterpart in the reference, whose waits are host synchronisations.
 * AMICA_ERR_UNSUPPORTED for contexts that do not use the cooperative solver. */
int amica_test_arm_wait_fault(amica_ctx *ctx, int64_t wait_cycles);

/* E-step sufficient statistics with no allocation at all, for callers that
 * cannot call cudaMalloc (code running inside another framework's memory pool,
 * or a process that forbids device allocations after start-up).  No
 * counterpart in the reference: its EM loop allocates per-block buffers.
 * All pointers are DEVICE memory owned by the caller: x is T x ldx float32
 * sphered data with ldx the channel count padded to 32, 64, 128 or 256 (padding
 * channels zero); A (M x n x n), c, alpha, mu, beta, rho, gm as in
 * amica_set_params(); keep (T bytes) may be NULL, and then nkeep must be T;
 * stats receives amica_stats_len(n, M, m) doubles.  Intermediate data lives in
 * a fixed 5 MiB device array inside this library (held by every GPU that loads
 * it until exit).  The E-step grid shrinks, down to a single cluster, until its
 * per-cluster partial sums fit that array; shapes that do not fit even then
 * return AMICA_ERR_UNSUPPORTED (at n = 256 only M = 1 fits; at n = 128, M up
 * to 8 fits).  The array's device address is looked up in the current CUDA
 * context on every call, so device resets and caller-owned contexts are safe.
 * Calls share the array: calls whose GPU work overlaps race, so serialise
 * them.  The call enqueues on `stream` (a cudaStream_t, NULL = default), then
 * copies a status word to the host and synchronises that stream; it must
 * never be made while the stream is being captured into a CUDA graph. */
int amica_estep_stats_noalloc(const float *x, int64_t ldx, int64_t n, int64_t T, int64_t M,
                              int64_t m, const double *A, const double *c, const double *alpha,
                              const double *mu, const double *beta, const double *rho,
                              const double *gm, double ldetS, const uint8_t *keep, int64_t nkeep,
                              int64_t update_rho, double *stats, void *stream);

/* amica_run() in two halves, for driving several contexts (one per subject of
 * a cohort, each on its own stream) concurrently: amica_run_async() enqueues
 * `iters` replays of the iteration graph on the context's stream and returns
 * at once; amica_run_wait() waits for them, fills hist[0..iters-1] when hist
 * is not NULL, checks the device error flag and the LLs (rolling back to the
 * parameters before the batch on NaN/Inf, as amica_run does).  No counterpart
 * in the reference (its loop is synchronous). */
int amica_run_async(amica_ctx *ctx, int64_t iters);
/* Re-size the E-step grid of a created context to at most max_clusters clusters
 * (0: as many as fit); *nclusters (may be NULL) receives the grid in effect.
 * The iteration graph is re-captured on the next run.  No counterpart in the
 * reference. */
int amica_set_grid(amica_ctx *ctx, int64_t max_clusters, int64_t *nclusters);
int amica_run_wait(amica_ctx *ctx, amica_iter_out *hist);

/* A cohort: several single-model fits (nmmodels = 1, the same nsdm, the mixed
 * form, up to 128 channels each, with their own channel counts and lengths)
 * advanced together with ONE persistent tensor-core E-step launch per
 * iteration over all subjects' sample tiles (a work list of (subject, tile
 * range) items dealt evenly to one CTA per SM), each subject's inverse and
 * M-step running on its own stream around it; an iteration of the whole
 * cohort is one CUDA graph.  The subjects stay ordinary contexts (parameters,
 * outputs and history through the per-context calls).  No counterpart in the
 * reference (one fit per process).
 * amica_cohort_create: the contexts must be created, and before
 * amica_cohort_run also sphered and initialised; AMICA_ERR_UNSUPPORTED for
 * M > 1 or the plain form.  The cohort does not own the contexts.
 * amica_cohort_run: `iters` iterations of every subject; hist (may be NULL)
 * receives nsubjects x iters records, subject-major; *ms_per_iter (may be NULL)
 * the device time of one cohort iteration.  Returns the first subject's error
 * (each subject rolls back to its parameters before the call on NaN/Inf). */
typedef struct amica_cohort amica_cohort;
int amica_cohort_create(amica_ctx *const *subjects, int64_t nsubjects, amica_cohort **out);
int amica_cohort_run(amica_cohort *cohort, int64_t iters, amica_iter_out *hist, double *ms_per_iter);
int amica_cohort_destroy(amica_cohort *cohort);

/* Last CUDA runtime error code seen by any call (0 = none). */
int amica_last_cuda_error(void);

/* Message for a status code (replaces cGetErrorString, src/error.cu:14-16). */
const char *amica_status_string(int status);

/* Name of the E-step kernel a context runs ("plain_fp32" / "tc_tf32"). */
const char *amica_kernel_name(amica_ctx *ctx);

#ifdef __cplusplus
}
#endif
#endif
