/*
 * FP64 CPU oracle for one AMICA EM iteration -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the reference's iteration body
 * (src/amica.cu:820-2541 with the kernels of src/kernels.cu:227-1081 of
 * fraimondo/cudamica), used by the tests, by __graft_entry__.smoke() and by
 * bench.py's CPU-baseline leg as the checker.  The CUDA engine never calls it.
 *
 * Parity is pinned against the reference's own CUDA build run on the same
 * inputs (tests/golden/ref_*.npz, made by tests/golden/make_ref_goldens.py).
 *
 * Layouts (identical to the engine's host-facing layouts):
 *   x            T x n   sample-major (each sample's n channels contiguous)
 *   A, W         M x n x n, column-major per model (A[h][col*n + row])
 *   c            M x n
 *   alpha/mu/beta/rho  M x m x n  (channel fastest)
 *   stats        flat float64 vector, see amo_stats_len()
 */
#ifndef AMICA_ORACLE_H
#define AMICA_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int64_t n, T, M, m;
    int64_t do_newton, update_rho, rho_start_iter, newt_start_iter, maxdec;
    int64_t update_gm, update_alpha, update_A, update_mu, update_beta, do_reparm;
    int64_t do_reject, rejstart, rejint, maxrej;
    int64_t ref_y_slab_bug;   /* 1: read y of slab h*M+j in the lambda / mu-beta /
                                 rho sums, as src/amica.cu:1462,1481,1519 do */
    int64_t nthreads;
    double lrate0, lratemax, lnatrate, lratefact, rho0, rholrate, rhomin, rhomax, rejsig;
} amo_cfg;

typedef struct {
    double *A, *c, *alpha, *mu, *beta, *rho, *gm;   /* parameters, in/out */
    double *W, *ldet;                               /* out: W = A^-1 and log|det W| used */
    uint8_t *keep;                                  /* T: 1 = sample used (rejection mask) */
    double *Lt;                                     /* M x T, optional out (NULL = skip) */
    double *P;                                      /* T, optional out (needed for rejection) */
    double ldetS;
    double lrate, lratemax, ll_prev, ll;
    int64_t numdec, iter, nrej, newton, nkeep;
} amo_state;

/* Number of doubles in the flat sufficient-statistics vector:
 *   [0]            sum_t P(t)                     (log-likelihood numerator)
 *   then per model h, S = 1 + 2n + n*n + 7*m*n doubles:
 *     vsum (1), cnew_sum (n), sigma2_num (n), phi (n*n, col-major phi(i,k) at k*n+i),
 *     usum, kappa_num, lambda_num, mu_num, mu_den, beta_den, rho_num  (m*n each)
 */
int64_t amo_stats_len(int64_t n, int64_t M, int64_t m);

void amo_default_cfg(amo_cfg *cfg);

/* W_h = A_h^{-1} (partial-pivot LU) and ldet_h = sum log|u_ii| for every model. */
int amo_prepare(const amo_cfg *cfg, amo_state *st);

/* E-step sums over the kept samples with the current parameters and W. */
int amo_estep(const amo_cfg *cfg, amo_state *st, const double *x, double *stats);

/* M-step from the sums (LL bookkeeping, parameter updates, Newton / natural
 * gradient A update, reparametrisation).  Advances st->iter. */
int amo_mstep(const amo_cfg *cfg, amo_state *st, const double *stats);

/* One full iteration: prepare + estep + mstep (+ rejection on schedule). */
int amo_em_step(const amo_cfg *cfg, amo_state *st, const double *x, double *stats_scratch);

/* Rejection rule: over kept samples, mean and standard deviation (n-1) of P in
 * FP64 with a fixed reduction order (4096-sample chunks summed sequentially,
 * chunk sums summed sequentially); drop kept samples with P < mean - k*std.
 * Returns the number of newly rejected samples. */
int64_t amo_reject(const double *P, uint8_t *keep, int64_t T, double rejsig,
                   double *mean_out, double *std_out);

/* Preprocessing: means (FP64), C = Xc Xc^T / T, sphere S per do_sphere
 * (1: 2*C^{-1/2} via cyclic Jacobi eigendecomposition, 2: diag(1/std),
 * 0: I), ldetS = -log|det S|, xs = S (x - mean).  x is T x n float32. */
int amo_preprocess(const float *x, int64_t n, int64_t T, int64_t do_sphere,
                   double *xs, double *means, double *sphere, double *ldetS);

/* Symmetric eigendecomposition by cyclic Jacobi (ascending eigenvalues,
 * eigenvectors in the columns of V, column-major). */
int amo_jacobi_eig(const double *C, int64_t n, double *evals, double *V);

/* Digamma from the shifted asymptotic series used by the reference's rho update. */
double amo_psi(double x);

#ifdef __cplusplus
}
#endif
#endif
