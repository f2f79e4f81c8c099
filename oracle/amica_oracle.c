/*
 * FP64 CPU oracle for the AMICA EM iteration -- TEST INFRASTRUCTURE ONLY.
 *
 * Restates, in plain C and double precision, what the reference computes in
 * one iteration (fraimondo/cudamica, src/amica.cu:820-2541 and the kernels of
 * src/kernels.cu).  Each step below names the reference lines it follows.
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load
 * this code; the CUDA engine never does.
 *
 * Deliberate, documented departures from the reference (all measure-zero or
 * numerically equivalent):
 *   - W = A^{-1} by partial-pivot LU instead of pinv() by SVD
 *     (src/amica.cu:27-127); identical for every non-singular A.
 *   - log|det W| = -sum_i log|u_ii| of A's LU instead of the log of the LU
 *     diagonal product of W (src/amica.cu:881-919, src/kernels.cu:190-196);
 *     same value without the overflow of the product.
 *   - |y| is clamped below at FLT_MIN before pow/log/division, so y == 0
 *     exactly gives finite sums where the reference gives NaN
 *     (src/kernels.cu:717, :805-807).
 */
#define _GNU_SOURCE
#include "amica_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

#define TINY_ABS 1.1754943508222875e-38 /* FLT_MIN: guard for |y| == 0 */

int64_t amo_stats_len(int64_t n, int64_t M, int64_t m) {
    return 1 + M * (1 + 2 * n + n * n + 7 * m * n);
}

/* offsets inside one model's block of the stats vector */
typedef struct {
    int64_t S, vs, cn, s2, phi, us, kn, ln, mn, md, bd, rn;
} amo_off;

static amo_off offsets(int64_t n, int64_t m) {
    amo_off o;
    int64_t mn = m * n;
    o.vs = 0;
    o.cn = 1;
    o.s2 = 1 + n;
    o.phi = 1 + 2 * n;
    o.us = o.phi + n * n;
    o.kn = o.us + mn;
    o.ln = o.kn + mn;
    o.mn = o.ln + mn;
    o.md = o.mn + mn;
    o.bd = o.md + mn;
    o.rn = o.bd + mn;
    o.S = o.rn + mn;
    return o;
}

void amo_default_cfg(amo_cfg *c) {
    /* include/config.h:46-83 of the reference */
    memset(c, 0, sizeof(*c));
    c->M = 1;
    c->m = 3;
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
    c->rejsig = 3.0;
    c->nthreads = 1;
    c->lrate0 = 0.1;
    c->lratemax = 1.0;
    c->lnatrate = 0.1;
    c->lratefact = 0.5;
    c->rho0 = 1.5;
    c->rholrate = 0.1;
    c->rhomin = 1.0;
    c->rhomax = 2.0;
}

/* ---------------------------------------------------------------- algebra */

/* In-place partial-pivot LU of a column-major n x n matrix. */
static int lu_factor(double *a, int64_t n, int64_t *piv) {
    for (int64_t k = 0; k < n; k++) {
        int64_t p = k;
        double best = fabs(a[k * n + k]);
        for (int64_t i = k + 1; i < n; i++) {
            double v = fabs(a[k * n + i]);
            if (v > best) { best = v; p = i; }
        }
        piv[k] = p;
        if (best == 0.0) return -1;
        if (p != k)
            for (int64_t j = 0; j < n; j++) {
                double t = a[j * n + k];
                a[j * n + k] = a[j * n + p];
                a[j * n + p] = t;
            }
        double inv = 1.0 / a[k * n + k];
        for (int64_t i = k + 1; i < n; i++) a[k * n + i] *= inv;
        for (int64_t j = k + 1; j < n; j++) {
            double f = a[j * n + k];
            if (f != 0.0)
                for (int64_t i = k + 1; i < n; i++) a[j * n + i] -= a[k * n + i] * f;
        }
    }
    return 0;
}

/* W = A^{-1}; returns log|det A| in *logdet. */
static int inverse(const double *A, int64_t n, double *W, double *logdet) {
    double *lu = malloc(sizeof(double) * n * n);
    int64_t *piv = malloc(sizeof(int64_t) * n);
    memcpy(lu, A, sizeof(double) * n * n);
    int rc = lu_factor(lu, n, piv);
    if (rc == 0) {
        double ld = 0.0;
        for (int64_t k = 0; k < n; k++) ld += log(fabs(lu[k * n + k]));
        *logdet = ld;
        for (int64_t j = 0; j < n; j++) {
            double *col = W + j * n;
            for (int64_t i = 0; i < n; i++) col[i] = (i == j) ? 1.0 : 0.0;
            for (int64_t k = 0; k < n; k++) {
                int64_t p = piv[k];
                if (p != k) { double t = col[k]; col[k] = col[p]; col[p] = t; }
            }
            for (int64_t k = 0; k < n; k++) {        /* L y = b (unit lower) */
                double v = col[k];
                for (int64_t i = k + 1; i < n; i++) col[i] -= lu[k * n + i] * v;
            }
            for (int64_t k = n - 1; k >= 0; k--) {   /* U x = y */
                col[k] /= lu[k * n + k];
                double v = col[k];
                for (int64_t i = 0; i < k; i++) col[i] -= lu[k * n + i] * v;
            }
        }
    }
    free(lu);
    free(piv);
    return rc;
}

double amo_psi(double x) {
    /* Digamma: recurrence psi(x) = psi(x+6) - sum_{k=0}^{5} 1/(x+k), then the
     * Stirling-type asymptotic series of psi at x+6 with the Bernoulli
     * coefficients B_2k/(2k) up to x^-18 -- the method of the reference's
     * psi() (src/kernels.cu:906-929). */
    static const double coef[9] = {
        1.0 / 12.0, -1.0 / 120.0, 1.0 / 252.0, -1.0 / 240.0, 1.0 / 132.0,
        -691.0 / 32760.0, 1.0 / 12.0, -3617.0 / 8160.0, 43867.0 / 14364.0};
    double s = x + 6.0;
    double r = log(s) - 1.0 / (2.0 * s);
    double s2 = s * s, p = s2;
    for (int k = 0; k < 9; k++) {
        r -= coef[k] / p;
        p *= s2;
    }
    for (int k = 5; k >= 0; k--) r -= 1.0 / (x + k);
    return r;
}

int amo_jacobi_eig(const double *Cin, int64_t n, double *evals, double *V) {
    double *a = malloc(sizeof(double) * n * n);
    memcpy(a, Cin, sizeof(double) * n * n);
    for (int64_t i = 0; i < n * n; i++) V[i] = 0.0;
    for (int64_t i = 0; i < n; i++) V[i * n + i] = 1.0;
    double fro = 0.0;
    for (int64_t i = 0; i < n * n; i++) fro += a[i] * a[i];
    for (int sweep = 0; sweep < 100; sweep++) {
        double off = 0.0;
        for (int64_t q = 0; q < n; q++)
            for (int64_t p = 0; p < q; p++) off += a[q * n + p] * a[q * n + p];
        if (off <= 1e-30 * fro) break;
        for (int64_t p = 0; p < n - 1; p++) {
            for (int64_t q = p + 1; q < n; q++) {
                double apq = a[q * n + p];
                if (fabs(apq) < 1e-300) continue;
                double app = a[p * n + p], aqq = a[q * n + q];
                double theta = (aqq - app) / (2.0 * apq);
                double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
                double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
                for (int64_t k = 0; k < n; k++) {   /* columns p, q */
                    double akp = a[p * n + k], akq = a[q * n + k];
                    a[p * n + k] = c * akp - s * akq;
                    a[q * n + k] = s * akp + c * akq;
                }
                for (int64_t k = 0; k < n; k++) {   /* rows p, q */
                    double apk = a[k * n + p], aqk = a[k * n + q];
                    a[k * n + p] = c * apk - s * aqk;
                    a[k * n + q] = s * apk + c * aqk;
                }
                for (int64_t k = 0; k < n; k++) {
                    double vkp = V[p * n + k], vkq = V[q * n + k];
                    V[p * n + k] = c * vkp - s * vkq;
                    V[q * n + k] = s * vkp + c * vkq;
                }
            }
        }
    }
    for (int64_t i = 0; i < n; i++) evals[i] = a[i * n + i];
    /* selection sort, ascending, with the eigenvector columns */
    for (int64_t i = 0; i < n; i++) {
        int64_t b = i;
        for (int64_t j = i + 1; j < n; j++)
            if (evals[j] < evals[b]) b = j;
        if (b != i) {
            double t = evals[i]; evals[i] = evals[b]; evals[b] = t;
            for (int64_t k = 0; k < n; k++) {
                double u = V[i * n + k]; V[i * n + k] = V[b * n + k]; V[b * n + k] = u;
            }
        }
    }
    free(a);
    return 0;
}

int amo_preprocess(const float *x, int64_t n, int64_t T, int64_t do_sphere,
                   double *xs, double *means, double *S, double *ldetS) {
    /* centring: src/preprocess.cu:31-85 (the reference accumulates in float,
     * src/kernels.cu:66; this restatement uses double) */
    for (int64_t i = 0; i < n; i++) means[i] = 0.0;
    for (int64_t t = 0; t < T; t++)
        for (int64_t i = 0; i < n; i++) means[i] += (double)x[t * n + i];
    for (int64_t i = 0; i < n; i++) means[i] /= (double)T;
    for (int64_t t = 0; t < T; t++)
        for (int64_t i = 0; i < n; i++) xs[t * n + i] = (double)x[t * n + i] - means[i];

    for (int64_t i = 0; i < n * n; i++) S[i] = 0.0;
    double ld = 0.0;
    if (do_sphere == 1) {
        /* src/preprocess.cu:110-282: C = X X^T / T, S = 2 C^{-1/2} */
        double *C = calloc(n * n, sizeof(double));
        for (int64_t t = 0; t < T; t++) {
            const double *r = xs + t * n;
            for (int64_t k = 0; k < n; k++) {
                double v = r[k];
                for (int64_t i = 0; i <= k; i++) C[k * n + i] += r[i] * v;
            }
        }
        for (int64_t k = 0; k < n; k++)
            for (int64_t i = 0; i <= k; i++) {
                C[k * n + i] /= (double)T;
                C[i * n + k] = C[k * n + i];
            }
        double *ev = malloc(sizeof(double) * n), *V = malloc(sizeof(double) * n * n);
        amo_jacobi_eig(C, n, ev, V);
        for (int64_t e = 0; e < n; e++) {
            double f = 2.0 / sqrt(ev[e]);
            ld += log(f);
            for (int64_t k = 0; k < n; k++)
                for (int64_t i = 0; i < n; i++) S[k * n + i] += V[e * n + i] * f * V[e * n + k];
        }
        free(C); free(ev); free(V);
    } else if (do_sphere == 2) {
        /* src/kernels.cu:148-161: 1/sqrt(sum (x - mean)^2 / (T-1)) */
        for (int64_t i = 0; i < n; i++) {
            double mu = 0.0, m2 = 0.0;
            for (int64_t t = 0; t < T; t++) mu += xs[t * n + i];
            mu /= (double)T;
            for (int64_t t = 0; t < T; t++) {
                double d = fabs(xs[t * n + i] - mu);
                m2 += d * d;
            }
            double f = 1.0 / sqrt(m2 / (double)(T - 1));
            S[i * n + i] = f;
            ld += log(fabs(f));
        }
    } else {
        for (int64_t i = 0; i < n; i++) S[i * n + i] = 1.0;
    }
    *ldetS = -ld;
    if (do_sphere != 0) {
        double *row = malloc(sizeof(double) * n);
        for (int64_t t = 0; t < T; t++) {
            double *r = xs + t * n;
            for (int64_t i = 0; i < n; i++) {
                double acc = 0.0;
                for (int64_t k = 0; k < n; k++) acc += S[k * n + i] * r[k];
                row[i] = acc;
            }
            memcpy(r, row, sizeof(double) * n);
        }
        free(row);
    }
    return 0;
}

/* ---------------------------------------------------------------- E-step */

/* Per-sample arithmetic type.  The default build is FP64 throughout; built
 * with -DAMO_FP32_ESTEP (liboracle32.so) the per-sample quantities (b, y, the
 * densities, z, Lt, P, v, g) are FP32 and only the sums over samples stay
 * FP64: the FP32 host rendering that the CPU baseline times beside the FP64
 * one.  The M-step is FP64 in both. */
#ifdef AMO_FP32_ESTEP
typedef float ereal;
#define EPOW powf
#define EEXP expf
#define ELOG logf
#define EFABS fabsf
#define ECOPYSIGN copysignf
#define ETINY ((float)TINY_ABS)
#else
typedef double ereal;
#define EPOW pow
#define EEXP exp
#define ELOG log
#define EFABS fabs
#define ECOPYSIGN copysign
#define ETINY TINY_ABS
#endif

typedef struct {
    const amo_cfg *cfg;
    amo_state *st;
    const double *x;
    const double *Cq, *sqb, *wc, *ltc;
    int64_t t0, t1;
    double *acc;
} ework;

static void *estep_worker(void *arg) {
    ework *w = (ework *)arg;
    const amo_cfg *cfg = w->cfg;
    amo_state *st = w->st;
    const int64_t n = cfg->n, M = cfg->M, m = cfg->m, T = cfg->T;
    const amo_off o = offsets(n, m);
    ereal *b = malloc(sizeof(ereal) * M * n);
    ereal *y = malloc(sizeof(ereal) * M * m * n);
    ereal *z = malloc(sizeof(ereal) * M * m * n);
    ereal *Lt = malloc(sizeof(ereal) * M);
    ereal *v = malloc(sizeof(ereal) * M);
    ereal *g = malloc(sizeof(ereal) * n);
    ereal *xt = malloc(sizeof(ereal) * n);
    /* the parameters in the per-sample type */
    ereal *W = malloc(sizeof(ereal) * M * n * n);
    ereal *wc = malloc(sizeof(ereal) * M * n);
    ereal *sqb = malloc(sizeof(ereal) * M * m * n);
    ereal *mu = malloc(sizeof(ereal) * M * m * n);
    ereal *rho = malloc(sizeof(ereal) * M * m * n);
    ereal *Cq = malloc(sizeof(ereal) * M * m * n);
    for (int64_t e = 0; e < M * n * n; e++) W[e] = (ereal)st->W[e];
    for (int64_t e = 0; e < M * n; e++) wc[e] = (ereal)w->wc[e];
    for (int64_t e = 0; e < M * m * n; e++) {
        sqb[e] = (ereal)w->sqb[e];
        mu[e] = (ereal)st->mu[e];
        rho[e] = (ereal)st->rho[e];
        Cq[e] = (ereal)w->Cq[e];
    }
    double *acc = w->acc;

    for (int64_t t = w->t0; t < w->t1; t++) {
        const double *xd = w->x + t * n;
        for (int64_t k = 0; k < n; k++) xt[k] = (ereal)xd[k];
        for (int64_t h = 0; h < M; h++) {
            /* b = W x - W c: cublasDgemm + Dgemv + substract, src/amica.cu:1054-1102 */
            const ereal *Wh = W + h * n * n;
            ereal *bh = b + h * n;
            for (int64_t i = 0; i < n; i++) bh[i] = 0;
            for (int64_t k = 0; k < n; k++) {
                ereal xk = xt[k];
                const ereal *col = Wh + k * n;
                for (int64_t i = 0; i < n; i++) bh[i] += col[i] * xk;
            }
            for (int64_t i = 0; i < n; i++) bh[i] -= wc[h * n + i];
            ereal sum_lse = 0;
            for (int64_t i = 0; i < n; i++) {
                ereal q[64];
                ereal qmax = -INFINITY;
                for (int64_t j = 0; j < m; j++) {
                    int64_t idx = (h * m + j) * n + i;
                    /* betabyxminusmu, src/kernels.cu:251-272 */
                    ereal yv = sqb[idx] * (bh[i] - mu[idx]);
                    y[idx] = yv;
                    ereal ay = EFABS(yv);
                    if (ay < ETINY) ay = ETINY;
                    /* logalogblogpfun, src/kernels.cu:282-307 */
                    q[j] = Cq[idx] - EPOW(ay, rho[idx]);
                    if (q[j] > qmax) qmax = q[j];
                }
                /* updateltz, src/kernels.cu:317-366 */
                ereal s = 0;
                for (int64_t j = 0; j < m; j++) s += EEXP(q[j] - qmax);
                ereal lse = qmax + ELOG(s);
                for (int64_t j = 0; j < m; j++) z[(h * m + j) * n + i] = (ereal)1 / EEXP(lse - q[j]);
                sum_lse += lse;
            }
            Lt[h] = (ereal)w->ltc[h] + sum_lse;
        }
        /* updatell, src/kernels.cu:376-450 */
        ereal lmax = Lt[0];
        for (int64_t h = 1; h < M; h++) if (Lt[h] > lmax) lmax = Lt[h];
        ereal s = 0;
        for (int64_t h = 0; h < M; h++) s += EEXP(Lt[h] - lmax);
        ereal P = lmax + ELOG(s);
        for (int64_t h = 0; h < M; h++) v[h] = (ereal)1 / EEXP(P - Lt[h]);
        if (st->Lt) for (int64_t h = 0; h < M; h++) st->Lt[h * T + t] = Lt[h];
        if (st->P) st->P[t] = P;
        if (st->keep && !st->keep[t]) continue;

        acc[0] += P;
        for (int64_t h = 0; h < M; h++) {
            double *A = acc + 1 + h * o.S;
            const ereal vh = v[h];
            const ereal *bh = b + h * n;
            A[o.vs] += vh;                                   /* Dasum, src/amica.cu:1585 */
            for (int64_t i = 0; i < n; i++) {
                A[o.cn + i] += vh * xt[i];                   /* cnew Dgemv, :1280-1292 */
                A[o.s2 + i] += vh * (bh[i] * bh[i]);         /* pow2 + Dgemv, :1300-1323 */
                g[i] = 0;
            }
            for (int64_t j = 0; j < m; j++) {
                for (int64_t i = 0; i < n; i++) {
                    int64_t idx = (h * m + j) * n + i;
                    ereal rh = rho[idx];
                    ereal u = vh * z[idx];                   /* computeu, src/kernels.cu:473-484 */
                    ereal yv = y[idx];
                    ereal ay = EFABS(yv);
                    if (ay < ETINY) ay = ETINY;
                    /* computefp, src/kernels.cu:540-553 */
                    ereal fp = rh * ECOPYSIGN(EPOW(ay, rh - 1), yv);
                    ereal ufp = u * fp;
                    g[i] += sqb[idx] * ufp;                  /* computeg, :561-574 */
                    int64_t mi = j * n + i;
                    A[o.us + mi] += u;                       /* getusum, :495-532 */
                    A[o.kn + mi] += ufp * fp;                /* getdkappanumer, :583-621 */
                    ereal yy = yv;
                    if (cfg->ref_y_slab_bug) {               /* OFFSET4D2D(y, j, h, M) */
                        int64_t slab = h * M + j;
                        yy = y[slab * n + i];
                    }
                    ereal ayy = EFABS(yy);
                    if (ayy < ETINY) ayy = ETINY;
                    ereal yys = ECOPYSIGN(ayy, yy);
                    ereal lv = fp * yy - 1;                  /* getdlambdanumer, :630-671 */
                    A[o.ln + mi] += u * (lv * lv);
                    A[o.mn + mi] += ufp;                     /* getbetamu, :680-763 */
                    if (rh <= 2) {
                        A[o.md + mi] += ufp / yys;
                        A[o.bd + mi] += ufp * yy;
                    } else {
                        A[o.md + mi] += ufp * fp;
                        A[o.bd + mi] += u * EPOW(ayy, rh);
                    }
                    if (cfg->update_rho) {                   /* getdrhonumer, :785-827 */
                        ereal pv = EPOW(ayy, rh);
                        A[o.rn + mi] += u * (pv * ELOG(pv));
                    }
                }
            }
            /* phi = g b^T, src/amica.cu:1535-1550 */
            double *phi = A + o.phi;
            for (int64_t k = 0; k < n; k++) {
                ereal bk = bh[k];
                double *col = phi + k * n;
                for (int64_t i = 0; i < n; i++) col[i] += g[i] * bk;
            }
        }
    }
    free(b); free(y); free(z); free(Lt); free(v); free(g); free(xt);
    free(W); free(wc); free(sqb); free(mu); free(rho); free(Cq);
    return NULL;
}

int amo_prepare(const amo_cfg *cfg, amo_state *st) {
    const int64_t n = cfg->n;
    for (int64_t h = 0; h < cfg->M; h++) {
        double ldA = 0.0;
        if (inverse(st->A + h * n * n, n, st->W + h * n * n, &ldA) != 0) return -10;
        st->ldet[h] = -ldA;
    }
    return 0;
}

int amo_estep(const amo_cfg *cfg, amo_state *st, const double *x, double *stats) {
    const int64_t n = cfg->n, M = cfg->M, m = cfg->m;
    if (m > 64) return -3;
    const amo_off o = offsets(n, m);
    const int64_t L = amo_stats_len(n, M, m);
    double *Cq = malloc(sizeof(double) * M * m * n);
    double *sqb = malloc(sizeof(double) * M * m * n);
    double *wc = malloc(sizeof(double) * M * n);
    double *ltc = malloc(sizeof(double) * M);
    for (int64_t idx = 0; idx < M * m * n; idx++) {
        /* constant part of Q: log(alpha) + 0.5 log(beta) - log 2 - lgamma(1 + 1/rho) */
        double a = st->alpha[idx], be = st->beta[idx], r = st->rho[idx];
        Cq[idx] = log(a) + 0.5 * log(be) - M_LN2 - lgamma(1.0 + 1.0 / r);
        sqb[idx] = sqrt(be);
    }
    for (int64_t h = 0; h < M; h++) {
        /* Lt = log(gm) + ldet + ldetS, src/amica.cu:1009 */
        ltc[h] = log(st->gm[h]) + st->ldet[h] + st->ldetS;
        const double *Wh = st->W + h * n * n;
        for (int64_t i = 0; i < n; i++) {
            double acc = 0.0;
            for (int64_t k = 0; k < n; k++) acc += Wh[k * n + i] * st->c[h * n + k];
            wc[h * n + i] = acc;
        }
    }
    int64_t nt = cfg->nthreads > 0 ? cfg->nthreads : 1;
    if (nt > cfg->T) nt = 1;
    ework *ws = calloc(nt, sizeof(ework));
    pthread_t *th = calloc(nt, sizeof(pthread_t));
    for (int64_t k = 0; k < nt; k++) {
        ws[k].cfg = cfg; ws[k].st = st; ws[k].x = x;
        ws[k].Cq = Cq; ws[k].sqb = sqb; ws[k].wc = wc; ws[k].ltc = ltc;
        ws[k].t0 = cfg->T * k / nt;
        ws[k].t1 = cfg->T * (k + 1) / nt;
        ws[k].acc = calloc(L, sizeof(double));
        if (nt > 1) pthread_create(&th[k], NULL, estep_worker, &ws[k]);
    }
    if (nt == 1) estep_worker(&ws[0]);
    for (int64_t i = 0; i < L; i++) stats[i] = 0.0;
    for (int64_t k = 0; k < nt; k++) {
        if (nt > 1) pthread_join(th[k], NULL);
        for (int64_t i = 0; i < L; i++) stats[i] += ws[k].acc[i];
        free(ws[k].acc);
    }
    /* per-block factors applied after the sample sums:
     * kappa_numer = beta * sum (src/kernels.cu:616), mu_denom = sqrt(beta) * sum
     * (:745), beta_denom = rho * sum for rho > 2 (:748-750) */
    for (int64_t h = 0; h < M; h++) {
        double *A = stats + 1 + h * o.S;
        for (int64_t mi = 0; mi < m * n; mi++) {
            int64_t idx = h * m * n + mi;
            A[o.kn + mi] *= st->beta[idx];
            A[o.md + mi] *= sqb[idx];
            if (st->rho[idx] > 2.0) A[o.bd + mi] *= st->rho[idx];
        }
    }
    int64_t nk = 0;
    for (int64_t t = 0; t < cfg->T; t++) nk += (st->keep == NULL) || st->keep[t];
    st->nkeep = nk;
    free(ws); free(th); free(Cq); free(sqb); free(wc); free(ltc);
    return 0;
}

/* ---------------------------------------------------------------- M-step */

int amo_mstep(const amo_cfg *cfg, amo_state *st, const double *stats) {
    const int64_t n = cfg->n, M = cfg->M, m = cfg->m, mn = m * n;
    const amo_off o = offsets(n, m);
    const int64_t iter = st->iter + 1;
    const double Tk = (double)st->nkeep;

    /* LL = sum P / (n T) and the lrate decay, src/amica.cu:1981-1993 */
    st->ll = stats[0] / ((double)n * Tk);
    if (iter > 1 && st->ll < st->ll_prev) {
        st->lrate *= cfg->lratefact;
        st->numdec += 1;
        if (st->numdec > cfg->maxdec) {
            st->lratemax *= cfg->lratefact;   /* never read again: :2281-2285 use the config value */
            st->numdec = 0;
        }
    }
    st->ll_prev = st->ll;

    double *kappa = calloc(M * n, sizeof(double)), *lambda = calloc(M * n, sizeof(double));
    double *sig2 = malloc(sizeof(double) * M * n), *cnew = malloc(sizeof(double) * M * n);
    double *phi = malloc(sizeof(double) * M * n * n);
    /* A model whose responsibilities sum to less than one sample explains no
     * data: it is frozen (A, c and its mixture parameters kept, gm floored at
     * 1e-300), where the reference's divisions by vsum and usum would make its
     * parameters non-finite.  The GPU engine applies the same rule. */
    int *frozen = calloc(M, sizeof(int));
    for (int64_t h = 0; h < M; h++) {
        const double *S = stats + 1 + h * o.S;
        const double vsum = S[o.vs];
        if (!(vsum >= 1.0)) {
            frozen[h] = 1;
            if (cfg->update_gm) st->gm[h] = fmax(vsum / Tk, 1e-300);
            for (int64_t i = 0; i < n; i++) cnew[h * n + i] = st->c[h * n + i];
            continue;
        }
        if (cfg->update_gm) st->gm[h] = vsum / Tk;                 /* :1995-2000 */
        for (int64_t mi = 0; mi < mn; mi++)                         /* alpha = usum / vsum, :2006-2023 */
            if (cfg->update_alpha) st->alpha[h * mn + mi] = S[o.us + mi] * (1.0 / vsum);
        for (int64_t i = 0; i < n; i++) {                           /* :2025-2053 */
            sig2[h * n + i] = S[o.s2 + i] * (1.0 / vsum);
            cnew[h * n + i] = S[o.cn + i] * (1.0 / vsum);
        }
        for (int64_t k = 0; k < n * n; k++) phi[h * n * n + k] = S[o.phi + k] * (1.0 / vsum);
        /* updatekappalambda (new alpha, old mu), src/kernels.cu:848-867 */
        for (int64_t j = 0; j < m; j++)
            for (int64_t i = 0; i < n; i++) {
                int64_t mi = j * n + i, idx = h * mn + mi;
                double us = S[o.us + mi];
                if (!(us > 0.0)) continue;    /* a component with no responsibility (see below) */
                double dk = S[o.kn + mi] / us;
                double a = st->alpha[idx];
                kappa[h * n + i] += dk * a;
                double muv = st->mu[idx];
                lambda[h * n + i] += (muv * muv * dk + S[o.ln + mi] / us) * a;
            }
        /* A mixture component with no responsibility at all (usum = 0) keeps its
         * mu, beta and rho and is left out of kappa and lambda (its alpha is 0),
         * where the reference's 0/0 would make the model non-finite; the GPU
         * engine applies the same rule. */
        for (int64_t mi = 0; mi < mn; mi++) {
            int64_t idx = h * mn + mi;
            if (!(S[o.us + mi] > 0.0)) continue;
            if (cfg->update_mu)                                     /* divide + acumulate, :2095-2115 */
                st->mu[idx] += S[o.mn + mi] / S[o.md + mi];
            if (cfg->update_beta) {                                 /* getbetanumer + divide + multiply */
                double bnum = (st->rho[idx] > 2.0) ? 0.0 : S[o.us + mi];
                st->beta[idx] *= bnum / S[o.bd + mi];
            }
        }
        if (cfg->update_rho && iter >= cfg->rho_start_iter) {       /* updaterho, src/kernels.cu:937-954 */
            for (int64_t mi = 0; mi < mn; mi++) {
                int64_t idx = h * mn + mi;
                if (!(S[o.us + mi] > 0.0)) continue;
                double r = st->rho[idx];
                double ps = amo_psi(1.0 + 1.0 / r);
                double d = 1.0 - (r / ps) * S[o.rn + mi] / S[o.us + mi];
                r = r + cfg->rholrate * d;
                if (r > cfg->rhomax) r = cfg->rhomax;
                else if (r < cfg->rhomin) r = cfg->rhomin;
                st->rho[idx] = r;
            }
        }
    }

    st->newton = 0;
    if (cfg->update_A) {
        double *B = malloc(sizeof(double) * M * n * n);
        int *use_newton = calloc(M, sizeof(int));
        int no_newt = 0;
        for (int64_t h = 0; h < M; h++) {
            const double *ph = phi + h * n * n;
            double *Bh = B + h * n * n;
            if (frozen[h]) continue;
            /* denoms = (kappa sigma2)(kappa sigma2)^T; bflag counts entries <= 1
             * over the full n x n grid, diagonal included (src/kernels.cu:975-979) */
            int64_t bflag = 0;
            for (int64_t c = 0; c < n; c++)
                for (int64_t r = 0; r < n; r++) {
                    double d = (kappa[h * n + r] * sig2[h * n + r]) * (kappa[h * n + c] * sig2[h * n + c]);
                    if (d <= 1.0) bflag++;
                }
            if (bflag > 0) no_newt = 1;
            use_newton[h] = (bflag == 0 && cfg->do_newton && iter >= cfg->newt_start_iter);
            if (use_newton[h]) {
                /* getB + updateBDiagonal, src/kernels.cu:982-1000 */
                for (int64_t c = 0; c < n; c++)
                    for (int64_t r = 0; r < n; r++) {
                        double ksr = kappa[h * n + r] * sig2[h * n + r];
                        double ksc = kappa[h * n + c] * sig2[h * n + c];
                        double nom = -sig2[h * n + r] * kappa[h * n + c];
                        Bh[c * n + r] = (nom * (-ph[c * n + r]) + (-ph[r * n + c])) / (ksr * ksc - 1.0);
                    }
                for (int64_t i = 0; i < n; i++)
                    Bh[i * n + i] = (1.0 - ph[i * n + i]) / lambda[h * n + i];
            } else {
                /* geteyemphi, src/kernels.cu:1003-1014 */
                for (int64_t c = 0; c < n; c++)
                    for (int64_t r = 0; r < n; r++)
                        Bh[c * n + r] = (r == c ? 1.0 : 0.0) - ph[c * n + r];
            }
        }
        /* lrate schedule, src/amica.cu:2281-2285 */
        double step = st->lrate < 0.1 ? st->lrate : 0.1;
        if (iter >= cfg->newt_start_iter && cfg->do_newton && no_newt == 0) {
            st->lrate = fmin(cfg->lratemax, st->lrate + step);
            st->newton = 1;
        } else {
            st->lrate = fmin(cfg->lnatrate, st->lrate + step);
        }
        double *Anew = malloc(sizeof(double) * n * n);
        double *norms = malloc(sizeof(double) * n);
        double *dc = malloc(sizeof(double) * n);
        for (int64_t h = 0; h < M; h++) {
            /* A <- A +/- lrate * A * B, src/amica.cu:2317-2342 */
            if (frozen[h]) continue;
            double *Ah = st->A + h * n * n;
            const double *Bh = B + h * n * n;
            double al = use_newton[h] ? st->lrate : -st->lrate;
            for (int64_t c = 0; c < n; c++)
                for (int64_t r = 0; r < n; r++) {
                    double acc = 0.0;
                    for (int64_t k = 0; k < n; k++) acc += Ah[k * n + r] * Bh[c * n + k];
                    Anew[c * n + r] = al * acc + Ah[c * n + r];
                }
            memcpy(Ah, Anew, sizeof(double) * n * n);
        }
        if (cfg->do_reparm) {
            for (int64_t h = 0; h < M; h++) {
                /* normalizeAsave + normalizemubeta, src/kernels.cu:1023-1052 */
                if (frozen[h]) continue;
                double *Ah = st->A + h * n * n;
                for (int64_t c = 0; c < n; c++) {
                    double s = 0.0;
                    for (int64_t r = 0; r < n; r++) s += Ah[c * n + r] * Ah[c * n + r];
                    norms[c] = sqrt(s);
                    for (int64_t r = 0; r < n; r++) Ah[c * n + r] /= norms[c];
                }
                for (int64_t j = 0; j < m; j++)
                    for (int64_t i = 0; i < n; i++) {
                        int64_t idx = h * mn + j * n + i;
                        st->mu[idx] *= norms[i];
                        st->beta[idx] /= (norms[i] * norms[i]);
                    }
            }
            for (int64_t h = 0; h < M; h++) {
                /* cnewminusc + W (cnew - c) + substract, src/amica.cu:2402-2437,
                 * with W from the start of the iteration */
                if (frozen[h]) continue;
                const double *Wh = st->W + h * n * n;
                for (int64_t k = 0; k < n; k++) dc[k] = cnew[h * n + k] - st->c[h * n + k];
                for (int64_t i = 0; i < n; i++) {
                    double acc = 0.0;
                    for (int64_t k = 0; k < n; k++) acc += Wh[k * n + i] * dc[k];
                    for (int64_t j = 0; j < m; j++) st->mu[h * mn + j * n + i] -= acc;
                }
            }
        }
        free(Anew); free(norms); free(dc); free(B); free(use_newton);
    }
    /* c <- cnew, src/amica.cu:2456-2462 */
    memcpy(st->c, cnew, sizeof(double) * M * n);
    st->iter = iter;
    free(kappa); free(lambda); free(sig2); free(cnew); free(phi); free(frozen);
    return 0;
}

int64_t amo_reject(const double *P, uint8_t *keep, int64_t T, double rejsig,
                   double *mean_out, double *std_out) {
    const int64_t CH = 4096;
    double s1 = 0.0;
    int64_t nk = 0;
    for (int64_t c0 = 0; c0 < T; c0 += CH) {
        double cs = 0.0;
        int64_t c1 = c0 + CH < T ? c0 + CH : T;
        for (int64_t t = c0; t < c1; t++)
            if (keep[t]) { cs = cs + P[t]; nk++; }
        s1 = s1 + cs;
    }
    if (nk < 2) return 0;
    double mean = s1 / (double)nk;
    double s2 = 0.0;
    for (int64_t c0 = 0; c0 < T; c0 += CH) {
        double cs = 0.0;
        int64_t c1 = c0 + CH < T ? c0 + CH : T;
        for (int64_t t = c0; t < c1; t++)
            if (keep[t]) {
                double d = P[t] - mean;
                double dd = d * d;
                cs = cs + dd;
            }
        s2 = s2 + cs;
    }
    double sd = sqrt(s2 / (double)(nk - 1));
    double thr = mean - rejsig * sd;
    int64_t dropped = 0;
    for (int64_t t = 0; t < T; t++)
        if (keep[t] && P[t] < thr) { keep[t] = 0; dropped++; }
    if (mean_out) *mean_out = mean;
    if (std_out) *std_out = sd;
    return dropped;
}

int amo_em_step(const amo_cfg *cfg, amo_state *st, const double *x, double *stats) {
    int rc = amo_prepare(cfg, st);
    if (rc) return rc;
    rc = amo_estep(cfg, st, x, stats);
    if (rc) return rc;
    rc = amo_mstep(cfg, st, stats);
    if (rc) return rc;
    const int64_t it = st->iter;
    if (cfg->do_reject && st->P && st->keep && st->nrej < cfg->maxrej &&
        it >= cfg->rejstart && ((it - cfg->rejstart) % (cfg->rejint > 0 ? cfg->rejint : 1)) == 0) {
        amo_reject(st->P, st->keep, cfg->T, cfg->rejsig, NULL, NULL);
        st->nrej += 1;
    }
    return 0;
}
