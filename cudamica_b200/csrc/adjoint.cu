// Hand-written adjoint of the AMICA log-likelihood.
//
// L = sum_t P(t),  P(t) = log sum_h exp(Lt_h(t)),
// Lt_h(t) = log gm_h + log|det W_h| + ldetS + sum_i log sum_j exp(Q_hij(t)),
// Q = log alpha + 0.5 log beta - log 2 - lgamma(1 + 1/rho) - |y|^rho,
// y = sqrt(beta) (b - mu),  b = W_h (x_t - c_h)
// (the density of src/kernels.cu:282-307 and the likelihood of :317-450).
//
// With u = v_h z_hij = dP/dQ and f' = rho sign(y) |y|^(rho-1):
//   dL/dmu   = sqrt(beta) sum u f'
//   dL/dbeta = (sum u - sum u f' y) / (2 beta)
//   dL/drho  = sum u psi(1 + 1/rho) / rho^2 - sum u |y|^rho log|y|^rho / rho
//   dL/dW_h  = (sum v_h) W_h^{-T} - (sum g (x - c_h)^T),  g = sum_j sqrt(beta) u f'
// Every sum is one the fused E-step already forms per tile (it recomputes the
// responsibilities from b and never stores the M*m*n*T posterior), so the
// adjoint sweep IS the E-step kernel run in gradient mode, followed by this
// FP64 finalisation.  The natural-gradient direction the M-step uses,
// I - phi, equals (dL/dW_h) W_h^T / vsum_h.
#include <cmath>

#include "common.cuh"

namespace amica {
cudaError_t launch_estep_plain(const EStepArgs& a, int NP, int nclusters, cudaStream_t st);
cudaError_t launch_estep_tc(const EStepArgs& a, int NP, int nclusters, cudaStream_t st, int split, int shape);
}

using namespace amica;

namespace {

__device__ double psi_dev(double x) {
    const double coef[9] = {1.0 / 12.0, -1.0 / 120.0, 1.0 / 252.0, -1.0 / 240.0, 1.0 / 132.0,
                            -691.0 / 32760.0, 1.0 / 12.0, -3617.0 / 8160.0, 43867.0 / 14364.0};
    const double s = x + 6.0;
    double r = log(s) - 1.0 / (2.0 * s);
    const double s2 = s * s;
    double p = s2;
    for (int k = 0; k < 9; k++) { r -= coef[k] / p; p *= s2; }
    for (int k = 5; k >= 0; k--) r -= 1.0 / (x + k);
    return r;
}

__global__ void k_adjoint_reduce(const double* __restrict__ partial, double* __restrict__ raw,
                                 int nclusters, int M, int stride) {
    const int64_t total = (int64_t)M * stride;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total;
         e += (int64_t)gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int q = 0; q < nclusters; q++) s += partial[(size_t)q * total + e];
        raw[e] = s;
    }
}

// out: [0] sum P (relative), then dW (M n n, column-major), dmu, dbeta, drho (M m n)
__global__ void k_adjoint_finalize(const double* __restrict__ raw, const double* __restrict__ A,
                                   const double* __restrict__ c, const double* __restrict__ beta,
                                   const double* __restrict__ rho, double* __restrict__ out, int n,
                                   int m, int M, int psi_is_phi) {
    const int h = blockIdx.x;
    PartLayout PL{n, m};
    const double* R = raw + (size_t)h * PL.stride();
    const double vsum = R[1];
    if (h == 0 && threadIdx.x == 0) out[0] = R[0];
    double* dW = out + 1 + (size_t)h * n * n;
    const double* Ah = A + (size_t)h * n * n;
    const double* Psi = R + PL.psi();
    const double* gs = R + PL.gs();
    for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
        const int i = e % n, k = e / n;   // dW(i,k) stored at k*n + i
        // W^{-T}(i,k) = A(k,i); sum_t g (x - c)^T = Psi - gsum c^T = phi W^{-T} = phi A^T
        double gx;
        if (psi_is_phi) {
            gx = 0.0;
            for (int l = 0; l < n; l++) gx += Psi[(size_t)l * n + i] * Ah[(size_t)l * n + k];
        } else {
            gx = Psi[(size_t)k * n + i] - gs[i] * c[(size_t)h * n + k];
        }
        dW[e] = vsum * Ah[(size_t)i * n + k] - gx;
    }
    const size_t off_mu = 1 + (size_t)M * n * n;
    const size_t mnM = (size_t)M * m * n;
    for (int e = threadIdx.x; e < m * n; e += blockDim.x) {
        const size_t idx = (size_t)h * m * n + e;
        const double bt = beta[idx], r = rho[idx];
        const double us = R[PL.mix(kUs) + e];
        out[off_mu + idx] = sqrt(bt) * R[PL.mix(kMn) + e];
        out[off_mu + mnM + idx] = (us - R[PL.mix(kBd) + e]) / (2.0 * bt);
        out[off_mu + 2 * mnM + idx] = us * psi_dev(1.0 + 1.0 / r) / (r * r) - R[PL.mix(kRn) + e] / r;
    }
}

}  // namespace

namespace amica {

// The adjoint sweep: the fused E-step in gradient mode into `partial`.
cudaError_t launch_adjoint(const EStepArgs& a0, int NP, double* grad_partial, int nclusters,
                           cudaStream_t st, bool use_tc, int tc_shape) {
    EStepArgs a = a0;
    a.grad_mode = 1;
    a.update_rho = 1;
    a.partial = grad_partial;
    a.split_phi = nullptr;   // the gradient sweep does not need phi's split correction
    return use_tc ? launch_estep_tc(a, NP, nclusters, st, 0, tc_shape) : launch_estep_plain(a, NP, nclusters, st);
}

cudaError_t launch_adjoint_finalize(const double* grad_partial, double* raw, int nclusters, int n,
                                    int m, int M, const double* A, const double* c,
                                    const double* beta, const double* rho, double* out,
                                    int psi_is_phi, cudaStream_t st) {
    PartLayout PL{n, m};
    const int64_t total = (int64_t)M * PL.stride();
    int grid = (int)((total + 255) / 256);
    if (grid > 4096) grid = 4096;
    k_adjoint_reduce<<<grid, 256, 0, st>>>(grad_partial, raw, nclusters, M, PL.stride());
    k_adjoint_finalize<<<M, 256, 0, st>>>(raw, A, c, beta, rho, out, n, m, M, psi_is_phi);
    return cudaGetLastError();
}

}  // namespace amica
