"""Float64 PyTorch restatement of the AMICA log-likelihood, the reference for
the engine's hand-written adjoint (test infrastructure only).

L = sum_t P(t) / (n T),  P(t) = log sum_h exp(Lt_h(t)),
Lt_h(t) = log gm_h + log|det W_h| + ldetS + sum_i log sum_j exp(Q_hij(t)),
Q = log alpha + 0.5 log beta - log 2 - lgamma(1 + 1/rho) - |sqrt(beta) (b - mu)|^rho,
b = W_h (x_t - c_h): the density of src/kernels.cu:282-307 and the
likelihood of src/kernels.cu:317-450.

W is passed in the engine's storage order (column-major per model, i.e. the
numpy array W[h][k][i] holds W_h(i, k)), so gradients line up entry by entry
with what amica_loglik_adjoint returns.
"""
import math

import torch


def loglik(x, W, c, gm, alpha, mu, beta, rho, ldetS):
    """x: (T, n); W: (M, n, n) storage order; c: (M, n); gm: (M,);
    alpha, mu, beta, rho: (M, m, n).  Returns the scalar LL per sample and channel."""
    T, n = x.shape
    Wm = W.transpose(1, 2)                                    # Wm[h][i][k] = W_h(i, k)
    xc = x[:, None, :] - c[None, :, :]                        # (T, M, n)
    b = torch.einsum("hik,thk->thi", Wm, xc)                  # (T, M, n)
    y = torch.sqrt(beta)[None] * (b[:, :, None, :] - mu[None])  # (T, M, m, n)
    Q = (torch.log(alpha) + 0.5 * torch.log(beta) - math.log(2.0)
         - torch.lgamma(1.0 + 1.0 / rho))[None] - torch.abs(y) ** rho[None]
    lse = torch.logsumexp(Q, dim=2)                           # (T, M, n)
    logdet = torch.linalg.slogdet(Wm)[1]                      # (M,)
    Lt = (torch.log(gm) + logdet + ldetS)[None, :] + lse.sum(-1)
    P = torch.logsumexp(Lt, dim=1)
    return P.sum() / (n * T)
