"""The float64 torch log-likelihood used to check the adjoint agrees with the
FP64 oracle's E-step at the same (non-default) parameters."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from cudamica_b200 import synth
from oracle import oracle as O
import torch_ll


def random_params(rng, M, m, n):
    alpha = rng.dirichlet([2.0] * m, size=(M, n)).transpose(0, 2, 1).copy()
    mu = rng.normal(0.0, 0.5, size=(M, m, n))
    beta = np.exp(rng.uniform(np.log(0.5), np.log(2.0), size=(M, m, n)))
    rho = rng.uniform(1.1, 2.4, size=(M, m, n))
    return alpha, mu, beta, rho


def test_torch_loglik_matches_oracle():
    rng = np.random.default_rng(5)
    n, T, M, m = 8, 4000, 2, 3
    d = synth.config2(seed=3, n=n, T=T, M=M, m=m, block_lo=300, block_hi=900)
    xs, means, S, ldetS = O.preprocess(d.x, 1)
    A0, c0 = synth.norand_init(n, M)
    orc = O.Oracle(xs, M, m, A0, c0, ldetS, nthreads=2)
    alpha, mu, beta, rho = random_params(rng, M, m, n)
    orc.alpha[...] = alpha
    orc.mu[...] = mu
    orc.beta[...] = beta
    orc.rho[...] = rho
    orc.gm[...] = np.array([0.4, 0.6])
    orc.prepare()
    ll_o = orc.estep()[0] / (n * T)
    p = orc.params()
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64))
    ll_t = torch_ll.loglik(t(xs), t(p["W"]), t(p["c"]), t(p["gm"]), t(alpha), t(mu), t(beta),
                           t(rho), ldetS).item()
    assert abs(ll_t - ll_o) < 1e-12
