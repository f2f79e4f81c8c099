"""The hand-written adjoint (amica_loglik_adjoint) against a float64 torch
likelihood (itself pinned to the FP64 oracle in test_torch_ll_cpu.py): its
autograd gradient, and central finite differences (step 1e-4, FP64) on 256
random coordinates of W, mu, beta and rho; and the adjoint through the
torch.autograd.Function wrapper.

Both forms compute the likelihood sweep in FP32 (the mixed form with TF32
contractions), so the tolerances are relative to the largest entry of each
gradient: 2e-4 for the plain form, 2e-3 for the mixed form; the likelihood
itself to 1e-6 / 1e-5 nats per sample and channel.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from cudamica_b200 import synth
from oracle import oracle as O
import torch_ll

pytestmark = pytest.mark.gpu

TOL = {0: (1e-6, 2e-4), 1: (1e-5, 2e-3)}


def setup_engine(precision, n=16, T=20000, M=2, m=3, steps=3):
    from cudamica_b200.engine import Amica
    d = synth.config2(seed=7, n=n, T=T, M=M, m=m, block_lo=500, block_hi=1500)
    xs, means, S, ldetS = O.preprocess(d.x, 1)
    A0, c0 = synth.norand_init(n, M)
    eng = Amica(n, T, M, m, precision=precision, update_rho=1)
    eng.set_sphered(xs, means, S, ldetS)
    eng.init(A0, c0)
    eng.run(steps)                      # move away from the symmetric start
    return eng, xs, ldetS


def torch_reference(eng, xs, ldetS):
    p = eng.params()
    t = lambda a, g=False: torch.tensor(np.ascontiguousarray(a, dtype=np.float64), requires_grad=g)
    W, mu, beta, rho = t(p["W"], True), t(p["mu"], True), t(p["beta"], True), t(p["rho"], True)
    args = dict(x=t(xs), c=t(p["c"]), gm=t(p["gm"]), alpha=t(p["alpha"]), ldetS=ldetS)
    f = lambda W_, mu_, beta_, rho_: torch_ll.loglik(W=W_, mu=mu_, beta=beta_, rho=rho_, **args)
    L = f(W, mu, beta, rho)
    L.backward()
    grads = dict(W=W.grad.numpy(), mu=mu.grad.numpy(), beta=beta.grad.numpy(), rho=rho.grad.numpy())
    base = dict(W=p["W"], mu=p["mu"], beta=p["beta"], rho=p["rho"])
    return L.item(), grads, f, base


def rel_err(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


@pytest.mark.parametrize("precision", [0, 1])
def test_adjoint_matches_float64_autograd(precision):
    eng, xs, ldetS = setup_engine(precision)
    ll_g, g_g = eng.adjoint()
    ll_t, g_t, _, _ = torch_reference(eng, xs, ldetS)
    tol_ll, tol_g = TOL[precision]
    assert abs(ll_g - ll_t) < tol_ll, (ll_g, ll_t)
    for k in ("W", "mu", "beta", "rho"):
        assert rel_err(g_g[k], g_t[k]) < tol_g, (k, rel_err(g_g[k], g_t[k]))
    eng.close()


def test_adjoint_matches_central_differences():
    eng, xs, ldetS = setup_engine(0)
    _, g_g = eng.adjoint()
    _, g_t, f, base = torch_reference(eng, xs, ldetS)
    rng = np.random.default_rng(11)
    keys = ("W", "mu", "beta", "rho")
    sizes = [base[k].size for k in keys]
    picks = rng.integers(0, sum(sizes), size=256)
    h = 1e-4
    fd, ad, tg = [], [], []
    with torch.no_grad():
        for flat in picks:
            ki = int(np.searchsorted(np.cumsum(sizes), flat, side="right"))
            k = keys[ki]
            idx = np.unravel_index(int(flat - (sum(sizes[:ki]))), base[k].shape)
            vals = {kk: torch.tensor(base[kk]) for kk in keys}
            vals[k][idx] += h
            lp = f(vals["W"], vals["mu"], vals["beta"], vals["rho"]).item()
            vals[k][idx] -= 2 * h
            lm = f(vals["W"], vals["mu"], vals["beta"], vals["rho"]).item()
            fd.append((lp - lm) / (2 * h))
            ad.append(g_g[k][idx])
            tg.append(g_t[k][idx])
    fd, ad, tg = map(np.array, (fd, ad, tg))
    scale = np.max(np.abs(fd))
    # The central difference itself carries the truncation error h^2 f'''/6
    # (about 1e-5 of the gradient's scale here), and |y|^rho has unbounded
    # curvature at y = 0 for rho < 2, which puts up to ~1e-3 on coordinates
    # that move samples across y = 0.  The adjoint must agree with the
    # differences as well as the exact float64 gradient does.
    assert np.max(np.abs(tg - fd)) / scale < 1e-3        # the reference itself
    assert np.max(np.abs(ad - fd)) / scale < 1e-3        # the hand-written adjoint
    assert np.median(np.abs(tg - fd)) / scale < 5e-5
    assert np.median(np.abs(ad - fd)) / scale < 5e-5
    eng.close()


def test_autograd_function_wrapper():
    from cudamica_b200.torch_adjoint import AmicaLogLik
    eng, xs, ldetS = setup_engine(0)
    p = eng.params()
    t = lambda a: torch.tensor(np.ascontiguousarray(a, dtype=np.float64), requires_grad=True)
    W, mu, beta, rho = t(p["W"]), t(p["mu"]), t(p["beta"]), t(p["rho"])
    L = AmicaLogLik.apply(W, mu, beta, rho, eng)
    L.backward()
    ll_t, g_t, _, _ = torch_reference(eng, xs, ldetS)
    assert abs(L.item() - ll_t) < 1e-6
    for k, v in (("W", W), ("mu", mu), ("beta", beta), ("rho", rho)):
        assert rel_err(v.grad.numpy(), g_t[k]) < 2e-4, k
    eng.close()
