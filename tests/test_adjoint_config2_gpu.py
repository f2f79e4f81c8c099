"""The hand-written adjoint at the multi-model configuration: n = 128
channels, M = 3 models, m = 3 mixtures, on a 20,000-sample slice of the
model-switching data, in both forms (the mixed form at n = 128 is the
tensor-core kernel the bench times), and the split mixed form at n = 160.

Checks, as for the small case in test_adjoint_gpu.py:
  * against the float64 autograd gradient of the torch likelihood
    (tests/torch_ll.py, pinned to the FP64 oracle on the CPU);
  * against central differences of that float64 likelihood (step 1e-4) on
    256 random coordinates of W, mu, beta and rho.
The float64 torch likelihood runs on the GPU here (512 evaluations on 20,000
samples x 128 channels x 9 mixture terms); torch is only the reference.

The mixed form stores the sphered data rounded to TF32, which moves the mu
and W gradients by ~2e-3 of their largest entries (the same data effect that
moves the mu sums, test_parity_headline_gpu.py); its gradient is therefore
checked against the reference on the data as it stores it, and its distance
from the exact-data gradient is printed.  Bands, relative to the largest entry
of each gradient: 2e-4 (plain; measured 2.6e-5) and 5e-4 (mixed; measured
7.9e-5: dW and dmu are differences of nearly cancelling terms, vsum W^-T -
phi A^T and sqrt(beta) sum u f', so phi's FP32-level error shows there
amplified); finite differences: the median gap within 1e-4 / 2e-4 of the
gradient's scale and the largest within the float64 gradient's own largest
gap plus the gradient band (the differences carry their own truncation error,
largest on coordinates that move samples across the kink of |y|^rho at y = 0).
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from cudamica_b200 import synth
from golden.cases import sphere_numpy
import torch_ll

pytestmark = pytest.mark.gpu

TOL = {0: dict(ll=1e-6, g=2e-4, fd_med=1e-4),
       1: dict(ll=2e-6, g=5e-4, fd_med=2e-4)}


def _as_stored(xs, precision):
    """The sphered data as the form holds it: FP32, or FP32 rounded to TF32
    (to nearest, ties away from zero) for the mixed form."""
    a = np.ascontiguousarray(xs, dtype=np.float32).copy()
    if precision:
        u = a.view(np.uint32)
        u += np.uint32(0x1000)
        u &= np.uint32(0xFFFFE000)
    return a.astype(np.float64)


def _slice(n, M, T=20_000, full_T=1_000_000, seed=0):
    d = synth.config2(seed=seed, n=n, T=full_T, M=M, m=3)
    return sphere_numpy(np.ascontiguousarray(d.x[:T]))


@pytest.fixture(scope="module")
def c2_slice():
    return _slice(128, 3)


def _engine(xs, means, S, ldetS, n, M, precision, steps=3):
    from cudamica_b200.engine import Amica
    T = xs.shape[0]
    A0, c0 = synth.norand_init(n, M)
    eng = Amica(n, T, M, 3, precision=precision, update_rho=1)
    eng.set_sphered(xs, means, S, ldetS)
    eng.init(A0, c0)
    eng.run(steps)                      # away from the deterministic start
    return eng


def _torch_ref(eng, xs, ldetS, dev):
    p = eng.params()
    t = lambda a, g=False: torch.tensor(np.ascontiguousarray(a, dtype=np.float64), device=dev,
                                        requires_grad=g)
    W, mu, beta, rho = t(p["W"], True), t(p["mu"], True), t(p["beta"], True), t(p["rho"], True)
    args = dict(x=t(xs), c=t(p["c"]), gm=t(p["gm"]), alpha=t(p["alpha"]), ldetS=ldetS)
    f = lambda W_, mu_, beta_, rho_: torch_ll.loglik(W=W_, mu=mu_, beta=beta_, rho=rho_, **args)
    L = f(W, mu, beta, rho)
    L.backward()
    grads = {k: v.grad.cpu().numpy() for k, v in (("W", W), ("mu", mu), ("beta", beta), ("rho", rho))}
    base = {k: torch.tensor(np.ascontiguousarray(p[k], dtype=np.float64), device=dev)
            for k in ("W", "mu", "beta", "rho")}
    return L.item(), grads, f, base


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


@pytest.mark.parametrize("precision", [0, 1])
def test_adjoint_vs_float64_autograd_and_differences(precision, c2_slice):
    xs, means, S, ldetS = c2_slice
    eng = _engine(xs, means, S, ldetS, 128, 3, precision)
    assert eng.kernel == ("tc_tf32" if precision else "plain_fp32")
    dev = torch.device("cuda:0")
    ll_g, g_g = eng.adjoint()
    ll_t, g_t, f, base = _torch_ref(eng, _as_stored(xs, precision), ldetS, dev)
    tol = TOL[precision]
    errs = {k: _rel(g_g[k], g_t[k]) for k in ("W", "mu", "beta", "rho")}
    print(f"precision={precision}: dLL {abs(ll_g - ll_t):.2e} gradient errors "
          + " ".join(f"{k}={v:.2e}" for k, v in errs.items()))
    if precision:
        _, g_x, _, _ = _torch_ref(eng, xs, ldetS, dev)
        print("  against the exact-data gradient: "
              + " ".join(f"{k}={_rel(g_g[k], g_x[k]):.2e}" for k in ("W", "mu", "beta", "rho")))
    assert abs(ll_g - ll_t) < tol["ll"]
    for k, v in errs.items():
        assert v < tol["g"], (k, v)
    # central differences of the float64 likelihood on 256 random coordinates
    rng = np.random.default_rng(2026)
    keys = ("W", "mu", "beta", "rho")
    sizes = [base[k].numel() for k in keys]
    picks = rng.integers(0, sum(sizes), size=256)
    h = 1e-4
    fd, ad, tg = [], [], []
    with torch.no_grad():
        for flat in picks:
            ki = int(np.searchsorted(np.cumsum(sizes), flat, side="right"))
            k = keys[ki]
            idx = np.unravel_index(int(flat - sum(sizes[:ki])), tuple(base[k].shape))
            vals = {kk: base[kk].clone() for kk in keys}
            vals[k][idx] += h
            lp = f(vals["W"], vals["mu"], vals["beta"], vals["rho"]).item()
            vals[k][idx] -= 2 * h
            lm = f(vals["W"], vals["mu"], vals["beta"], vals["rho"]).item()
            fd.append((lp - lm) / (2 * h))
            ad.append(g_g[k][idx])
            tg.append(g_t[k][idx])
    fd, ad, tg = map(np.array, (fd, ad, tg))
    scale = np.max(np.abs(fd))
    gap_t, gap_a = np.abs(tg - fd) / scale, np.abs(ad - fd) / scale
    print(f"precision={precision}: differences vs float64 gradient max {gap_t.max():.2e} "
          f"median {np.median(gap_t):.2e}; vs adjoint max {gap_a.max():.2e} median {np.median(gap_a):.2e}")
    # the float64 gradient itself: the differences carry their own truncation
    # error, largest on coordinates that move samples across the kink of
    # |y|^rho at y = 0 (up to 1.5e-3 of the scale at some parameter points)
    assert np.median(gap_t) < 1e-4 and gap_t.max() < 2e-3
    # the adjoint: as close to the differences as the float64 gradient, up to
    # its own gradient band
    assert np.median(gap_a) < tol["fd_med"] and gap_a.max() < gap_t.max() + tol["g"]
    eng.close()


def test_split_form_adjoint_above_128_channels():
    """n = 160, M = 2: the mixed form above 128 channels (TF32 tensor-core
    contractions around a density-only kernel) computes its gradient with the
    plain gradient kernel on its own grid, on the same buffers as its own E-step
    (which runs just before).  That gradient must equal, bit for bit, the one a
    plain-form context computes at the same parameters on the same stored data,
    and match float64 autograd there.  After three iterations from the
    deterministic start the W and mu gradients are small (max |dW| ~3e-4, max
    |dmu| ~5e-5 here), so their error relative to the largest entry is larger
    than at n = 128: the band is 2e-3."""
    from cudamica_b200.engine import Amica
    xs, means, S, ldetS = _slice(160, 2, T=20_000, full_T=200_000, seed=3)
    eng = _engine(xs, means, S, ldetS, 160, 2, 1)
    assert eng.kernel == "split_tf32"
    p = eng.params()
    eng.estep_stats()                   # the split form's own E-step ran last
    ll_g, g_g = eng.adjoint()
    stored = _as_stored(xs, 1)
    ll_t, g_t, _, _ = _torch_ref(eng, stored, ldetS, torch.device("cuda:0"))
    errs = {k: _rel(g_g[k], g_t[k]) for k in ("W", "mu", "beta", "rho")}
    print(f"split form n=160: dLL {abs(ll_g - ll_t):.2e} " + " ".join(f"{k}={v:.2e}" for k, v in errs.items()))
    assert abs(ll_g - ll_t) < 2e-6
    for k, v in errs.items():
        assert v < 2e-3, (k, v)
    e0 = Amica(160, xs.shape[0], 2, 3, precision=0, update_rho=1)
    e0.set_sphered(stored, means, S, ldetS)
    e0.init(*synth.norand_init(160, 2))
    e0.set_params(**{k: p[k] for k in ("A", "c", "gm", "alpha", "mu", "beta", "rho")})
    ll0, g0 = e0.adjoint()
    assert ll0 == ll_g
    for k in g0:
        assert np.array_equal(g0[k], g_g[k]), k
    e0.close()
    eng.close()
