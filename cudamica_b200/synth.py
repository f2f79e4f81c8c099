"""Seeded synthetic EEG-like data for the AMICA EM workloads.

The reference publishes no dataset; these generators stand in for recordings
with the shapes and value distributions of the five workloads the engine is
measured on (independent sources mixed by random matrices, FP32 raw files in
the reference's ``datafile`` layout: T samples x n channels, sample-major,
raw float32, no header -- the layout read by ``loadMatrix``,
src/helpers.cu:513-553 of the reference).

Source recipes (all sources scaled to unit variance):
  * Laplacian;
  * generalized Gaussian with shape rho: |s|^rho ~ Gamma(1/rho, 1);
  * sub-Gaussian: uniform on [-sqrt(3), sqrt(3)];
  * bimodal: 0.5*N(-1.2, 0.4) + 0.5*N(+1.2, 0.4).
Mixing matrices are A = U diag(s) V^T with Haar-orthogonal U, V and singular
values log-spaced to a target condition number.  Sensor noise has variance
1e-3.
"""
from __future__ import annotations

import dataclasses
import numpy as np


def haar_orthogonal(rng: np.random.Generator, n: int) -> np.ndarray:
    q, r = np.linalg.qr(rng.standard_normal((n, n)))
    return q * np.sign(np.diag(r))[None, :]


def mixing_matrix(rng: np.random.Generator, n: int, cond: float) -> np.ndarray:
    u = haar_orthogonal(rng, n)
    v = haar_orthogonal(rng, n)
    s = np.logspace(0.0, -np.log10(cond), n)
    return (u * s[None, :]) @ v.T


def gg_samples(rng, rho: float, size) -> np.ndarray:
    g = rng.gamma(1.0 / rho, 1.0, size=size)
    s = np.power(g, 1.0 / rho) * rng.choice([-1.0, 1.0], size=size)
    return s


def unit(s: np.ndarray) -> np.ndarray:
    s = s - s.mean()
    return s / s.std()


def sources_basic(rng, T: int, kinds: list[tuple[str, float]]) -> np.ndarray:
    """kinds: list of (kind, rho) with kind in lap/gg/sub/bimodal."""
    out = np.empty((len(kinds), T), dtype=np.float64)
    for k, (kind, rho) in enumerate(kinds):
        if kind == "lap":
            s = rng.laplace(0.0, 1.0, T)
        elif kind == "gg":
            s = gg_samples(rng, rho, T)
        elif kind == "sub":
            s = rng.uniform(-np.sqrt(3.0), np.sqrt(3.0), T)
        elif kind == "bimodal":
            s = rng.normal(0.0, 0.4, T) + np.where(rng.random(T) < 0.5, -1.2, 1.2)
        else:
            raise ValueError(kind)
        out[k] = unit(s)
    return out


def source_kinds(rng, n_lap: int, n_gg: int, n_sub: int, rho_lo: float, rho_hi: float,
                 n_bimodal: int = 0) -> list[tuple[str, float]]:
    kinds = [("lap", 1.0)] * n_lap
    kinds += [("gg", float(r)) for r in rng.uniform(rho_lo, rho_hi, n_gg)]
    kinds += [("sub", 0.0)] * n_sub
    kinds += [("bimodal", 0.0)] * n_bimodal
    return kinds


def pink_noise(rng, T: int) -> np.ndarray:
    """1/f-coloured noise by spectral shaping of white noise."""
    w = rng.standard_normal(T)
    f = np.fft.rfft(w)
    freqs = np.arange(f.shape[0], dtype=np.float64)
    freqs[0] = 1.0
    f /= np.sqrt(freqs)
    return unit(np.fft.irfft(f, n=T))


def model_blocks(rng, T: int, M: int, lo: int, hi: int) -> np.ndarray:
    """Per-sample model index: contiguous blocks with lengths uniform in [lo, hi]."""
    labels = np.empty(T, dtype=np.int32)
    t = 0
    h = 0
    while t < T:
        ln = int(rng.integers(lo, hi + 1))
        labels[t:t + ln] = h
        t += ln
        h = (h + 1 + int(rng.integers(0, max(M - 1, 1)))) % M if M > 1 else 0
    return labels


def mixture_sources(rng, n: int, T: int, m: int, rho_lo: float, rho_hi: float):
    """Sources drawn from per-source generalized-Gaussian mixtures."""
    out = np.empty((n, T), dtype=np.float64)
    for i in range(n):
        alpha = rng.dirichlet([2.0] * m)
        mu = rng.normal(0.0, 0.5, m)
        beta = np.exp(rng.uniform(np.log(0.5), np.log(2.0), m))
        rho = rng.uniform(rho_lo, rho_hi, m)
        comp = rng.choice(m, size=T, p=alpha)
        s = np.empty(T)
        for j in range(m):
            sel = comp == j
            s[sel] = mu[j] + gg_samples(rng, rho[j], int(sel.sum())) / np.sqrt(beta[j])
        out[i] = unit(s)
    return out


@dataclasses.dataclass
class Dataset:
    x: np.ndarray          # T x n float32, sample-major (reference datafile layout)
    n: int
    T: int
    M: int
    m: int
    labels: np.ndarray | None = None
    outliers: np.ndarray | None = None


def finish(rng, xs: np.ndarray, noise_var: float = 1e-3) -> np.ndarray:
    xs = xs + rng.normal(0.0, np.sqrt(noise_var), xs.shape)
    return np.ascontiguousarray(xs.T.astype(np.float32))


def config0(seed: int = 0, n: int = 32, T: int = 60_000) -> Dataset:
    """Plain AMICA, small: 12 Laplacian, 12 GG rho~U[1.2,3], 8 uniform; cond 10."""
    rng = np.random.default_rng(seed)
    scale = n / 32.0
    n_lap, n_gg = int(round(12 * scale)), int(round(12 * scale))
    kinds = source_kinds(rng, n_lap, n_gg, n - n_lap - n_gg, 1.2, 3.0)
    s = sources_basic(rng, T, kinds)
    A = mixing_matrix(rng, n, 10.0)
    return Dataset(finish(rng, A @ s), n, T, 1, 3)


def config1(seed: int = 0, n: int = 64, T: int = 500_000, cond: float = 30.0,
            outlier_frac: float = 0.005) -> Dataset:
    """EEG-scale single model: 24 Lap, 28 GG, 12 uniform (scaled to n), 1/f
    common mode at 0.1x, 0.5% of samples as 20-sigma outlier bursts."""
    rng = np.random.default_rng(seed)
    n_lap = int(round(24 * n / 64))
    n_gg = int(round(28 * n / 64))
    kinds = source_kinds(rng, n_lap, n_gg, n - n_lap - n_gg, 1.2, 3.0)
    s = sources_basic(rng, T, kinds)
    A = mixing_matrix(rng, n, cond)
    xs = A @ s
    xs += 0.1 * pink_noise(rng, T)[None, :] * np.sqrt(np.mean(xs ** 2))
    out = np.zeros(T, dtype=bool)
    n_bad = int(outlier_frac * T)
    if n_bad:
        burst = 50
        starts = rng.choice(T // burst, size=max(n_bad // burst, 1), replace=False) * burst
        for st in starts:
            out[st:st + burst] = True
        sig = xs.std(axis=1, keepdims=True)
        xs[:, out] += 20.0 * sig * rng.choice([-1.0, 1.0], size=(n, int(out.sum())))
    return Dataset(finish(rng, xs), n, T, 1, 3, outliers=out)


def config2(seed: int = 0, n: int = 128, T: int = 1_000_000, M: int = 3, m: int = 3,
            block_lo: int = 500, block_hi: int = 2500, cond: float = 30.0,
            rho_lo: float = 1.0, rho_hi: float = 2.5) -> Dataset:
    """Multi-model AMICA: the generating model switches in contiguous blocks;
    each model has its own mixing matrix and per-source GG mixtures."""
    rng = np.random.default_rng(seed)
    labels = model_blocks(rng, T, M, block_lo, block_hi)
    xs = np.empty((n, T), dtype=np.float64)
    for h in range(M):
        sel = labels == h
        Th = int(sel.sum())
        s = mixture_sources(rng, n, Th, m, rho_lo, rho_hi)
        A = mixing_matrix(rng, n, cond)
        xs[:, sel] = A @ s
    return Dataset(finish(rng, xs), n, T, M, m, labels=labels)


def config4(seed: int = 0, n: int = 256, T: int = 2_000_000, M: int = 4, m: int = 5) -> Dataset:
    """Large multi-model: 40% Lap, 40% GG rho~U[1,3], 20% bimodal; cond 100."""
    rng = np.random.default_rng(seed)
    labels = model_blocks(rng, T, M, 1000, 5000)
    xs = np.empty((n, T), dtype=np.float64)
    for h in range(M):
        sel = labels == h
        Th = int(sel.sum())
        kinds = source_kinds(rng, int(0.4 * n), int(0.4 * n), 0, 1.0, 3.0,
                             n_bimodal=n - 2 * int(0.4 * n))
        s = sources_basic(rng, Th, kinds)
        A = mixing_matrix(rng, n, 100.0)
        xs[:, sel] = A @ s
    return Dataset(finish(rng, xs), n, T, M, m, labels=labels)


def cohort_subject(i: int, n: int, T: int) -> Dataset:
    """Cohort member i: config-1 recipe, seed 1000+i, cond ~ U[10, 50]."""
    rng = np.random.default_rng(1000 + i)
    cond = float(rng.uniform(10.0, 50.0))
    return config1(seed=1000 + i, n=n, T=T, cond=cond)


def cohort_shapes(num: int = 48, seed: int = 7) -> list[tuple[int, int]]:
    """(n, T) per subject: n from {32, 64, 128} (equal counts), T ~ U[1e5, 8e5]."""
    rng = np.random.default_rng(seed)
    ns = np.repeat([32, 64, 128], num // 3)
    rng.shuffle(ns)
    Ts = rng.integers(100_000, 800_001, num)
    return [(int(a), int(b)) for a, b in zip(ns, Ts)]


def norand_init(n: int, M: int, seed: int = 1234) -> tuple[np.ndarray, np.ndarray]:
    """Deterministic initial A (M x n x n, column-major per model) and c (M x n):
    A = I + 0.05*(U - 0.5) with unit-norm columns, c = 0.1*N(0, 1).  The
    reference's deterministic mode reads A/c for model 0 from one file pair and
    for every model > 0 from a second pair (src/amica.cu:314-322); models
    1..M-1 therefore share an initial state, and so do these arrays."""
    rng = np.random.default_rng(seed)
    A = np.empty((M, n, n), dtype=np.float64)
    c = np.empty((M, n), dtype=np.float64)
    for h in range(min(M, 2)):
        a = np.eye(n) + 0.05 * (rng.random((n, n)) - 0.5)
        a /= np.linalg.norm(a, axis=0, keepdims=True)
        A[h] = a.T  # store column-major: row k of A[h] is column k
        c[h] = 0.1 * rng.standard_normal(n)
    for h in range(2, M):
        A[h] = A[1]
        c[h] = c[1]
    # the files are float32: round the same way the reference does on load
    A = A.astype(np.float32).astype(np.float64)
    c = c.astype(np.float32).astype(np.float64)
    return A, c
