"""Parity cases shared by the golden-fixture generator and the tests.

Each case regenerates its raw data from a seed (cudamica_b200.synth), spheres
it in float64 with numpy, and builds the deterministic initial state, so that
the reference binary, the FP64 oracle and the CUDA engine all start from the
same whitened data, A and c.
"""
from __future__ import annotations

import dataclasses
import hashlib
import numpy as np

from cudamica_b200 import synth


@dataclasses.dataclass(frozen=True)
class Case:
    name: str
    n: int
    T: int
    M: int
    m: int
    maxiter: int
    newt_start_iter: int
    update_rho: bool
    recipe: str
    seed: int
    keep_iters: tuple[int, ...]


CASES = {
    # the small plain-AMICA workload: n=32, T=60k, M=1, m=3, 100 iterations
    "c0": Case("c0", 32, 60_000, 1, 3, 100, 50, True, "config0", 0,
               (1, 2, 3, 5, 10, 20, 30, 50, 51, 52, 60, 75, 100)),
    # two models with distinct initial A: exercises the model-level
    # log-sum-exp, the model weights and the Newton phase
    "m2": Case("m2", 16, 20_000, 2, 2, 60, 20, True, "config2", 3,
               (1, 2, 5, 10, 20, 21, 22, 30, 45, 60)),
    # three models / three mixtures (models 1 and 2 share their initial state,
    # as in the reference's deterministic mode)
    "m3": Case("m3", 24, 30_000, 3, 3, 40, 15, True, "config2", 5,
               (1, 2, 5, 10, 15, 16, 20, 30, 40)),
}


def raw_data(case: Case) -> np.ndarray:
    if case.recipe == "config0":
        return synth.config0(seed=case.seed, n=case.n, T=case.T).x
    if case.recipe == "config2":
        return synth.config2(seed=case.seed, n=case.n, T=case.T, M=case.M, m=case.m,
                             block_lo=500, block_hi=2500).x
    raise ValueError(case.recipe)


def sphere_numpy(x: np.ndarray):
    """Centre and sphere in float64 the way the reference does
    (src/preprocess.cu:31-85 centring, :100-230 sphering with do_sphere=1):
    C = Xc Xc^T / T, S = 2 C^{-1/2}, ldetS = -log|det S|."""
    xd = x.astype(np.float64)
    means = xd.mean(axis=0)
    xc = xd - means[None, :]
    C = (xc.T @ xc) / xc.shape[0]
    d, V = np.linalg.eigh(C)
    S = (V * (2.0 / np.sqrt(d))[None, :]) @ V.T
    ldetS = -float(np.sum(np.log(2.0 / np.sqrt(d))))
    xs = xc @ S.T
    return np.ascontiguousarray(xs), means, S, ldetS


def digest(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()[:16]


def prepared(case: Case):
    x = raw_data(case)
    xs, means, S, ldetS = sphere_numpy(x)
    A0, c0 = synth.norand_init(case.n, case.M)
    return dict(x=x, xs=xs, means=means, sphere=S, ldetS=ldetS, A0=A0, c0=c0)


def ref_ltall_source(T: int, block_size: int, stride: int = 97, count: int | None = None):
    """Where the reference's ltallfile entries come from.

    The reference copies each block's Lt into its per-model ltall buffer at
    ``OFFSET1D(dev_ltall, start)`` (src/amica.cu:1203-1209), and OFFSET1D adds
    ``start`` BYTES, not elements (include/tools.h:140-141).  Block b therefore
    lands at element b * block_size / 8, the blocks overlap (later blocks win),
    and elements past (nblocks - 1) * block_size / 8 + block_size are never
    written (uninitialised memory in the file).  The goldens keep every
    ``stride``-th element of that file.

    Returns (positions in the strided golden that hold a real Lt value, the
    sample index t each of them holds)."""
    nb = T // block_size
    step = block_size // 8
    n_el = -(-T // stride) if count is None else count
    e = np.arange(n_el, dtype=np.int64) * stride
    valid = e < (nb - 1) * step + block_size
    blk = np.minimum(e // step, nb - 1)
    src = blk * block_size + e - blk * step
    return np.nonzero(valid)[0], src[valid]
