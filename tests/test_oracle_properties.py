"""Properties of the EM iteration, checked on the FP64 oracle (CPU):
responsibilities sum to one, over models per sample and over mixtures per
(model, channel), and the log-likelihood does not decrease under natural-
gradient steps with a small learning rate."""
import numpy as np
import pytest

from cudamica_b200 import synth
from oracle import oracle as O

N, T = 16, 8000


@pytest.fixture(scope="module")
def data():
    d = synth.config2(seed=4, n=N, T=T, M=2, m=3, block_lo=500, block_hi=1500)
    return O.preprocess(d.x, 1)


def test_responsibilities_sum_to_one(data):
    xs, means, S, ldetS = data
    M, m = 2, 3
    A0, c0 = synth.norand_init(N, M)
    orc = O.Oracle(xs, M, m, A0, c0, ldetS, nthreads=4, keep_Lt=True)
    for _ in range(3):
        orc.step()
    orc.prepare()
    st = O.split_stats(orc.estep(), N, M, m)
    # models: sum_h v_h(t) = sum_h exp(Lt_h(t) - P(t)) = 1 for every sample
    v = np.exp(orc.Lt - orc.P[None, :])
    assert np.max(np.abs(v.sum(0) - 1.0)) < 1e-12
    # mixtures: sum_j u_hij(t) = v_h(t), so sum_j usum_hij = vsum_h for every channel
    us = np.asarray(st["us"]).reshape(M, m, N)
    vs = np.asarray(st["vs"]).reshape(M)
    assert np.max(np.abs(us.sum(1) / vs[:, None] - 1.0)) < 1e-12


@pytest.mark.parametrize("M", [1, 2])
def test_loglik_does_not_decrease_under_natural_gradient(data, M):
    xs, means, S, ldetS = data
    A0, c0 = synth.norand_init(N, M)
    orc = O.Oracle(xs, M, 3, A0, c0, ldetS, nthreads=4, do_newton=0, lrate0=0.05, lnatrate=0.05,
                   lratemax=0.05)
    lls = np.array([orc.step() for _ in range(30)])
    assert np.all(np.diff(lls) >= 0.0), np.diff(lls)
