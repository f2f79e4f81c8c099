"""Sample rejection is integer work and must be bit-exact: the GPU mask after a
rejection pass equals the oracle's rule (src: engine-defined; FP64 mean and
n-1 std of P over kept samples, 4096-sample chunks summed in order) applied to
the same P vector and the same previous mask."""
import numpy as np
import pytest

from cudamica_b200 import synth
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def make(precision, **cfg):
    from cudamica_b200.engine import Amica
    n, T = 16, 60000
    d = synth.config1(seed=4, n=n, T=T)
    xs, means, S, ldetS = O.preprocess(d.x, 1)
    A0, c0 = synth.norand_init(n, 1)
    eng = Amica(n, T, 1, 3, precision=precision, **cfg)
    eng.set_sphered(xs, means, S, ldetS)
    eng.init(A0, c0)
    return eng, d


@pytest.mark.parametrize("precision", [0, 1])
def test_reject_now_is_bit_exact(precision):
    eng, d = make(precision, rejsig=3.0)
    eng.run(2)
    for _ in range(3):
        P = eng.p_relative().astype(np.float64)
        keep0 = eng.loglik()[2].copy()
        dropped = eng.reject_now()
        keep1 = eng.loglik()[2]
        k_o, d_o, _, _ = O.reject(P, keep0, 3.0)
        assert dropped == d_o
        assert np.array_equal(keep1, k_o)
        eng.step()
    # the 20-sigma bursts are the samples that went first
    rejected = eng.loglik()[2] == 0
    assert rejected[d.outliers].mean() > 0.9
    eng.close()


def test_scheduled_rejection_is_bit_exact():
    eng, d = make(1, do_reject=1, rejstart=2, rejint=2, maxrej=3, rejsig=3.0)
    keep_prev = np.ones(eng.T, dtype=np.uint8)
    passes = 0
    for it in range(1, 9):
        out = eng.step()
        P = eng.p_relative().astype(np.float64)
        keep = eng.loglik()[2].copy()
        due = it >= 2 and (it - 2) % 2 == 0 and passes < 3
        if due:
            k_o, d_o, _, _ = O.reject(P, keep_prev, 3.0)
            assert np.array_equal(keep, k_o), it
            assert out.nrejected == d_o
            passes += 1
        else:
            assert np.array_equal(keep, keep_prev), it
        keep_prev = keep
    assert passes == 3
    eng.close()


def test_rejection_bit_exact_at_full_size():
    # the single-model EEG-scale workload: n = 64, T = 500,000, 0.5% of the
    # samples in 20-sigma bursts, rejection every 10 iterations at 3 sigma
    from cudamica_b200.engine import Amica
    d = synth.config1(seed=0, n=64, T=500_000)
    A0, c0 = synth.norand_init(64, 1)
    for precision in (1, 0):
        eng = Amica(64, 500_000, 1, 3, precision=precision, do_reject=1, rejstart=10, rejint=10,
                    maxrej=3, rejsig=3.0)
        eng.load_data(d.x.astype(np.float32))
        eng.preprocess()
        eng.init(A0, c0)
        eng.run(9)
        keep_prev = eng.loglik()[2].copy()
        out = eng.step()                                  # iteration 10: a rejection pass
        P = eng.p_relative().astype(np.float64)
        keep = eng.loglik()[2]
        k_o, d_o, _, _ = O.reject(P, keep_prev, 3.0)
        assert np.array_equal(keep, k_o)
        assert out.nrejected == d_o > 0
        assert (keep == 0)[d.outliers].mean() > 0.95
        eng.close()
