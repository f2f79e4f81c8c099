"""A bounded device wait that runs out: the error comes back to the host and
the context stays usable.

The cooperative eigensolver of the GPU preprocessing (above 128 channels)
synchronises its blocks with grid barriers whose waits are bounded.  The test
hook amica_test_arm_wait_fault makes one block skip its first arrival and
bounds the waits of that one launch by a short limit (1e6 cycles, about half a
millisecond), so every other block's wait runs out: each records the timeout,
sets the launch's abort flag and returns.  Nothing is left waiting and no GPU
fault is involved; the next preprocessing of the same context runs normally and
the fit proceeds.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_missed_grid_barrier_arrival_times_out_and_context_recovers():
    from cudamica_b200 import synth
    from cudamica_b200.engine import Amica, AmicaError
    n, T, M, m = 144, 20_000, 1, 3
    x = synth.config1(seed=4, n=n, T=T).x
    A0, c0 = synth.norand_init(n, M)
    eng = Amica(n, T, M, m, precision=1)
    eng.load_data(x)
    eng.arm_wait_fault(1_000_000)
    with pytest.raises(AmicaError) as ei:
        eng.preprocess()
    assert ei.value.code == -24                     # AMICA_ERR_TIMEOUT
    # the hook armed one launch: the same context now preprocesses, initialises
    # and iterates normally
    eng.preprocess()
    S, means, ldetS = eng.sphere()
    ref = Amica(n, T, M, m, precision=1)
    ref.load_data(x)
    ref.preprocess()
    S2, _, ld2 = ref.sphere()
    assert np.max(np.abs(S - S2)) < 1e-12 and abs(ldetS - ld2) < 1e-10
    eng.init(A0, c0)
    outs = eng.run(3)
    assert all(np.isfinite(o.ll) for o in outs)
    ref.close()
    eng.close()


def test_hook_refused_where_there_is_no_grid_barrier():
    from cudamica_b200.engine import Amica, AmicaError
    eng = Amica(32, 10_000, 1, 3, precision=1)
    with pytest.raises(AmicaError) as ei:
        eng.arm_wait_fault(1_000_000)
    assert ei.value.code == -25
    eng.close()
