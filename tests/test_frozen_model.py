"""A model that explains no data is frozen.

Two models, the second started from A = 0.01 I: its W = 100 I puts every
sample tens of thousands of nats below the first model, so its responsibilities
v_1(t) are 0 and vsum_1 = 0.  The reference's M-step would divide by vsum_1 and
usum_1 (src/amica.cu:1995-2154) and turn the model's parameters non-finite; the
oracle and the engine keep its A, c and mixture parameters and floor gm_1 at
1e-300, while the first model is fitted as usual.  The CPU test runs the
oracle; the GPU test runs both forms of the engine against it.
"""
import numpy as np
import pytest

from cudamica_b200 import synth
from oracle import oracle as O

N, T, M, MIX = 16, 4000, 2, 3


def tf32(a):
    """Round to TF32 (nearest, ties away), as the mixed forms store the data."""
    u = np.ascontiguousarray(a, dtype=np.float32).copy().view(np.uint32)
    u += np.uint32(0x1000)
    u &= np.uint32(0xFFFFE000)
    return u.view(np.float32).astype(np.float64)


def frozen_case():
    d = synth.config0(seed=5, n=N, T=T)
    xs, means, S, ldetS = O.preprocess(d.x, 1)
    A0, c0 = synth.norand_init(N, M)
    A0 = A0.reshape(M, N, N).copy()
    A0[1] = 0.01 * np.eye(N)
    return d.x, xs, means, S, ldetS, A0, c0.reshape(M, N)


def test_oracle_freezes_a_model_without_data():
    x, xs, means, S, ldetS, A0, c0 = frozen_case()
    orc = O.Oracle(xs, M, MIX, A0, c0, ldetS, nthreads=4)
    p0 = orc.params()
    lls = [orc.step() for _ in range(6)]
    p = orc.params()
    assert np.all(np.isfinite(lls)) and lls[-1] > lls[0]
    for k, v in p.items():
        assert np.all(np.isfinite(v)), k
    assert p["gm"][1] == 1e-300 and p["gm"][0] == 1.0
    for k in ("A", "c", "alpha", "mu", "beta", "rho"):
        assert np.array_equal(p[k][1], p0[k][1]), k
        assert not np.array_equal(p[k][0], p0[k][0]), k


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [0, 1])
def test_engine_freezes_a_model_without_data(precision):
    from cudamica_b200.engine import Amica
    x, xs, means, S, ldetS, A0, c0 = frozen_case()
    # the mixed form holds the data rounded to TF32: the oracle gets the same data
    orc = O.Oracle(tf32(xs) if precision else xs, M, MIX, A0, c0, ldetS, nthreads=4)
    eng = Amica(N, T, M, MIX, precision=precision)
    eng.set_sphered(xs, means, S, ldetS)
    eng.init(A0, c0)
    for it in range(1, 5):
        out = eng.step()
        ll = orc.step()
        assert abs(out.ll - ll) < 2e-6 * 5 ** (it - 1), (it, out.ll, ll)
    p = eng.params()
    for k in ("A", "c", "alpha", "mu", "beta", "rho", "gm"):
        assert np.all(np.isfinite(p[k])), k
    assert p["gm"][1] <= 1e-299
    assert np.array_equal(p["A"][1], A0[1])
    assert np.array_equal(p["c"][1], c0[1])
    eng.close()


def test_oracle_keeps_a_component_without_responsibility():
    """alpha = 0 for one mixture component of one model: its log-density is
    -inf, its responsibilities and usum are 0, and its mu, beta and rho get no
    update (mu and beta still follow the reparametrisation of their channel,
    the column scaling of A and the shift of c) while the other components
    and the model are updated; the reference's 0/0 would have made kappa,
    lambda and then A non-finite."""
    d = synth.config0(seed=6, n=N, T=T)
    xs, means, S, ldetS = O.preprocess(d.x, 1)
    A0, c0 = synth.norand_init(N, 1)
    # Newton from the first iteration, so that kappa and lambda enter the A update
    orc = O.Oracle(xs, 1, MIX, A0, c0, ldetS, nthreads=4, newt_start_iter=1)
    orc.alpha[0, 1, 3] = 0.0                  # shared with the oracle's state
    p0 = orc.params()
    lls = [orc.step() for _ in range(5)]
    p = orc.params()
    assert np.all(np.isfinite(lls)) and lls[-1] > lls[0]
    for k, v in p.items():
        assert np.all(np.isfinite(v)), k
    assert p["rho"][0, 1, 3] == p0["rho"][0, 1, 3]
    for k in ("mu", "beta", "rho"):
        assert p[k][0, 0, 3] != p0[k][0, 0, 3], k
    assert p["alpha"][0, 1, 3] == 0.0
    assert not np.array_equal(p["A"], p0["A"])
    assert orc.st.newton == 1                 # the Newton step ran
