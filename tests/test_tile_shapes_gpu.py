"""The fused E-step's tile shapes (amica_cfg.tc_shape / amica_set_tile_shape):
0 = 3 density warpgroups, 48-sample tiles, 2 x stages; 1 = 2 warpgroups,
32-sample tiles, 2 stages; 2 = 2 warpgroups, 3 stages.

Every shape computes the same E-step: against the FP64 oracle on the data as
the mixed form stores it (TF32) at each lane packing (n = 32: R = 4; n = 64:
R = 2; n = 128: R = 1) and at m = 3 and m = 5 (whose log2|y| cache no longer
fits beside a 48-sample tile: the 3-warpgroup shape recomputes log2|y|, the
2-warpgroup shapes keep it), and against shape 0 itself (the same sums in a
different grouping: FP32-level differences).  The split correction of phi runs
in every shape, and the measuring autotuner picks one and leaves the context in
it.
"""
import numpy as np
import pytest

from oracle import oracle as O
from test_parity_headline_gpu import _as_stored, _errs

pytestmark = pytest.mark.gpu

CASES = [(32, 60_000, 1, 3), (64, 90_000, 2, 5), (128, 90_000, 3, 3), (128, 60_000, 2, 5)]


def _data(n, T, M, m, seed=7):
    from cudamica_b200 import synth
    from golden.cases import sphere_numpy
    x = synth.config2(seed=seed, n=n, T=T, M=M, m=m).x
    xs, means, S, ldetS = sphere_numpy(x)
    A0, c0 = synth.norand_init(n, M)
    return xs, means, S, ldetS, A0, c0


@pytest.mark.parametrize("n,T,M,m", CASES)
def test_every_tile_shape_matches_the_oracle_and_shape_0(n, T, M, m):
    from cudamica_b200.engine import Amica
    xs, means, S, ldetS, A0, c0 = _data(n, T, M, m)
    orc = O.Oracle(_as_stored(xs, 1), M, m, A0, c0, ldetS, nthreads=8)
    orc.prepare()
    s_orc = orc.estep()
    stats = {}
    for shape in (0, 1, 2):
        eng = Amica(n, T, M, m, precision=1, tc_shape=shape)
        assert eng.kernel == "tc_tf32"
        eng.set_sphered(xs, means, S, ldetS)
        eng.init(A0, c0)
        s = eng.estep_stats()
        stats[shape] = s
        dll = abs(s[0] - s_orc[0]) / (n * T)
        errs = _errs(s, s_orc, n, M, m)
        print(f"n={n} M={M} m={m} shape={shape}: dLL {dll:.2e} "
              + " ".join(f"{k}={v:.1e}" for k, v in errs.items()))
        assert dll < 2e-6, dll
        for k in ("vs", "cn", "s2", "us", "kn", "ln", "bd", "rn", "phi"):
            assert errs[k] < 2e-4, (shape, k, errs[k])
        assert errs["mn"] < 2e-5 and errs["md_med"] < 2e-3, errs
        eng.close()
    for shape in (1, 2):
        d = _errs(stats[shape], stats[0], n, M, m)
        assert abs(stats[shape][0] - stats[0][0]) / (n * T) < 1e-6
        for k in ("vs", "cn", "s2", "us", "kn", "ln", "bd", "rn", "phi"):
            assert d[k] < 1e-4, (shape, k, d[k])


def test_tile_shapes_along_a_fit_and_with_the_split_correction():
    """Five iterations in each shape (the first LL equal to 1e-7 nats, the EM
    map's amplification allowed after), and the split correction of phi
    (phi_split = 1) in each shape against shape 0's."""
    from cudamica_b200.engine import Amica
    n, T, M, m = 128, 90_000, 3, 3
    xs, means, S, ldetS, A0, c0 = _data(n, T, M, m, seed=11)
    lls = {}
    for shape in (0, 1, 2):
        eng = Amica(n, T, M, m, precision=1, tc_shape=shape, phi_split=1)
        eng.set_sphered(xs, means, S, ldetS)
        eng.init(A0, c0)
        outs = eng.run(5)
        assert all(o.phi_split == 1 for o in outs)
        lls[shape] = np.array([o.ll for o in outs])
        eng.close()
    for shape in (1, 2):
        d = np.abs(lls[shape] - lls[0])
        print(f"shape {shape}: LL differences from shape 0 over 5 iterations {d}")
        assert d[0] < 1e-7 and np.all(d < 1e-7 * 30.0 ** np.arange(5)), d


def test_autotuner_picks_a_measured_shape_and_keeps_it():
    from cudamica_b200 import autotune
    from cudamica_b200.engine import Amica
    n, T, M, m = 64, 200_000, 1, 3
    xs, means, S, ldetS, A0, c0 = _data(n, T, M, m, seed=3)
    eng = Amica(n, T, M, m, precision=1)
    eng.set_sphered(xs, means, S, ldetS)
    eng.init(A0, c0)
    s0 = eng.estep_stats()
    prof = autotune.tile_shape_profile(eng, reps=3)
    print("E-step ms per tile shape:", prof)
    assert set(prof) == {0, 1, 2} and all(v > 0 for v in prof.values())
    best = autotune.best_tile_shape(eng, reps=3)
    assert best in (0, 1, 2)
    s1 = eng.estep_stats()                 # the context now runs the chosen shape
    assert abs(s1[0] - s0[0]) / (n * T) < 1e-6
    eng.close()
    plain = Amica(n, T, M, m, precision=0)
    assert autotune.best_tile_shape(plain) == -1
    with pytest.raises(Exception):
        plain.set_tile_shape(1)
    plain.close()


def test_adjoint_in_every_tile_shape():
    """The gradient sweep runs the fused kernel in the context's tile shape:
    in every shape LL and gradients match float64 autograd of the likelihood on
    the data as the form stores it, within the mixed form's bands (dW and dmu
    are differences of nearly cancelling sums, so the shapes' different FP32
    summation orders move them by a few 1e-4 of their largest entries)."""
    import torch
    from cudamica_b200.engine import Amica
    from test_adjoint_config2_gpu import _as_stored as stored_adj, _rel, _torch_ref
    n, T, M, m = 64, 60_000, 2, 3
    xs, means, S, ldetS, A0, c0 = _data(n, T, M, m, seed=5)
    dev = torch.device("cuda:0")
    for shape in (0, 1, 2):
        eng = Amica(n, T, M, m, precision=1, tc_shape=shape, update_rho=1)
        eng.set_sphered(xs, means, S, ldetS)
        eng.init(A0, c0)
        eng.run(2)
        ll_g, g_g = eng.adjoint()
        ll_t, g_t, _, _ = _torch_ref(eng, stored_adj(xs, 1), ldetS, dev)
        errs = {k: _rel(g_g[k], g_t[k]) for k in ("W", "mu", "beta", "rho")}
        print(f"shape {shape}: dLL {abs(ll_g - ll_t):.2e} " + " ".join(f"{k}={v:.2e}" for k, v in errs.items()))
        assert abs(ll_g - ll_t) < 2e-6
        for k, v in errs.items():
            assert v < 5e-4, (shape, k, v)
        eng.close()
