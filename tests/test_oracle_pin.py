"""Pins the FP64 oracle against the reference's own CUDA build.

The golden fixtures tests/golden/ref_{c0,m2,m3}.npz were produced by
tests/golden/make_ref_goldens.py running fraimondo/cudamica's sources (built for
sm_100a by oracle/Makefile) in its deterministic mode on a B200.

Two FP64 implementations that sum in different orders agree to ~1e-15 after
one iteration and then drift apart geometrically (x10..x100 per iteration in
the multi-model cases): the mixture updates amplify rounding noise.  So the
trajectory is pinned tightly over its first iterations, the full c0 LL
trajectory within 1e-5 nats, and mid-trajectory behaviour (Newton phase
included) by one-step checks that restart from the reference's own dumped
state.
"""
import numpy as np
import pytest

from golden.cases import CASES, prepared, digest, ref_ltall_source
from oracle import oracle as O


def load(name):
    return np.load(f"{pytest.golden_dir}/ref_{name}.npz")


@pytest.fixture(scope="module")
def prep_cache():
    return {name: prepared(CASES[name]) for name in CASES}


def make_oracle(case, p, ref, **over):
    return O.Oracle(p["xs"], case.M, case.m, p["A0"], p["c0"], float(ref["ldetS"][0]),
                    nthreads=8, newt_start_iter=case.newt_start_iter,
                    update_rho=int(case.update_rho), **over)


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.mark.parametrize("name", ["c0", "m2", "m3"])
def test_inputs_and_sphere_match_reference(name, prep_cache):
    ref = load(name)
    p = prep_cache[name]
    assert digest(p["xs"][:1000]) == str(ref["xs_digest"])
    # the reference's own sphering of the same raw file (src/preprocess.cu:110-282)
    assert np.max(np.abs(ref["sphere"] - p["sphere"])) < 1e-11
    assert abs(float(ref["ldetS"][0]) - p["ldetS"]) < 1e-11


def test_oracle_preprocess_matches_numpy(prep_cache):
    p = prep_cache["c0"]
    xs, means, S, ld = O.preprocess(p["x"], 1)
    assert np.max(np.abs(S - p["sphere"])) < 1e-10
    assert abs(ld - p["ldetS"]) < 1e-10
    assert np.max(np.abs(xs - p["xs"])) < 1e-9
    assert np.max(np.abs(means - p["means"])) < 1e-12


@pytest.mark.parametrize("name,iters", [("c0", 10), ("m2", 5), ("m3", 4)])
def test_first_iterations_match_reference(name, iters, prep_cache):
    case, ref, p = CASES[name], load(name), prep_cache[name]
    orc = make_oracle(case, p, ref)
    keep = list(ref["keep_iters"])
    for it in range(1, iters + 1):
        orc.step()
        dll = abs(orc.ll_hist[-1] - ref["ll"][it - 1])
        assert dll < (1e-12 if it <= 2 else 1e-6), (it, dll)
        assert abs(orc.lrate_hist[-1] - ref["lrate"][it - 1]) < 1e-15
        if it in keep:
            a = keep.index(it)
            tol = 1e-9 if it == 1 else (1e-5 if it == 2 else 1e-2)
            for key in ("A", "alpha", "beta", "rho"):
                assert rel(getattr(orc, key), ref["iter_" + key][a]) < tol, (it, key)
            assert rel(orc.mu, ref["iter_mu"][a]) < (1e-8 if it == 1 else 1e-2), it
            assert np.max(np.abs(orc.c - ref["iter_c"][a])) < (1e-12 if it == 1 else (1e-8 if it == 2 else 1e-4))


def test_full_c0_trajectory_ll(prep_cache):
    case, ref, p = CASES["c0"], load("c0"), prep_cache["c0"]
    orc = make_oracle(case, p, ref)
    for _ in range(case.maxiter):
        orc.step()
    d = np.abs(np.array(orc.ll_hist) - ref["ll"])
    assert d.max() < 1e-5
    np.testing.assert_allclose(orc.lrate_hist, ref["lrate"], rtol=0, atol=1e-15)
    # Two FP64 implementations after 100 iterations of a chaotic map: the final
    # W (the reference's weightsfile) and mixture parameters agree to this band
    # only (W 1.4e-3, alpha/rho 4e-3, mu 5.8e-3, beta 8.3e-3 of the largest
    # entry), which bounds what any other arithmetic can be asked to match.
    prm = orc.params()
    band = {"W": 2e-3, "alpha": 6e-3, "rho": 6e-3, "mu": 8e-3, "beta": 1.2e-2}
    for k, tol in band.items():
        assert np.max(np.abs(prm[k] - ref[k])) / np.max(np.abs(ref[k])) < tol, k


@pytest.mark.parametrize("k", [1, 2, 50, 51, 75])
def test_one_step_from_reference_state(k, prep_cache):
    """Restart the oracle from the reference's dumped state after iteration k
    (c0, M=1 so gm stays 1) and compare with its dump after k+1."""
    case, ref, p = CASES["c0"], load("c0"), prep_cache["c0"]
    keep = list(ref["keep_iters"])
    if k + 1 not in keep:
        pytest.skip("no dump")
    a, b = keep.index(k), keep.index(k + 1)
    orc = make_oracle(case, p, ref)
    for key in ("A", "c", "alpha", "mu", "beta", "rho"):
        getattr(orc, key)[...] = ref["iter_" + key][a]
    orc.st.iter = k
    orc.st.lrate = float(ref["lrate"][k])          # lrate printed at iteration k+1
    orc.st.ll_prev = float(ref["ll"][k - 1])
    orc.step()
    assert abs(orc.ll_hist[-1] - ref["ll"][k]) < 1e-11
    for key in ("A", "alpha", "beta", "rho"):
        assert rel(getattr(orc, key), ref["iter_" + key][b]) < 1e-8, key
    assert rel(orc.mu, ref["iter_mu"][b]) < 1e-6


@pytest.mark.parametrize("name", ["c0", "m2", "m3"])
def test_final_lt_matches_reference_ltall(name, prep_cache):
    """The reference's ltallfile (its Lt_h(t) of the last iteration,
    src/amica.cu:1203-1209) against the oracle's Lt at the state entering the
    last iteration, through the byte-offset placement of that file
    (ref_ltall_source).  After maxiter - 1 steps of a chaotic map the two FP64
    trajectories differ by ~1e-4 nats per channel and sample, so that is the
    band.  With several models the Lt of a model that carries
    almost no weight at a sample is the most sensitive quantity of the fit, so
    m2/m3 get a wider band (measured: c0 6e-4 max / 1.1e-4 median; m2 4.6e-2 /
    1.3e-3; m3 1.2e-2 / 6.9e-4, against a spread of Lt/n of 0.14, 5.1, 2.5)."""
    case, ref, p = CASES[name], load(name), prep_cache[name]
    band_max, band_med = (2e-3, 3e-4) if case.M == 1 else (0.1, 3e-3)
    orc = make_oracle(case, p, ref, keep_Lt=True)
    for _ in range(case.maxiter - 1):
        orc.step()
    orc.prepare()
    s = orc.estep()
    assert abs(s[0] / (case.n * case.T) - ref["ll"][-1]) < 3e-4
    golden = ref["ltall_stride"]
    pos, src = ref_ltall_source(case.T, 5000, 97, golden.shape[1])
    assert len(pos) > 60
    d = np.abs(orc.Lt[:, src] - golden[:, pos]) / case.n
    assert d.max() < band_max, d.max()
    assert np.median(d) < band_med, np.median(d)
    # positions the reference never wrote hold no Lt value (its own bug)
    assert np.all(golden[:, pos] < -1.0)


def test_psi_against_scipy():
    sp = pytest.importorskip("scipy.special")
    xs = np.linspace(1.2, 2.2, 11)
    got = np.array([O.psi(x) for x in xs])
    np.testing.assert_allclose(got, sp.digamma(xs), rtol=0, atol=1e-13)


def test_jacobi_eig():
    rng = np.random.default_rng(3)
    a = rng.standard_normal((40, 40))
    C = a @ a.T
    ev, V = O.jacobi_eig(C)
    ev_np = np.linalg.eigvalsh(C)
    np.testing.assert_allclose(ev, ev_np, rtol=1e-11)
    np.testing.assert_allclose(V @ np.diag(ev) @ V.T, C, atol=1e-9)


def test_reject_rule_small():
    P = np.array([0.0, 1.0, 2.0, 3.0, 4.0, -50.0, 2.0, 1.0])
    keep = np.ones_like(P, dtype=np.uint8)
    keep[7] = 0
    k2, dropped, mean, sd = O.reject(P, keep, 1.0)
    kept = P[keep.astype(bool)]
    assert mean == pytest.approx(kept.mean())
    assert sd == pytest.approx(kept.std(ddof=1))
    assert dropped == 1 and k2[5] == 0 and k2[7] == 0 and k2.sum() == 6
