"""The allocation-free E-step entry point (amica_estep_stats_noalloc) against
the context-based one (amica_estep_stats) and against the FP64 oracle.

Callers that cannot allocate device memory -- code inside another framework's
memory pool, or a process that forbids cudaMalloc after start-up -- hand in
their own device buffers and get the same sufficient statistics back; the
library's fixed scratch array holds everything in between.  Both paths run the
same plain FP32 E-step kernel, only on grids of different sizes (the
allocation-free one shrinks its grid until its partial sums fit the array), so
the sums agree to FP32 summation-order noise (relative 2e-5, the tolerance the
plain path's tests use), and both sit within the plain form's bands of the
oracle.  The call is made twice in a row: the second call reuses the scratch
array the first one left behind and must give the same bits.

Shapes: the small golden cases (n <= 32), n = 64 (M = 1), n = 128 with four
models (the grid shrinks to fit) and n = 256 (channel blocks, one cluster).

This file is collected last on purpose.
"""
import numpy as np
import pytest

from golden.cases import CASES, prepared, sphere_numpy
from oracle import oracle as O

pytestmark = pytest.mark.gpu

KEYS = ("vs", "cn", "s2", "phi", "us", "kn", "ln", "mn", "bd", "rn")


def _case_data(name):
    from cudamica_b200 import synth
    if name in CASES:
        case = CASES[name]
        p = prepared(case)
        return case.n, case.T, case.M, case.m, p["xs"], p["means"], p["sphere"], p["ldetS"], \
            p["A0"], p["c0"]
    n, T, M, m = {"n64": (64, 40_000, 1, 3), "n128m4": (128, 30_000, 4, 3),
                  "n256": (256, 20_000, 1, 3)}[name]
    if M == 1:
        x = synth.config1(seed=2, n=n, T=T).x
    else:
        x = synth.config2(seed=2, n=n, T=T, M=M, m=m).x
    xs, means, S, ldetS = sphere_numpy(x)
    A0, c0 = synth.norand_init(n, M)
    return n, T, M, m, xs, means, S, ldetS, A0, c0


def _errors(got, ref, n, M, m):
    a, b = O.split_stats(got, n, M, m), O.split_stats(ref, n, M, m)
    vsum = float(np.max(b["vs"]))
    out = {}
    for k in KEYS + ("md",):
        scale = max(np.max(np.abs(b[k])), vsum if k == "cn" else 0.0)
        out[k] = float(np.max(np.abs(a[k] - b[k])) / scale)
    return out


@pytest.mark.parametrize("name", ["c0", "m3", "n64", "n128m4", "n256"])
def test_noalloc_matches_context_entry_point_and_oracle(name):
    import torch
    from cudamica_b200 import engine as E

    n, T, M, m, xs, means, S, ldetS, A0, c0 = _case_data(name)
    eng = E.Amica(n, T, M, m, precision=0, update_rho=1)
    eng.set_sphered(xs, means, S, ldetS)
    eng.init(A0, c0)
    ref = eng.estep_stats()
    prm = eng.params()
    eng.close()
    # the oracle on the data as this form stores it (FP32): the mu denominator
    # follows the data's last bits near y = 0 (see test_parity_headline_gpu.py)
    orc = O.Oracle(np.asarray(xs, dtype=np.float32).astype(np.float64), M, m, A0, c0, ldetS,
                   nthreads=8)
    orc.prepare()
    s_orc = orc.estep()

    NP = 32 if n <= 32 else (64 if n <= 64 else (128 if n <= 128 else 256))
    dev = torch.device("cuda:0")
    x = torch.zeros((T, NP), dtype=torch.float32, device=dev)
    x[:, :n] = torch.from_numpy(np.ascontiguousarray(xs, dtype=np.float32)).to(dev)
    dt = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).to(dev)
    A, c, al, mu_d, be, rh, g = (dt(prm[k]) for k in ("A", "c", "alpha", "mu", "beta", "rho", "gm"))
    L = E.lib().amica_stats_len(n, M, m)
    outs = []
    for _ in range(2):
        stats = torch.full((L,), float("nan"), dtype=torch.float64, device=dev)
        E.estep_stats_noalloc(x.data_ptr(), NP, n, T, M, m, A.data_ptr(), c.data_ptr(),
                              al.data_ptr(), mu_d.data_ptr(), be.data_ptr(), rh.data_ptr(),
                              g.data_ptr(), ldetS, stats.data_ptr())
        torch.cuda.synchronize()
        outs.append(stats.cpu().numpy())
    for got in outs:
        assert np.all(np.isfinite(got))
        # against the context entry point: the same kernel, another grid
        assert abs(got[0] - ref[0]) / (n * T) < 1e-6
        errs = _errors(got, ref, n, M, m)
        for k in KEYS + ("md",):
            assert errs[k] < 2e-5, (k, errs)
        # against the FP64 oracle: the plain form's bands
        assert abs(got[0] - s_orc[0]) / (n * T) < 2e-6
        errs_o = _errors(got, s_orc, n, M, m)
        print(name, "vs oracle", {k: f"{v:.1e}" for k, v in errs_o.items()})
        for k in KEYS:
            assert errs_o[k] < 2e-5, (k, errs_o)
        # the mu denominator by its distribution (its largest entries follow the
        # sample nearest y = 0; see test_parity_headline_gpu.py)
        b = O.split_stats(s_orc, n, M, m)
        rel_md = np.abs(O.split_stats(got, n, M, m)["md"] - b["md"]) / np.abs(b["md"])
        assert np.median(rel_md) < 2e-3, np.median(rel_md)
    assert np.array_equal(outs[0], outs[1])


def test_noalloc_rejects_shapes_beyond_its_scratch():
    from cudamica_b200 import engine as E
    with pytest.raises(E.AmicaError) as ei:
        # n = 256 with M = 2 models needs about 8 MiB even on a single cluster;
        # the size check comes before any pointer is used
        E.estep_stats_noalloc(1, 256, 256, 100000, 2, 3, 1, 1, 1, 1, 1, 1, 1, 0.0, 1)
    assert ei.value.code == -25
