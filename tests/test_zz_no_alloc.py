"""The allocation-free E-step entry point (amica_estep_stats_noalloc) against
the context-based one (amica_estep_stats).

Callers that cannot allocate device memory -- code inside another framework's
memory pool, or a process that forbids cudaMalloc after start-up -- hand in
their own device buffers and get the same sufficient statistics back; the
library's fixed scratch array holds everything in between.  Both paths run the
same plain FP32 E-step kernel, only on grids of different sizes, so the sums
agree to FP32 summation-order noise (relative 2e-5 is the tolerance the plain
path's tests use).  The call is made twice in a row: the second call reuses the
scratch array the first one left behind.

This file is collected last on purpose.
"""
import numpy as np
import pytest

from golden.cases import CASES, prepared
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["c0", "m3"])
def test_noalloc_matches_context_entry_point(name):
    import torch
    from cudamica_b200 import engine as E

    case = CASES[name]
    p = prepared(case)
    n, T, M, m = case.n, case.T, case.M, case.m
    eng = E.Amica(n, T, M, m, precision=0, update_rho=1)
    eng.set_sphered(p["xs"], p["means"], p["sphere"], p["ldetS"])
    eng.init(p["A0"], p["c0"])
    ref = eng.estep_stats()
    prm = eng.params()
    eng.close()

    NP = 32 if n <= 32 else (64 if n <= 64 else 128)
    dev = torch.device("cuda:0")
    x = torch.zeros((T, NP), dtype=torch.float32, device=dev)
    x[:, :n] = torch.from_numpy(np.ascontiguousarray(p["xs"], dtype=np.float32)).to(dev)
    dt = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).to(dev)
    A, c, al, mu_d, be, rh, g = (dt(prm[k]) for k in ("A", "c", "alpha", "mu", "beta", "rho", "gm"))
    L = E.lib().amica_stats_len(n, M, m)
    outs = []
    for _ in range(2):
        stats = torch.full((L,), float("nan"), dtype=torch.float64, device=dev)
        E.estep_stats_noalloc(x.data_ptr(), NP, n, T, M, m, A.data_ptr(), c.data_ptr(),
                              al.data_ptr(), mu_d.data_ptr(), be.data_ptr(), rh.data_ptr(),
                              g.data_ptr(), p["ldetS"], stats.data_ptr())
        torch.cuda.synchronize()
        outs.append(stats.cpu().numpy())
    for got in outs:
        assert np.all(np.isfinite(got))
        a, b = O.split_stats(got, n, M, m), O.split_stats(ref, n, M, m)
        assert abs(got[0] - ref[0]) / (n * T) < 1e-6
        vsum = float(np.max(b["vs"]))
        for k in ("vs", "cn", "s2", "phi", "us", "kn", "ln", "mn", "md", "bd", "rn"):
            scale = max(np.max(np.abs(b[k])), vsum if k == "cn" else 0.0)
            err = np.max(np.abs(a[k] - b[k])) / scale
            assert err < 2e-5, (k, err)
    assert np.array_equal(outs[0], outs[1])


def test_noalloc_rejects_shapes_beyond_its_scratch():
    from cudamica_b200 import engine as E
    with pytest.raises(E.AmicaError) as ei:
        # n = 128 with M = 8 models needs far more than the fixed 5 MiB
        E.estep_stats_noalloc(1, 128, 128, 100000, 8, 3, 1, 1, 1, 1, 1, 1, 1, 0.0, 1)
    assert ei.value.code == -25
