"""Sample-sharded fitting on one GPU: two contexts, each over half of the
samples, against one context over all of them.

The E-step statistics are sums over samples, so the two shards' vectors add up
to the whole fit's (up to the grouping of the FP32 per-tile partial sums); the
M-step of each shard context then runs on the added vector with the sample
count of both (amica_shard_mstep) and both contexts hold bit-identical
parameters, which follow the single-context fit.  This is the per-rank work of
a multi-GPU run (cudamica_b200.sharded.ShardedFit), without the all-reduce,
which here is a torch addition.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from cudamica_b200 import synth
from cudamica_b200.sharded import shard_range, sharded_sphere

pytestmark = pytest.mark.gpu


def _sections(n, M, m):
    """(name, slice) of the flat statistics vector: the LL numerator, then per
    model vsum, cnew, sigma2 numerator, phi and the seven mixture sums."""
    S = 1 + 2 * n + n * n + 7 * m * n
    out = [("ll", slice(0, 1))]
    for h in range(M):
        b = 1 + h * S
        out += [(f"vsum{h}", slice(b, b + 1)), (f"cn{h}", slice(b + 1, b + 1 + n)),
                (f"s2{h}", slice(b + 1 + n, b + 1 + 2 * n)),
                (f"phi{h}", slice(b + 1 + 2 * n, b + 1 + 2 * n + n * n))]
        for k, nm in enumerate(("us", "kn", "ln", "mn", "md", "bd", "rn")):
            o = b + 1 + 2 * n + n * n + k * m * n
            out.append((f"{nm}{h}", slice(o, o + m * n)))
    return out


@pytest.mark.parametrize("precision", [0, 1])
def test_two_shards_match_one_context(precision):
    from cudamica_b200.engine import Amica
    n, T, M, m = 128, 200_000, 3, 3
    d = synth.config2(seed=5, n=n, T=T, M=M, m=m)
    xs, mean, S, ldetS, Tt = sharded_sphere(d.x)
    assert Tt == T
    A0, c0 = synth.norand_init(n, M)

    def ctx(lo, hi):
        e = Amica(n, hi - lo, M, m, precision=precision, update_rho=1)
        e.set_sphered(xs[lo:hi], mean, S, ldetS)
        e.init(A0, c0)
        return e

    full = ctx(0, T)
    shards = [ctx(*shard_range(T, r, 2)) for r in range(2)]
    L = full.stats_len
    dev = torch.device("cuda:0")
    bufs = [torch.zeros(L, dtype=torch.float64, device=dev) for _ in range(3)]
    for it in range(3):
        full.shard_estep(bufs[2].data_ptr())
        for e, b in zip(shards, bufs):
            e.shard_estep(b.data_ptr())
        torch.cuda.synchronize()                # the E-steps run on the contexts' streams
        tot = bufs[0] + bufs[1]
        torch.cuda.synchronize()
        if it == 0:
            # linearity of the statistics in the samples, per section
            a, f = tot.cpu().numpy(), bufs[2].cpu().numpy()
            worst = max(((float(np.max(np.abs(a[s] - f[s])) / max(np.max(np.abs(f[s])), 1e-300)), nm)
                         for nm, s in _sections(n, M, m)))
            print(f"precision={precision}: shard sum vs whole, worst section {worst[1]} {worst[0]:.2e}")
            assert worst[0] < (5e-5 if precision else 1e-5), worst
        outs = [e.shard_mstep(tot.data_ptr(), T) for e in shards]
        of = full.shard_mstep(bufs[2].data_ptr(), T)
        assert outs[0].ll == outs[1].ll and outs[0].nkeep == T
        p0, p1, pf = shards[0].params(), shards[1].params(), full.params()
        for k in p0:
            assert np.array_equal(p0[k], p1[k]), k          # the same M-step on the same vector
        print(f"  iteration {it + 1}: LL shards {outs[0].ll:.10f} whole {of.ll:.10f}")
        # the mixed form's statistics differ by its FP32 tensor-memory
        # accumulation over a different grouping of tiles (1.5e-5 of phi)
        assert abs(outs[0].ll - of.ll) < (1e-7 if precision else 1e-8) * 100 ** it
        if it == 0:
            # one M-step from statistics equal to ~1e-6: parameters equal to
            # that level (later iterations amplify it, the early EM map being
            # far from its fixed point)
            for k in ("A", "mu", "beta", "rho", "alpha"):
                err = np.max(np.abs(p0[k] - pf[k])) / np.max(np.abs(pf[k]))
                print(f"    {k}: {err:.2e}")
                assert err < 2e-5, (k, err)
    for e in shards + [full]:
        e.close()


@pytest.mark.parametrize("n", [64, 160])
def test_sharded_preprocessing_matches_one_context(n):
    """Raw data loaded shard by shard, centred and sphered on the GPU with the
    column sums and scatters of both shards added between the calls
    (amica_shard_colsum / _scatter / _sphere): the same mean, S and ldetS as
    amica_preprocess over all samples, and the same E-step statistics.  n = 160
    runs the cooperative eigensolver of the n > 128 path."""
    from cudamica_b200.engine import Amica
    T, M, m = 120_000, 2, 3
    d = synth.config2(seed=9, n=n, T=T, M=M, m=m)
    A0, c0 = synth.norand_init(n, M)
    dev = torch.device("cuda:0")
    full = Amica(n, T, M, m, precision=0)
    full.load_data(d.x)
    full.preprocess()
    rng = [shard_range(T, r, 2) for r in range(2)]
    shards = [Amica(n, hi - lo, M, m, precision=0) for lo, hi in rng]
    for e, (lo, hi) in zip(shards, rng):
        e.load_data(d.x[lo:hi])
    sums = [torch.zeros(n, dtype=torch.float64, device=dev) for _ in shards]
    scat = [torch.zeros(n * n, dtype=torch.float64, device=dev) for _ in shards]
    for e, s in zip(shards, sums):
        e.shard_colsum(s.data_ptr())
    st = sums[0] + sums[1]
    torch.cuda.synchronize()
    for e, s in zip(shards, scat):
        e.shard_scatter(st.data_ptr(), T, s.data_ptr())
    sc = scat[0] + scat[1]
    torch.cuda.synchronize()
    for e in shards:
        e.shard_sphere(sc.data_ptr(), T)
    Sf, mf, lf = full.sphere()
    for e in shards:
        S, mn, ld = e.sphere()
        assert np.max(np.abs(mn - mf)) < 1e-12 * max(1.0, np.max(np.abs(mf)))
        assert np.max(np.abs(S - Sf)) < 1e-9 * np.max(np.abs(Sf)), np.max(np.abs(S - Sf))
        assert abs(ld - lf) < 1e-9 * max(1.0, abs(lf))
    L = full.stats_len
    bufs = [torch.zeros(L, dtype=torch.float64, device=dev) for _ in range(3)]
    for e, b in zip(shards + [full], bufs):
        e.init(A0, c0)
        e.shard_estep(b.data_ptr())
    torch.cuda.synchronize()
    a, f = (bufs[0] + bufs[1]).cpu().numpy(), bufs[2].cpu().numpy()
    worst = max(((float(np.max(np.abs(a[s] - f[s])) / max(np.max(np.abs(f[s])), 1e-300)), nm)
                 for nm, s in _sections(n, M, m)))
    print(f"n={n}: sharded preprocessing, shard sum vs whole, worst section {worst[1]} {worst[0]:.2e}")
    assert worst[0] < 2e-5, worst
    for e in shards + [full]:
        e.close()
