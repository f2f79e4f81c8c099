"""Sample-sharded fitting on the CPU: two gloo ranks, each with half of the
samples, run cudamica_b200.sharded.ShardedFit (the orchestration the GPU
ranks use with NCCL: E-step per shard, one all-reduce of the statistics,
the same M-step on every rank) with the FP64 oracle as the shard's E-step and
M-step.  The trajectory and the parameters must equal a single oracle fitted
on all samples, up to FP64 summation order; the sharded sphering must equal the
single-process one.
"""
import os
import tempfile

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from cudamica_b200 import sharded, synth


class OracleShard:
    """The FP64 oracle on one shard's samples, behind the Shard interface."""

    def __init__(self, xs, M, m, A0, c0, ldetS):
        from oracle import oracle as O
        self.orc = O.Oracle(xs, M, m, A0, c0, ldetS, nthreads=2)
        self.stats_len = O.stats_len(xs.shape[1], M, m)

    def estep(self, out):
        self.orc.prepare()
        out.copy_(torch.from_numpy(self.orc.estep()))

    def mstep(self, stats, nkeep_total):
        return self.orc.mstep(stats.numpy(), nkeep_total)


N, T, M, m, ITERS = 12, 6000, 2, 3, 3


def _data():
    d = synth.config2(seed=21, n=N, T=T, M=M, m=m, block_lo=300, block_hi=900)
    A0, c0 = synth.norand_init(N, M)
    return d.x, A0, c0


def _rank(rank, world, init_file, out_dir):
    dist.init_process_group("gloo", init_method=f"file://{init_file}", rank=rank, world_size=world)
    try:
        x, A0, c0 = _data()
        xs, mean, S, ldetS, Ttot = sharded.sharded_sphere(sharded.split_samples(x, rank, world),
                                                          group=dist.group.WORLD)
        fit = sharded.ShardedFit(OracleShard(xs, M, m, A0, c0, ldetS), Ttot,
                                 group=dist.group.WORLD, device="cpu")
        lls = fit.run(ITERS)
        p = fit.shard.orc.params()
        np.savez(os.path.join(out_dir, f"rank{rank}.npz"), ll=np.array(lls), S=S, ldetS=ldetS,
                 T=Ttot, **{k: p[k] for k in ("A", "c", "alpha", "mu", "beta", "rho", "gm")})
    finally:
        dist.destroy_process_group()


def test_shard_ranges_cover_the_samples():
    for T_, w in ((10, 3), (7, 2), (1000, 8), (5, 5)):
        ranges = [sharded.shard_range(T_, r, w) for r in range(w)]
        assert ranges[0][0] == 0 and ranges[-1][1] == T_
        assert all(a[1] == b[0] for a, b in zip(ranges, ranges[1:]))
        sizes = [b - a for a, b in ranges]
        assert max(sizes) - min(sizes) <= 1


def test_two_gloo_ranks_match_one_oracle():
    from oracle import oracle as O
    world = 2
    with tempfile.TemporaryDirectory() as td:
        init_file = os.path.join(td, "init")
        mp.start_processes(_rank, args=(world, init_file, td), nprocs=world, join=True,
                           start_method="spawn")
        r = [np.load(os.path.join(td, f"rank{k}.npz")) for k in range(world)]
    x, A0, c0 = _data()
    xs, mean, S, ldetS, Ttot = sharded.sharded_sphere(x)
    assert Ttot == T and int(r[0]["T"]) == T
    assert np.max(np.abs(r[0]["S"] - S)) < 1e-12 and abs(float(r[0]["ldetS"]) - ldetS) < 1e-10
    orc = O.Oracle(xs, M, m, A0, c0, ldetS, nthreads=2)
    ll = [orc.step() for _ in range(ITERS)]
    # two FP64 summation orders: equal to ~1e-15 after one iteration, then the
    # EM map amplifies the difference (x10-x100 per iteration)
    for k in range(world):
        d = np.abs(r[k]["ll"] - np.array(ll))
        assert d[0] < 1e-13 and np.all(d < 1e-13 * 100.0 ** np.arange(ITERS)), (k, d)
    p = orc.params()
    for key in ("A", "c", "alpha", "mu", "beta", "rho", "gm"):
        # both ranks hold the same parameters, equal to the single fit's
        assert np.array_equal(r[0][key], r[1][key]), key
        err = np.max(np.abs(r[0][key] - p[key])) / max(np.max(np.abs(p[key])), 1e-300)
        assert err < 1e-7, (key, err)
