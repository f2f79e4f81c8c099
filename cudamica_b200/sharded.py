"""Sample-sharded fitting: one process per GPU, each holding a contiguous range
of the samples, one all-reduce per iteration.

The reference splits its sample blocks over devices and sums the per-device
statistics with peer copies (src/amica.cu:1618-1920, `acumulate` in
src/kernels.cu:834-839).  Here every rank runs the E-step over its own samples
(amica_shard_estep), the sufficient statistics -- sums over samples, about
M (n^2 + 8 n m + 2 n + 2) doubles, 0.47 MB at n = 128, M = 3, m = 3 -- are added
across ranks with one all-reduce (NCCL over NVLink for GPU ranks), and every
rank runs the same FP64 M-step on the same vector (amica_shard_mstep), so the
parameters stay identical without being broadcast.

The class is written against a small shard interface so that the same
orchestration drives the GPU engine (EngineShard, NCCL) and, in the CPU tests,
the FP64 oracle (gloo).
"""
from __future__ import annotations

from typing import Protocol

import numpy as np


def shard_range(T: int, rank: int, world: int) -> tuple[int, int]:
    """Contiguous sample range [t0, t1) of `rank`: the first T % world ranks
    take one sample more."""
    base, extra = divmod(T, world)
    t0 = rank * base + min(rank, extra)
    return t0, t0 + base + (1 if rank < extra else 0)


class Shard(Protocol):
    stats_len: int

    def estep(self, out) -> None:
        """The shard's sufficient statistics into the tensor `out`."""

    def mstep(self, stats, nkeep_total: int):
        """The M-step from the statistics of all shards; returns the
        iteration's record."""


class EngineShard:
    """A GPU context (cudamica_b200.engine.Amica) over one shard's samples.

    The whole iteration is ordered on the context's own stream: the E-step
    writes the statistics there without a host wait, torch takes that stream
    as its current one (an ExternalStream), so the all-reduce waits for the
    E-step and the stream waits for the all-reduce, and the M-step is queued
    behind it; the only host synchronisation is the M-step's read of its
    iteration record."""

    def __init__(self, engine):
        import torch
        self.engine = engine
        self.stats_len = engine.stats_len
        self.torch_stream = torch.cuda.ExternalStream(engine.stream)

    def stream(self):
        import torch
        return torch.cuda.stream(self.torch_stream)

    def estep(self, out) -> None:
        self.engine.shard_estep(out.data_ptr())

    def mstep(self, stats, nkeep_total: int):
        return self.engine.shard_mstep(stats.data_ptr(), nkeep_total)


class ShardedFit:
    """One EM iteration per step(): E-step of this rank's shard, all-reduce of
    the statistics over `group` (a torch.distributed process group, or None
    for a single shard), M-step.  `T_total` is the number of samples of all
    shards.  The statistics buffer lives on `device` (the GPU for NCCL)."""

    def __init__(self, shard: Shard, T_total: int, group=None, device="cuda"):
        import torch
        self.shard = shard
        self.T_total = int(T_total)
        self.group = group
        self.buf = torch.zeros(shard.stats_len, dtype=torch.float64, device=device)

    def step(self):
        import contextlib
        import torch.distributed as dist
        ctx = self.shard.stream() if hasattr(self.shard, "stream") else contextlib.nullcontext()
        with ctx:
            self.shard.estep(self.buf)
            if self.group is not None:
                dist.all_reduce(self.buf, op=dist.ReduceOp.SUM, group=self.group)
            return self.shard.mstep(self.buf, self.T_total)

    def run(self, iters: int) -> list:
        return [self.step() for _ in range(iters)]


def engine_shard_preprocess(engine, T_total: int, group=None) -> None:
    """Centring and sphering of a shard loaded with engine.load_data, on the
    GPU, over the samples of every shard: the column sums and then the scatter
    about the common mean are added across ranks (two all-reduces of n and
    n^2 doubles), and every rank derives the same S and ldetS from them
    (amica_shard_colsum / _scatter / _sphere)."""
    import torch
    import torch.distributed as dist
    n = engine.n
    dev = torch.device("cuda", torch.cuda.current_device())
    sums = torch.zeros(n, dtype=torch.float64, device=dev)
    scatter = torch.zeros(n * n, dtype=torch.float64, device=dev)
    engine.shard_colsum(sums.data_ptr())
    if group is not None:
        dist.all_reduce(sums, op=dist.ReduceOp.SUM, group=group)
    torch.cuda.current_stream(dev).synchronize()
    engine.shard_scatter(sums.data_ptr(), T_total, scatter.data_ptr())
    if group is not None:
        dist.all_reduce(scatter, op=dist.ReduceOp.SUM, group=group)
    torch.cuda.current_stream(dev).synchronize()
    engine.shard_sphere(scatter.data_ptr(), T_total)


def split_samples(x: np.ndarray, rank: int, world: int) -> np.ndarray:
    t0, t1 = shard_range(x.shape[0], rank, world)
    return np.ascontiguousarray(x[t0:t1])


def sharded_sphere(x_shard: np.ndarray, group=None, device="cpu"):
    """Centring and sphering of sharded data (do_sphere = 1): the sample count,
    sum and second-moment matrix of every shard are added with one all-reduce
    (FP64), and every rank forms the same C = E[x x^T] - mean mean^T,
    S = 2 C^{-1/2} and ldetS = -log|det S| (src/preprocess.cu:31-420) and applies
    them to its own samples.  Returns (sphered shard, mean, S, ldetS, T_total)."""
    import torch
    import torch.distributed as dist
    xd = np.asarray(x_shard, dtype=np.float64)
    n = xd.shape[1]
    buf = np.concatenate([[float(xd.shape[0])], xd.sum(0), (xd.T @ xd).ravel()])
    t = torch.tensor(buf, dtype=torch.float64, device=device)
    if group is not None:
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    v = t.cpu().numpy()
    T = int(round(v[0]))
    mean = v[1:n + 1] / T
    Cm = v[n + 1:].reshape(n, n) / T - np.outer(mean, mean)
    Cm = 0.5 * (Cm + Cm.T)
    d, V = np.linalg.eigh(Cm)
    S = (V * (2.0 / np.sqrt(d))[None, :]) @ V.T
    ldetS = -float(np.sum(np.log(2.0 / np.sqrt(d))))
    xs = np.ascontiguousarray((xd - mean[None, :]) @ S.T)
    return xs, mean, S, ldetS, T
