"""The multi-process host path of bench.py (one process per GPU, timing taken
as the max over ranks, whole-job rate = ranks x iterations / slowest rank) on
two gloo ranks on the CPU."""
import os
import sys

import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world)
    ws, r, local = bench.dist_env()
    ms = [3.0 + rank, 8.0 - rank]                       # rank-dependent step times
    mx = bench.reduce_over_ranks(ms, dist, "max", device="cpu")
    mn = bench.reduce_over_ranks([100.0 + rank], dist, "min", device="cpu")
    q.put((r, ws, mx, mn, bench.whole_job_rate(mx[0], ws)))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_reduction_and_rate():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + (os.getpid() % 1000)
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r, (rank, ws, mx, mn, rate) in enumerate(res):
        assert (rank, ws) == (r, 2)
        assert mx == [4.0, 8.0]
        assert mn == [100.0]
        assert rate == pytest.approx(2 * 1000.0 / 4.0)
