"""Multi-process path of bench.py (replicas, no collective on the data path):
two gloo ranks on CPU run the same barrier / max-over-ranks timing as the
GPU ranks do over NCCL, and the whole-job value counts every rank's steps."""
import os

import pytest

torch = pytest.importorskip("torch")


def _rank(rank, world, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    ms = [120.0, 150.0][rank]
    out = bench.replica_aggregate(ms, steps=10, world=world, device="cpu")
    q.put((rank, out))
    dist.destroy_process_group()


def test_replica_timing_takes_the_slowest_rank():
    import multiprocessing as mp
    import random
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + random.randint(0, 2000)
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r in (0, 1):
        ms, value = res[r]
        assert ms == 150.0
        assert value == pytest.approx(2 * 10 / 0.150)
