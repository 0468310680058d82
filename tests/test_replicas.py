"""The multi-GPU form is independent replicas (no data-path collective):
bench.py takes the slowest rank's device time and sums the particles of all
replicas.  This runs that host logic as two gloo ranks on the CPU."""
import os
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank(rank, world, port, out):
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    local_ms = 100.0 + 50.0 * rank          # rank 1 is the slowest
    tmax = bench.max_over_ranks(local_ms, dist, "cpu")
    value = bench.replica_throughput(world, 1_000_000, 10, tmax)
    out.put((rank, tmax, value))
    dist.barrier()
    dist.destroy_process_group()


def test_two_replicas_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, tmax, value in res:
        assert tmax == 150.0
        assert value == pytest.approx(2 * 1_000_000 * 10 / 0.150)
