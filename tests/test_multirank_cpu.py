"""The multi-rank plumbing of bench.py on CPU: two gloo ranks (127.0.0.1) agree on the slowest rank's
time and the whole-job throughput, and the barrier holds. On the GPU box the same functions run over
NCCL, one rank per GPU, each rank solving its own replica of the workload."""
import os
import socket

import pytest

torch = pytest.importorskip("torch")


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench
    ms = 10.0 + 5.0 * rank                      # rank 1 is the slow one
    bench.barrier(world)
    value, slowest = bench.aggregate(1000, ms, world)
    out.put((rank, value, slowest))
    bench.barrier(world)
    dist.destroy_process_group()


def test_two_gloo_ranks_report_the_slowest_rank():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, value, slowest in res:
        assert slowest == 15.0
        assert abs(value - 2 * 1000 / 0.015) < 1e-6 * value
