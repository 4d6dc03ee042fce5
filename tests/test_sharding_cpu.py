"""Sharding a batch of coils over ranks (bachelors_b200/sharding.py, fmm_batch_partition) on the CPU: the
partition covers every coil once and balances the work, every rank computes the same assignment, and two
gloo ranks (127.0.0.1) that each solve only their own coils gather the batch's field in target order. The
per-shard solver here is the CPU restatement's direct sum (the product solves shards with a batched plan on
each rank's GPU, tests/test_gpu_sharding.py)."""
import os
import socket

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from bachelors_b200 import geometry as G  # noqa: E402
from bachelors_b200.sharding import Shard, partition_coils  # noqa: E402


def small_batch(seed=20260014, coils=9):
    return G.torus_batch(coils, seed=seed, count_range=(2 ** 7, 2 ** 10), targets_per_coil=64)


def test_partition_covers_and_balances():
    xyz, w, J, tgt, so, to = small_batch(coils=40)
    work = np.diff(so) + np.diff(to)
    for parts in (1, 2, 3, 8):
        part = partition_coils(so, to, parts)
        assert part.shape == (40,) and part.min() >= 0 and part.max() < parts
        load = np.bincount(part, weights=work, minlength=parts)
        # longest-processing-time-first: no part exceeds the mean by more than the largest coil
        assert load.max() <= load.sum() / parts + work.max()
        np.testing.assert_array_equal(part, partition_coils(so, to, parts))   # deterministic
    # more parts than coils: some parts are empty, each coil still in exactly one part
    part = partition_coils(so[:4], to[:4], 8)
    assert len(set(part.tolist())) == 3


def test_shard_reassembles_the_batch():
    xyz, w, J, tgt, so, to = small_batch()
    part = partition_coils(so, to, 3)
    seen_src, seen_tgt = [], []
    for r in range(3):
        sh = Shard(xyz, w, J, tgt, so, to, part, r)
        assert len(sh.src_offsets) == len(sh.coils) + 1 and sh.src_offsets[-1] == len(sh.xyz)
        np.testing.assert_array_equal(sh.xyz, xyz[sh.src_index])
        np.testing.assert_array_equal(sh.tgt, tgt[sh.tgt_index])
        seen_src.append(sh.src_index)
        seen_tgt.append(sh.tgt_index)
    np.testing.assert_array_equal(np.sort(np.concatenate(seen_src)), np.arange(len(xyz)))
    np.testing.assert_array_equal(np.sort(np.concatenate(seen_tgt)), np.arange(len(tgt)))


def _direct_per_coil(shard):
    from oracle import oracle as O
    out = np.zeros((len(shard.tgt), 3))
    for k in range(len(shard.coils)):
        s0, s1 = shard.src_offsets[k], shard.src_offsets[k + 1]
        t0, t1 = shard.tgt_offsets[k], shard.tgt_offsets[k + 1]
        if t1 > t0 and s1 > s0:
            out[t0:t1] = O.direct(shard.xyz[s0:s1], shard.w[s0:s1], shard.J[s0:s1], shard.tgt[t0:t1])
    return torch.from_numpy(out)


def _worker(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    from bachelors_b200.sharding import solve_batch_sharded
    xyz, w, J, tgt, so, to = small_batch()
    B, shard = solve_batch_sharded(xyz, w, J, tgt, so, to, rank, world, solve=_direct_per_coil)
    q.put((rank, B.numpy(), shard.coils.tolist()))
    dist.barrier()
    dist.destroy_process_group()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def test_two_gloo_ranks_gather_the_batch():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=180) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    xyz, w, J, tgt, so, to = small_batch()
    part = partition_coils(so, to, 1)
    ref = _direct_per_coil(Shard(xyz, w, J, tgt, so, to, part, 0)).numpy()
    (_, B0, c0), (_, B1, c1) = res
    assert sorted(c0 + c1) == list(range(len(so) - 1)) and c0 and c1   # both ranks worked, no coil twice
    np.testing.assert_allclose(B0, ref, rtol=0, atol=1e-20)
    np.testing.assert_array_equal(B0, B1)
