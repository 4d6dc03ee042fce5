"""Sharded batches on one GPU: the batch's coils split as two ranks would split them
(fmm_batch_partition), each shard solved by a batched plan of its own coils, one after the other, and the
shards' fields placed in target order equal the one-plan batch (each coil keeps its own root cube, so its
tree does not depend on the other coils). The gather between ranks is covered by the two-rank gloo test
(tests/test_sharding_cpu.py)."""
import numpy as np
import pytest

from bachelors_b200 import Plan, geometry as G
from bachelors_b200.sharding import Shard, partition_coils, solve_shard_on_gpu

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision,m2l,tol", [("fp64", "simt", 1e-12), ("fp32", "bf16x3", 1e-6)])
def test_two_shards_equal_the_one_plan_batch(precision, m2l, tol):
    xyz, w, J, tgt, so, to = G.torus_batch(12, seed=20260024, count_range=(2 ** 9, 2 ** 12), targets_per_coil=512)
    dt = np.float64 if precision == "fp64" else np.float32
    plan = Plan(order=8, leaf_capacity=32, precision=precision, m2l=m2l)
    plan.set_sources(xyz.astype(dt), w.astype(dt), J.astype(dt))
    plan.set_targets(tgt.astype(dt))
    plan.set_coils(so, to)
    Bref, _ = plan.solve(1.0, 1)
    plan.close()
    part = partition_coils(so, to, 2)
    B = np.zeros_like(tgt)
    for rank in range(2):
        sh = Shard(xyz.astype(dt), w.astype(dt), J.astype(dt), tgt.astype(dt), so, to, part, rank)
        assert len(sh.coils) > 0
        Bs = solve_shard_on_gpu(sh, order=8, leaf_capacity=32, precision=precision, m2l=m2l)
        B[sh.tgt_index] = Bs.cpu().numpy()
    assert np.linalg.norm(B - Bref) / np.linalg.norm(Bref) < tol
