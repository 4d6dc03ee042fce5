"""Sharding a batch of independent coils over ranks (one process per GPU).

The reference solves one coil per solver object on one device. Here a batch of coils (the batched plan of
fmm_batch_set_coils) is split by whole coils: every rank computes the same balanced assignment
(fmm_batch_partition: coils by decreasing work, sources + targets, each to the least-loaded rank), builds
a batched plan of its own coils and solves it; coils never interact, so no data crosses ranks until the
fields are gathered (torch.distributed all_gather: NCCL between GPUs, gloo on the CPU) into the targets'
input order on every rank.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib


def partition_coils(src_offsets, tgt_offsets, nparts):
    """part[c] in [0, nparts) for each coil (fmm_batch_partition)."""
    so = np.ascontiguousarray(np.asarray(src_offsets, dtype=np.int64))
    to = np.ascontiguousarray(np.asarray(tgt_offsets, dtype=np.int64))
    if so.shape != to.shape or so.ndim != 1 or len(so) < 1:
        raise ValueError("src_offsets and tgt_offsets must be 1-D with ncoils + 1 entries")
    part = np.zeros(len(so) - 1, dtype=np.int32)
    lib = _lib.load()
    _lib.check(lib.fmm_batch_partition(len(so) - 1, ctypes.c_void_p(so.ctypes.data), ctypes.c_void_p(to.ctypes.data),
                                       int(nparts), ctypes.c_void_p(part.ctypes.data)))
    return part


class Shard:
    """One rank's coils of a batch: their sources and targets (contiguous, in coil order), the local coil
    offsets, and where the shard's targets sit in the batch's target order."""

    def __init__(self, xyz, w, J, tgt, src_offsets, tgt_offsets, part, rank):
        so = np.asarray(src_offsets, dtype=np.int64)
        to = np.asarray(tgt_offsets, dtype=np.int64)
        self.coils = np.nonzero(np.asarray(part) == rank)[0]
        src_idx = [np.arange(so[c], so[c + 1]) for c in self.coils]
        tgt_idx = [np.arange(to[c], to[c + 1]) for c in self.coils]
        self.src_index = np.concatenate(src_idx) if len(src_idx) else np.zeros(0, np.int64)
        self.tgt_index = np.concatenate(tgt_idx) if len(tgt_idx) else np.zeros(0, np.int64)
        self.src_offsets = np.r_[0, np.cumsum([len(i) for i in src_idx])].astype(np.int64)
        self.tgt_offsets = np.r_[0, np.cumsum([len(i) for i in tgt_idx])].astype(np.int64)
        self.xyz = np.asarray(xyz)[self.src_index]
        self.w = np.asarray(w)[self.src_index]
        self.J = None if J is None else np.asarray(J)[self.src_index]
        self.tgt = np.asarray(tgt)[self.tgt_index]


def solve_shard_on_gpu(shard, order=8, leaf_capacity=32, precision="fp32", m2l="bf16x3", device=0, current=1.0):
    """B at the shard's targets ([m_r, 3] CUDA tensor) from a batched plan of the shard's coils."""
    import torch
    from .solver import Plan
    dt = torch.float32 if precision == "fp32" else torch.float64
    dev = f"cuda:{device}"
    if len(shard.coils) == 0 or len(shard.tgt) == 0:
        return torch.zeros((len(shard.tgt), 3), dtype=dt, device=dev)
    plan = Plan(order=order, leaf_capacity=leaf_capacity, precision=precision, m2l=m2l, device=device)
    t = lambda a: torch.as_tensor(np.ascontiguousarray(a), dtype=dt).to(dev)
    plan.set_sources(t(shard.xyz), t(shard.w), None if shard.J is None else t(shard.J))
    plan.set_targets(t(shard.tgt))
    plan.set_coils(shard.src_offsets, shard.tgt_offsets)
    B, _ = plan.solve(current, 1)
    plan.close()
    return B


def gather_fields(shard, B_local, n_targets, rank, world, group=None):
    """The batch's B in target input order on every rank: each rank's [m_r, 3] block goes to its targets'
    positions. Ranks pad their blocks to the largest shard (all_gather needs equal shapes)."""
    import torch
    import torch.distributed as dist
    m_local = torch.tensor([len(shard.tgt_index)], dtype=torch.int64, device=B_local.device)
    sizes = [torch.zeros_like(m_local) for _ in range(world)]
    dist.all_gather(sizes, m_local, group=group)
    sizes = [int(s.item()) for s in sizes]
    cap = max(max(sizes), 1)
    pad = torch.zeros((cap, 4), dtype=torch.float64, device=B_local.device)
    if sizes[rank]:
        pad[:sizes[rank], :3] = B_local.to(torch.float64)
        pad[:sizes[rank], 3] = torch.as_tensor(shard.tgt_index, dtype=torch.float64, device=B_local.device)
    blocks = [torch.empty_like(pad) for _ in range(world)]
    dist.all_gather(blocks, pad, group=group)
    out = torch.zeros((n_targets, 3), dtype=torch.float64, device=B_local.device)
    for r, blk in enumerate(blocks):
        if sizes[r]:
            idx = blk[:sizes[r], 3].round().to(torch.int64)
            out[idx] = blk[:sizes[r], :3]
    return out.to(B_local.dtype)


def solve_batch_sharded(xyz, w, J, tgt, src_offsets, tgt_offsets, rank, world, solve=None, group=None, **plan_kw):
    """Solves the batch with its coils split over `world` ranks (call on every rank, with the same batch).
    `solve(shard)` returns B at the shard's targets (default: solve_shard_on_gpu with plan_kw). Returns
    (B of the whole batch in target input order, this rank's Shard)."""
    part = partition_coils(src_offsets, tgt_offsets, world)
    shard = Shard(xyz, w, J, tgt, src_offsets, tgt_offsets, part, rank)
    B_local = solve(shard) if solve is not None else solve_shard_on_gpu(shard, **plan_kw)
    return gather_fields(shard, B_local, len(tgt), rank, world, group), shard
