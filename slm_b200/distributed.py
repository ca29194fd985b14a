"""Seed sharding across GPUs (one process per GPU).

The field pass shards by seed: rank r traces the contiguous range
``[n*r/W, n*(r+1)/W)`` of the shuffled seed list (``seeds_chunk_offset`` and
``n_seed_points`` select it; each trajectory's RNG stream follows its global
seed index, so no trajectory changes), keeps private uint64 slc/slt, and one
all-reduce (sum) combines them -- the path's only exchange.  Integer sums make
the result identical to one GPU whatever the world size.  uv and mask are
replicated on every rank.

``sharded_field_pass`` takes the tracing function as an argument so that the
same sharding and reduction logic runs with the CUDA kernels over NCCL in
production and can be exercised with a CPU stand-in over gloo in tests.
"""
from __future__ import annotations

import torch
import torch.distributed as dist


def shard_range(n_seeds, rank, world_size):
    """Contiguous seed range [begin, end) of one rank."""
    n = int(n_seeds)
    return (n * rank) // world_size, (n * (rank + 1)) // world_size


def shard_params(params, rank, world_size):
    """Copy of a field-pass parameter block restricted to this rank's seeds."""
    begin, end = shard_range(params.n_seed_points, rank, world_size)
    p = params.copy()
    p.seeds_chunk_offset = begin
    p.n_seed_points = end
    return p


def allreduce_counts(*tensors, group=None):
    """Sum uint64 accumulators over ranks (as int64: two's-complement addition
    is the same bit pattern as unsigned addition mod 2^64)."""
    for t in tensors:
        dist.all_reduce(t.view(torch.int64), op=dist.ReduceOp.SUM, group=group)


def sharded_field_pass(params, trace_fn, slc, slt, group=None):
    """Trace this rank's shard with ``trace_fn(shard_params, slc, slt) -> steps``
    then all-reduce slc/slt.  Returns (steps of this rank, total steps)."""
    if group is None and not dist.is_initialized():
        steps = int(trace_fn(params, slc, slt))
        return steps, steps
    rank = dist.get_rank(group)
    world = dist.get_world_size(group)
    steps = int(trace_fn(shard_params(params, rank, world), slc, slt))
    allreduce_counts(slc, slt, group=group)
    tot = torch.tensor([steps], dtype=torch.int64, device=slc.device)
    dist.all_reduce(tot, op=dist.ReduceOp.SUM, group=group)
    return steps, int(tot.item())
