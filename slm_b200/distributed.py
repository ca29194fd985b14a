"""Seed sharding across GPUs (one process per GPU).

The field pass shards by seed.  The tracer's queue (the spatial order, or the
shuffled list itself) is dealt to the ranks in chunks of ``SHARD_CHUNK``
consecutive queue positions, round robin: rank r takes chunks r, r+W, r+2W,
...  (``shard_queue``).  Each rank thus sweeps the whole grid in the same
spatial order as one GPU would, and no rank holds a whole region: trajectory
lengths cluster in space (the longest start on a few pixels of a valley
floor), so contiguous ranges of a spatial queue -- bands of the DTM -- load
the ranks unevenly.  Each trajectory's RNG stream follows its seed index, so
no trajectory changes; each rank keeps private uint64 slc/slt, and one
all-reduce (sum) combines them -- the path's only exchange.  Integer sums make
the result identical to one GPU whatever the world size and the dealing.  uv
and mask are replicated on every rank.

``shard_range`` / ``shard_params`` keep the contiguous form (a rank's range
of the queue through ``seeds_chunk_offset`` and ``n_seed_points``).

``sharded_field_pass`` takes the tracing function as an argument so that the
same sharding and reduction logic runs with the CUDA kernels over NCCL in
production and can be exercised with a CPU stand-in over gloo in tests.
"""
from __future__ import annotations

import numpy as np
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


SHARD_CHUNK = 64  # queue positions per dealt chunk (256 trajectories at d=2)


def shard_positions(n_seeds, rank, world_size, chunk=SHARD_CHUNK):
    """Queue positions (int64 array, ascending) one rank takes when chunks of
    ``chunk`` consecutive positions are dealt round robin."""
    n, w, c = int(n_seeds), int(world_size), int(chunk)
    if n <= 0:
        return np.zeros(0, np.int64)
    starts = np.arange(int(rank) * c, n, w * c, dtype=np.int64)
    pos = (starts[:, None] + np.arange(c, dtype=np.int64)[None, :]).reshape(-1)
    return pos[pos < n]


def shard_queue(order, n_seeds, rank, world_size, chunk=SHARD_CHUNK, device=None):
    """This rank's tracer queue: the seed indices (uint32 tensor) at its dealt
    positions of ``order`` (a uint32 tensor of seed indices, or None for the
    seed list's own order).  Trace it with ``shard_queue_params``."""
    n, w, c = int(n_seeds), int(world_size), int(chunk)
    dev = order.device if order is not None else device
    pos = torch.arange(n, dtype=torch.int64, device=dev)
    mine = pos[torch.remainder(torch.div(pos, c, rounding_mode="floor"), w) == int(rank)]
    if order is None:
        return mine.to(torch.int32).view(torch.uint32)
    return order.view(torch.int32)[:n].index_select(0, mine).view(torch.uint32)


def shard_queue_params(params, queue):
    """Copy of a field-pass parameter block that traces ``queue`` (the
    rank's seed indices, passed as the seed order, or their count) from
    position 0."""
    p = params.copy()
    p.seeds_chunk_offset = 0
    p.n_seed_points = int(queue) if isinstance(queue, (int, np.integer)) else int(queue.numel())
    return p


def allreduce_counts(*tensors, group=None):
    """Sum uint64 accumulators over ranks (as int64: two's-complement addition
    is the same bit pattern as unsigned addition mod 2^64)."""
    for t in tensors:
        dist.all_reduce(t.view(torch.int64), op=dist.ReduceOp.SUM, group=group)


def sharded_field_pass(params, trace_fn, slc, slt, group=None, order=None):
    """Trace this rank's shard, then all-reduce slc/slt.  Returns (steps of
    this rank, total steps).

    ``trace_fn(params, slc, slt, queue) -> steps`` traces the seed indices
    ``queue`` (uint32 tensor) with ``params`` sized for it; the rank's queue is
    its dealt share of ``order`` (None: the seed list's order)."""
    if group is None and not dist.is_initialized():
        n = int(params.n_seed_points)
        queue = order if order is not None else shard_queue(None, n, 0, 1, device=slc.device)
        steps = int(trace_fn(shard_queue_params(params, queue), slc, slt, queue))
        return steps, steps
    rank = dist.get_rank(group)
    world = dist.get_world_size(group)
    queue = shard_queue(order, int(params.n_seed_points), rank, world, device=slc.device)
    steps = int(trace_fn(shard_queue_params(params, queue), slc, slt, queue))
    allreduce_counts(slc, slt, group=group)
    tot = torch.tensor([steps], dtype=torch.int64, device=slc.device)
    dist.all_reduce(tot, op=dist.ReduceOp.SUM, group=group)
    return steps, int(tot.item())
