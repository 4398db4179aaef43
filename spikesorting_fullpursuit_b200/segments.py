"""Binary pursuit over many independent segments, sharded across GPUs.

The reference pursues a recording segment by segment, one after another
(spikesorting_fullpursuit/parallel/spikesorting_parallel.py:2161-2184, each
segment through full_binary_pursuit -> binary_pursuit).  Segments share no
data, so with one process per GPU (torch.distributed, NCCL or gloo) each rank
pursues its own share and nothing crosses the data path; the only collective is
the final gather of the per-segment results (spike indices, labels, bools and
clips), so every rank returns all results in segment order.

shard_segments() assigns segments to ranks deterministically: longest first,
each to the rank with the least total samples so far (ties to the lower rank).
"""
from __future__ import annotations

from typing import Callable, List, Sequence


def shard_segments(lengths: Sequence[int], world_size: int) -> List[List[int]]:
    """Segment indices per rank, balanced by total length."""
    if world_size < 1:
        raise ValueError("world_size must be >= 1")
    order = sorted(range(len(lengths)), key=lambda i: (-int(lengths[i]), i))
    load = [0] * world_size
    shards: List[List[int]] = [[] for _ in range(world_size)]
    for i in order:
        r = min(range(world_size), key=lambda k: (load[k], k))
        shards[r].append(i)
        load[r] += int(lengths[i])
    for sh in shards:
        sh.sort()
    return shards


def pursue_segments(segments, pursue: Callable = None, group=None, **kwargs):
    """Run ``pursue(*segment)`` for every segment on the rank that owns it.

    segments: sequence of argument tuples for ``pursue`` (by default the
    drop-in binary_pursuit: (voltage, v_dtype, sort_info, separability_metrics)).
    Returns the list of results in segment order on every rank.  Without an
    initialised process group everything runs locally."""
    import torch.distributed as dist

    if pursue is None:
        from .overlap.binary_pursuit_parallel import binary_pursuit as pursue
    dist_on = dist.is_available() and dist.is_initialized()
    world = dist.get_world_size(group) if dist_on else 1
    rank = dist.get_rank(group) if dist_on else 0
    lengths = [int(seg[0].shape[1]) for seg in segments]
    mine = shard_segments(lengths, world)[rank]
    local = {i: pursue(*segments[i], **kwargs) for i in mine}
    if not dist_on:
        return [local[i] for i in range(len(segments))]
    gathered = [None] * world
    dist.all_gather_object(gathered, local, group=group)
    out = {}
    for part in gathered:
        out.update(part)
    return [out[i] for i in range(len(segments))]
