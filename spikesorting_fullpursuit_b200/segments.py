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


def worker_budget(total_memory, streams, n_segments):
    """Device bytes each of ``min(streams, n_segments)`` concurrent pursuits
    plans its chunks for: an equal share of the budget the reference gives one
    pursuit, max(total / 2, total - 1 GiB) (binary_pursuit_parallel.py:389-408),
    so the workers together stay within it."""
    budget = max(0.5 * total_memory, total_memory - (1 << 30))
    return budget / max(1, min(int(streams), int(n_segments)))


def _run_local(segments, mine, lengths, pursue, streams, kwargs, pursue_is_default=False):
    """Results of this rank's segments, by segment index.  With streams > 1 the
    segments (longest first) are taken by that many worker threads; on a CUDA
    device each worker issues its segments on a stream of its own, so several
    segments' kernels run on the GPU at once (every call keeps its own
    workspace; the library's per-call state is thread-local)."""
    if streams <= 1 or len(mine) <= 1:
        return {i: pursue(*segments[i], **kwargs) for i in mine}
    import queue
    import threading

    import torch

    use_cuda = torch.cuda.is_available()
    device = torch.cuda.current_device() if use_cuda else None
    if use_cuda and pursue_is_default and kwargs.get("max_gpu_memory") is None:
        total = torch.cuda.get_device_properties(device).total_memory
        kwargs = dict(kwargs, max_gpu_memory=worker_budget(total, streams, len(mine)))
    todo = queue.Queue()
    for i in sorted(mine, key=lambda k: (-lengths[k], k)):
        todo.put(i)
    out, errors = {}, []

    def worker():
        stream = None
        if use_cuda:
            torch.cuda.set_device(device)
            stream = torch.cuda.Stream(device)
        while True:   # a failure does not stop the others: the lowest failing index is re-raised
            try:
                i = todo.get_nowait()
            except queue.Empty:
                return
            try:
                if stream is not None:
                    with torch.cuda.stream(stream):
                        out[i] = pursue(*segments[i], **kwargs)
                    stream.synchronize()
                else:
                    out[i] = pursue(*segments[i], **kwargs)
            except BaseException as exc:   # re-raised in the caller, in segment order
                errors.append((i, exc))

    threads = [threading.Thread(target=worker) for _ in range(min(streams, len(mine)))]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    if errors:
        raise min(errors, key=lambda e: e[0])[1]
    return out


def pursue_segments(segments, pursue: Callable = None, group=None, streams: int = 1, **kwargs):
    """Run ``pursue(*segment)`` for every segment on the rank that owns it.

    segments: sequence of argument tuples for ``pursue`` (by default the
    drop-in binary_pursuit: (voltage, v_dtype, sort_info, separability_metrics)).
    streams: segments of one rank pursued at once (worker threads, one CUDA
    stream each); 1 runs them one after another.  With the default pursuit and
    no ``max_gpu_memory``, each worker plans its chunks for 1/streams of the
    device budget; a segment longer than that share is then chunked where a
    sequential run would not chunk it (chunk boundaries, and the duplicates the
    reference leaves in chunk overlaps, follow the budget).
    Returns the list of results in segment order on every rank.  Without an
    initialised process group everything runs locally.  A rank whose pursuit
    fails still takes part in the final gather, so no rank waits on it: the
    failing rank re-raises its own error, the others raise RuntimeError naming
    the lowest failing rank."""
    import torch.distributed as dist

    default = pursue is None
    if default:
        from .overlap.binary_pursuit_parallel import binary_pursuit as pursue
    dist_on = dist.is_available() and dist.is_initialized()
    world = dist.get_world_size(group) if dist_on else 1
    rank = dist.get_rank(group) if dist_on else 0
    lengths = [int(seg[0].shape[1]) for seg in segments]
    mine = shard_segments(lengths, world)[rank]
    if not dist_on:
        local = _run_local(segments, mine, lengths, pursue, int(streams), kwargs, default)
        return [local[i] for i in range(len(segments))]
    error = None
    try:
        local = _run_local(segments, mine, lengths, pursue, int(streams), kwargs, default)
    except Exception as exc:   # every rank must still reach the gather below
        local, error = {}, exc
    gathered = [None] * world
    dist.all_gather_object(gathered, (local, None if error is None else "%s: %s" % (type(error).__name__, error)),
                           group=group)
    if error is not None:
        raise error
    failed = [(r, msg) for r, (_, msg) in enumerate(gathered) if msg is not None]
    if failed:
        raise RuntimeError("segment pursuit failed on rank %d: %s" % failed[0])
    out = {}
    for part, _ in gathered:
        out.update(part)
    return [out[i] for i in range(len(segments))]
