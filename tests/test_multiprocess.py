"""Sharding of independent segments across ranks (gloo, world size 2, CPU)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from spikesorting_fullpursuit_b200.overlap.binary_pursuit_parallel import plan_chunks
from spikesorting_fullpursuit_b200.segments import pursue_segments, shard_segments, worker_budget


def test_shards_are_balanced_and_deterministic():
    lengths = [50, 10, 40, 30, 30, 5, 60]
    sh = shard_segments(lengths, 3)
    assert sorted(i for s in sh for i in s) == list(range(len(lengths)))
    loads = [sum(lengths[i] for i in s) for s in sh]
    assert max(loads) - min(loads) <= max(lengths)
    assert sh == shard_segments(lengths, 3)
    assert shard_segments(lengths, 1) == [list(range(len(lengths)))]
    with pytest.raises(ValueError):
        shard_segments(lengths, 0)


def _fake_pursue(voltage, tag):
    # deterministic stand-in for binary_pursuit: indices of threshold crossings
    idx = np.flatnonzero(voltage[0] > 2.0).astype(np.int64)
    return idx, np.full(idx.size, tag, dtype=np.int64)


def _segments():
    rng = np.random.default_rng(3)
    return [(rng.standard_normal((2, n)).astype(np.float32), k) for k, n in enumerate([900, 300, 700, 500, 100])]


def _worker(rank, world, port, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        res = pursue_segments(_segments(), pursue=_fake_pursue)
        out[rank] = [(r[0].tolist(), r[1].tolist()) for r in res]
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_ranks_gather_every_segment_in_order():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        port = _free_port()
        procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        want = [(_fake_pursue(*seg)[0].tolist(), _fake_pursue(*seg)[1].tolist()) for seg in _segments()]
        assert out[0] == want
        assert out[1] == want


def _pursue_failing_on_segment_2(voltage, tag):
    if tag == 2:
        raise ValueError("bad segment %d" % tag)
    return _fake_pursue(voltage, tag)


def _failing_worker(rank, world, port, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    # a short timeout: a rank left waiting in the gather would fail this test, not hang it
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=30))
    try:
        pursue_segments(_segments(), pursue=_pursue_failing_on_segment_2)
        out[rank] = "returned"
    except Exception as exc:
        out[rank] = "%s: %s" % (type(exc).__name__, exc)
    finally:
        dist.destroy_process_group()


def test_a_failing_rank_does_not_leave_the_others_waiting():
    owner = next(r for r, sh in enumerate(shard_segments([s[0].shape[1] for s in _segments()], 2)) if 2 in sh)
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        port = _free_port()
        procs = [ctx.Process(target=_failing_worker, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        assert out[owner] == "ValueError: bad segment 2"
        assert out[1 - owner] == "RuntimeError: segment pursuit failed on rank %d: ValueError: bad segment 2" % owner


def test_without_process_group_runs_locally():
    res = pursue_segments(_segments(), pursue=_fake_pursue)
    assert len(res) == 5 and all(r[1][0] == k for k, r in enumerate(res) if r[1].size)


def test_concurrent_workers_return_results_in_segment_order():
    segs = _segments()
    want = pursue_segments(segs, pursue=_fake_pursue)
    got = pursue_segments(segs, pursue=_fake_pursue, streams=3)
    assert len(got) == len(want)
    for g, w in zip(got, want):
        assert np.array_equal(g[0], w[0]) and np.array_equal(g[1], w[1])


def test_concurrent_workers_reraise_the_first_failing_segment():
    def pursue(voltage, tag):
        if tag in (1, 3):
            raise RuntimeError("segment %d" % tag)
        return _fake_pursue(voltage, tag)

    with pytest.raises(RuntimeError, match="segment 1"):
        pursue_segments(_segments(), pursue=pursue, streams=4)


def test_concurrent_pursuits_share_one_pursuit_budget():
    gib = 1 << 30
    total = 183 * gib
    one = total - gib   # the reference's budget for one pursuit on a 183 GiB device
    assert worker_budget(total, 1, 5) == one
    assert worker_budget(total, 4, 5) * 4 == one
    assert worker_budget(total, 8, 3) * 3 == one   # no more workers than segments
    assert worker_budget(2 * gib, 2, 2) == gib / 2  # small devices keep half for one pursuit
    # chunks planned for a worker's share fit that share: a 30 min 64-channel segment that is
    # one chunk alone is cut into several when eight run at once
    args = (1800 * 30000, 64, 200, 76, 30000, 75, total)
    on1, chunk1 = plan_chunks(*args, max_gpu_memory=worker_budget(total, 1, 8))
    on8, chunk8 = plan_chunks(*args, max_gpu_memory=worker_budget(total, 8, 8))
    assert len(on1) == 1 and len(on8) > 1 and chunk8 < chunk1
