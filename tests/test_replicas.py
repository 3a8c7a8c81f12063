"""The multi-GPU plumbing on CPU: two gloo ranks (127.0.0.1) run the timing
reduction bench.py uses, with a different local time on each rank."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from charm_b200.replicas import (job_seconds_per_transform, max_over_ranks,
                                 split_range)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port),
                      RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        local = 1.5 + rank          # rank 1 is the slower replica
        m = max_over_ranks(local)
        lo, hi = split_range(10, rank, world)
        out.put((rank, m, lo, hi))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_max():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q))
             for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [2.5, 2.5]
    assert [(r[2], r[3]) for r in res] == [(0, 5), (5, 10)]
    # two replicas of 4 steps each in 2.5 s: 0.3125 s per transform
    assert job_seconds_per_transform(2.5, 4, world) == pytest.approx(0.3125)


def test_without_process_group():
    assert max_over_ranks(3.0) == 3.0


def test_split_range_covers_everything():
    for n in (0, 1, 7, 64):
        for world in (1, 2, 3, 8):
            parts = [split_range(n, r, world) for r in range(world)]
            assert parts[0][0] == 0 and parts[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(parts, parts[1:]))
            assert max(h - l for l, h in parts) - min(h - l for l, h in parts) <= 1
    with pytest.raises(ValueError):
        split_range(4, 2, 2)
    with pytest.raises(ValueError):
        job_seconds_per_transform(1.0, 0, 1)
