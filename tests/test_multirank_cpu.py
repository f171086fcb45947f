"""CPU: the N>1 path's host logic on two gloo ranks.

Each rank owns a disjoint transmitter slice (no collective on the data path);
the step time is the max over ranks, the work the sum, and the per-rank maps
join by concatenation in rank order.  Runs as two spawned processes over
gloo on 127.0.0.1.
"""

from __future__ import annotations

import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from witwin_channel_b200.sharding import gather_concat, reduce_step_time, shard_range


def test_shard_range_covers_every_unit_once():
    for count in (0, 1, 5, 64, 1000):
        for world in (1, 2, 3, 8):
            got = [shard_range(count, r, world) for r in range(world)]
            assert got[0][0] == 0 and got[-1][1] == count
            assert all(a[1] == b[0] for a, b in zip(got, got[1:]))
            sizes = [b - a for a, b in got]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        shard_range(4, 2, 2)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank: int, world: int, port: int, results) -> None:
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    from datetime import timedelta

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        num_tx, num_rx = 5, 7
        start, stop = shard_range(num_tx, rank, world)
        # stand-in per-rank radiomap: a deterministic function of (tx, rx)
        tx = torch.arange(start, stop, dtype=torch.float64)[:, None]
        rx = torch.arange(num_rx, dtype=torch.float64)[None, :]
        local = (tx * 100 + rx).contiguous()
        full = gather_concat(local)
        step_ms, units = reduce_step_time(10.0 + rank, float(local.numel()))
        results[rank] = (full.tolist(), step_ms, units)
    finally:
        dist.destroy_process_group()


def test_two_rank_gloo_shard_gather_and_timing():
    ctx = mp.get_context("spawn")
    world = 2
    manager = ctx.Manager()
    results = manager.dict()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, results)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    for p in procs:
        if p.is_alive():
            p.kill()
        assert p.exitcode == 0
    want = [[t * 100 + r for r in range(7)] for t in range(5)]
    for rank in range(world):
        full, step_ms, units = results[rank]
        assert full == want
        assert step_ms == 11.0  # max over ranks
        assert units == 35.0    # every cell once
