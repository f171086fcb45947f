"""Host logic of the benchmark's multi-GPU partition (no GPU needed)."""

from __future__ import annotations

import pytest

import bench


@pytest.mark.parametrize("world", [1, 2, 3, 4, 8])
def test_batched_jobs_partition_every_job_once(world):
    parts = [bench._batched_jobs(world, r) for r in range(world)]
    flat = sorted(j for p in parts for j in p)
    assert flat == sorted((s, t) for s in range(8) for t in range(4))
    assert all(p for p in parts)  # every rank gets work (32 jobs >= 8 ranks)


def test_batched_jobs_balance():
    from witwin_channel_b200.workloads import BATCH_BOXES, BATCH_GRID

    def cost(j):
        return BATCH_GRID[j[0]] ** 2 * BATCH_BOXES[j[0]]

    for world in (2, 4, 8):
        loads = [sum(cost(j) for j in bench._batched_jobs(world, r)) for r in range(world)]
        biggest = max(cost((s, 0)) for s in range(8))
        # longest processing time first: no rank exceeds the mean by more than one job
        assert max(loads) <= sum(loads) / world + biggest
