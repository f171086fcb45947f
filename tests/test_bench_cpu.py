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


def _reference_arm(env_extra):
    import os
    import subprocess
    import sys
    from pathlib import Path

    root = Path(__file__).resolve().parents[1]
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="", **env_extra)
    return subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "1", "--warmup", "0"],
                          cwd=root, env=env, capture_output=True, text=True, timeout=600)


def test_reference_arm_non_zero_rank_exits_without_work():
    """Under torchrun only rank 0 times the CPU reference; the others exit 0 silently."""
    r = _reference_arm({"RANK": "1", "LOCAL_RANK": "1", "WORLD_SIZE": "2"})
    assert r.returncode == 0, r.stderr[-2000:]
    assert r.stdout.strip() == ""


def test_reference_arm_prints_one_line_on_the_native_metric():
    """Rank 0 prints one JSON line on the native arm's metric, unit, direction
    and workload, with its cpu_baseline and a zero-copy e2e block."""
    import json

    r = _reference_arm({"RANK": "0", "LOCAL_RANK": "0", "WORLD_SIZE": "1"})
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert d["metric"] == bench.METRIC and d["unit"] == "rays/s" and d["higher_is_better"] is True
    assert d["config"]["workload"] == bench.BATCHED_WORKLOAD
    assert d["value"] > 0 and d["steps"] == 1
    cb = d["cpu_baseline"]
    assert cb["value"] == d["value"] and cb["kind"] == "port" and cb["cores"] >= 1 and cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
