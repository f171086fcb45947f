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


# ------------------------------------------------------ gradient reduction
def _grad_job():
    """A small reflection scene with an 8x3 receiver grid, its frozen path
    table (oracle, FP64) and the parameters of the gradient check."""
    import numpy as np

    from oracle import solve as osolve
    from tests import scenes
    from witwin_channel_b200.scene import Scene, make_receiver_grid

    base = scenes.two_wall_scene()
    grid = make_receiver_grid(origin=[0.2, 0.4, 0.6], x_axis=[0.0, 1.0, 0.0], y_axis=[1.0, 0.0, 0.0], shape=(8, 3),
                              spacing=(0.2, 0.3))
    scene = Scene(structures=base.structures, endpoints=[base.transmitters[0], grid])
    f = 3.0e9
    arrays = osolve.scene_arrays(scene, f)
    ref = osolve.solve(arrays, components={"los", "reflection"}, max_depth=2, frequency=f)
    table = {k: np.asarray(ref["rows"][k]) for k in ("tx_id", "rx_id", "component_id", "depth", "primitive_sequence",
                                                    "edge_id")}
    params = [("vertex", 0, 0), ("vertex", 3, 0), ("vertex", 5, 1), ("eps_r", 0, 0), ("sigma_e", 1, 0),
              ("tx", 0, 2)]
    return scene, grid, arrays, table, f, params


def _fd_gradient(arrays, table, f, params, cells):
    """Central differences (h = 1e-5) of sum_cells w_c |sum of the cell's path fields|^2."""
    import numpy as np

    from oracle import adjoint as oadj

    R = arrays["rx_pos"].shape[0]
    w = np.linspace(0.5, 1.5, R)

    def loss(a2):
        fields = oadj.fixed_topology_fields(a2, table, f)
        pg = oadj.cell_path_gain(fields, table, 1, R)[0]
        return float((w[cells] * pg[cells]).sum() / 1e-6)

    out = []
    for kind, i, c in params:
        def moved(h):
            a2 = dict(arrays)
            a2["face_mats"] = {k: v.copy() for k, v in arrays["face_mats"].items()}
            if kind == "vertex":
                a2["vertices"] = arrays["vertices"].copy()
                a2["vertices"][i, c] += h
            elif kind in ("eps_r", "sigma_e"):
                a2["face_mats"][kind][arrays["face_material"] == i] += h
            else:
                a2["tx_pos"] = arrays["tx_pos"].copy()
                a2["tx_pos"][i, c] += h
            return a2
        h = 1e-5
        out.append((loss(moved(h)) - loss(moved(-h))) / (2 * h))
    return np.array(out)


def _grad_worker(rank: int, world: int, port: int, results) -> None:
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    from datetime import timedelta

    import numpy as np

    from witwin_channel_b200.sharding import allreduce_gradients, shard_grid

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        scene, grid, arrays, table, f, params = _grad_job()
        sub, (start, stop) = shard_grid(grid, rank, world)
        cols = grid.shape[1]
        cells = np.arange(start * cols, stop * cols)  # this rank's receiver tile (its rows of the grid)
        pts_full = grid.points()[start * cols:stop * cols]
        g = _fd_gradient(arrays, table, f, params, cells)
        leaf = torch.zeros(len(params), dtype=torch.float64, requires_grad=True)
        leaf.grad = torch.tensor(g)
        allreduce_gradients([leaf])
        results[rank] = (leaf.grad.tolist(), torch.allclose(sub.points(), pts_full, atol=1e-5), stop - start)
    finally:
        dist.destroy_process_group()


def test_two_rank_gloo_gradient_allreduce():
    """Each rank takes half of the receiver rows (its tile), computes the
    oracle's FP64 fixed-topology gradient of its part of a sum-over-cells
    loss, and the all-reduced gradient equals the single-rank gradient of the
    whole job."""
    import numpy as np

    ctx = mp.get_context("spawn")
    world = 2
    manager = ctx.Manager()
    results = manager.dict()
    port = _free_port()
    procs = [ctx.Process(target=_grad_worker, args=(r, world, port, results)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(180)
    for p in procs:
        if p.is_alive():
            p.kill()
        assert p.exitcode == 0
    scene, grid, arrays, table, f, params = _grad_job()
    full = _fd_gradient(arrays, table, f, params, np.arange(grid.shape[0] * grid.shape[1]))
    assert np.abs(full).min() > 0
    for rank in range(world):
        reduced, same_points, rows = results[rank]
        assert same_points and rows == 4
        np.testing.assert_allclose(reduced, full, rtol=1e-9, atol=1e-12 * np.abs(full).max())
