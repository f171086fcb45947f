"""Process-parallel drivers of the FP64 oracle (test infrastructure only).

The oracle's discovery and per-cell evaluation are independent across
discovery directions and across receiver cells, so they split over worker
processes.  Pools use the ``spawn`` start method: a forked child of a process
that has already touched the GPU would inherit a CUDA context it must not use.
"""

from __future__ import annotations

import multiprocessing as mp
import os

import numpy as np

_STATE: dict = {}


def _init(state: dict) -> None:
    _STATE.clear()
    _STATE.update(state)


def _discover_chunk(task):
    from . import geom
    from . import solve as osolve

    tx, lo, hi = task
    dirs = geom.fibonacci_directions(_STATE["rays"])[lo:hi]
    return lo, osolve.discover_directions(_STATE["arrays"], _STATE["face_group_id"], tx, dirs,
                                          max_depth=_STATE["max_depth"])


def _cells_chunk(cells):
    from . import solve as osolve

    arrays = _STATE["arrays"]
    sub = dict(arrays)
    sub["rx_pos"] = arrays["rx_pos"][cells]
    sub["rx_pol"] = arrays["rx_pol"][cells]
    out = osolve.solve(sub, discovered=_STATE["discovered"], edge_visible=_STATE["edge_visible"], **_STATE["kw"])
    return cells, out


def workers(limit: int = 32) -> int:
    return max(1, min(limit, os.cpu_count() or 1))


def discover(arrays: dict, *, max_depth: int, rays: int, processes: int | None = None) -> list | None:
    """``solve.discover`` split over directions: per transmitter the ``(rays,
    max_depth)`` group chains, or ``None`` when the exhaustive plan applies."""
    from . import solve as osolve

    fg = osolve.discovery_groups(arrays, max_depth=max_depth)
    if fg is None:
        return None
    procs = processes or workers()
    chunk = max(1024, -(-rays // (4 * procs)))
    T = arrays["tx_pos"].shape[0]
    tasks = [(t, lo, min(lo + chunk, rays)) for t in range(T) for lo in range(0, rays, chunk)]
    state = {"arrays": arrays, "face_group_id": fg, "rays": rays, "max_depth": max_depth}
    out = [np.full((rays, max(max_depth, 1)), -1, dtype=np.int64) for _ in range(T)]
    with mp.get_context("spawn").Pool(procs, initializer=_init, initargs=(state,)) as pool:
        for (t, _, _), (lo, chains) in zip(tasks, pool.imap(_discover_chunk, tasks)):
            out[t][lo:lo + chains.shape[0]] = chains
    return out


def solve_cells(arrays: dict, cells: np.ndarray, *, discovered, edge_visible, processes: int | None = None,
                **kw) -> list:
    """``solve.solve`` on the receiver subset ``cells``, split into chunks of
    cells; returns ``[(cells_chunk, result), ...]`` in order."""
    procs = processes or workers()
    chunks = [c for c in np.array_split(np.asarray(cells), max(1, min(len(cells), 4 * procs))) if len(c)]
    state = {"arrays": arrays, "discovered": discovered, "edge_visible": edge_visible, "kw": kw}
    with mp.get_context("spawn").Pool(procs, initializer=_init, initargs=(state,)) as pool:
        return list(pool.imap(_cells_chunk, chunks))
