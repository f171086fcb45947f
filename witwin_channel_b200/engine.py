"""Host orchestration of the native solve.

Two execution shapes, both on the GPU:

* **cell mode** (radiomap only): one fused ``wcb_solve`` launch chain writes
  the per-cell slot sums directly (no per-path storage);
* **row mode** (``export_paths``, ``max_paths`` or AD): the same kernels also
  emit compact path records; ``wcb_rows_select`` puts them in canonical order
  (dedup, max_paths), ``wcb_rows_evaluate`` evaluates the path-table columns
  from the frozen topology, and ``wcb_rows_accumulate`` sums each cell's rows
  in canonical order.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import Any

import torch

from . import _native
from .compiler import CompiledScene, MaterialTables

DEFAULT_DISCOVERY_RAYS = 262_144
SLOT_COUNT = 6


@dataclass
class Endpoints:
    tx_pos: torch.Tensor      # (T,3) f32
    tx_power: torch.Tensor    # (T,)
    tx_pol: torch.Tensor      # (T,3)
    rx: dict                  # compiler.receiver_setup output

    @property
    def num_tx(self) -> int:
        return int(self.tx_pos.shape[0])

    @property
    def num_rx(self) -> int:
        return int(self.rx["count"])


def make_desc(ep: Endpoints, frequencies: list[float], components: int, max_depth: int, coherent: bool,
              precision: int = _native.PRECISION_MIXED, discovery_rays: int = 0,
              stack_entries: int = 0) -> tuple[_native.SolveDesc, Any]:
    d = _native.SolveDesc()
    d.num_tx = ep.num_tx
    d.tx_pos = _native.ptr(ep.tx_pos)
    d.tx_power = _native.ptr(ep.tx_power)
    d.tx_pol = _native.ptr(ep.tx_pol)
    rx = ep.rx
    if rx["kind"] == "grid":
        g = rx["grid"]
        d.rx_kind = 1
        d.num_rx = g.count
        for k in range(3):
            d.grid_origin[k] = float(g.origin[k])
            d.grid_x_axis[k] = float(g.x_axis[k])
            d.grid_y_axis[k] = float(g.y_axis[k])
        d.grid_rows, d.grid_cols = int(g.shape[0]), int(g.shape[1])
        d.grid_spacing[0], d.grid_spacing[1] = float(g.spacing[0]), float(g.spacing[1])
        d.rx_pos = None
    else:
        d.rx_kind = 0
        d.num_rx = rx["count"]
        d.rx_pos = _native.ptr(rx["positions"]) if rx["count"] else None
    d.rx_pol = _native.ptr(rx["pol"])
    d.rx_pol_stride = rx["pol_stride"]
    freqs = (ctypes.c_double * len(frequencies))(*[float(f) for f in frequencies])
    d.num_freq = len(frequencies)
    d.frequency_hz = freqs
    d.components = components
    d.max_depth = max_depth
    d.coherent = int(bool(coherent))
    d.precision = precision
    d.discovery_rays = discovery_rays
    d.stack_entries = int(stack_entries)
    return d, freqs


def check_device_status(status: torch.Tensor) -> None:
    """Raise if a solve's device status word has a failure bit set (reads it: a sync)."""
    st = int(status.item())
    if st != 0:
        raise RuntimeError(f"native solve reported device status bits {st:#x} (bit 0: traversal stack overflow)")


def component_bits(components) -> int:
    bits = 0
    if "los" in components:
        bits |= _native.COMPONENT_LOS
    if "reflection" in components:
        bits |= _native.COMPONENT_REFLECTION
    if "diffraction" in components:
        bits |= _native.COMPONENT_DIFFRACTION
    if "transmission" in components:
        bits |= _native.COMPONENT_TRANSMISSION
    return bits


class Workspace:
    """Grow-only device scratch buffer reused across solves."""

    def __init__(self) -> None:
        self.buf: torch.Tensor | None = None

    def get(self, nbytes: int, device: torch.device) -> torch.Tensor:
        nbytes = max(int(nbytes), 256)
        if self.buf is None or self.buf.numel() < nbytes or self.buf.device != device:
            self.buf = torch.empty(nbytes, dtype=torch.uint8, device=device)
        return self.buf


_WORKSPACE = Workspace()
_SELECT_WORKSPACE = Workspace()


@dataclass
class CellOutputs:
    path_gain: torch.Tensor       # (NF,T,R)
    field: torch.Tensor           # (NF,T,R) complex
    comp_power: torch.Tensor      # (6,NF,T,R)
    comp_field: torch.Tensor      # (6,NF,T,R) complex
    diff_vec_power: torch.Tensor  # (NF,T,R)


def alloc_cells(nf: int, T: int, R: int, device: torch.device, fp64: bool = False) -> CellOutputs:
    rd = torch.float64 if fp64 else torch.float32
    cd = torch.complex128 if fp64 else torch.complex64
    return CellOutputs(
        path_gain=torch.empty((nf, T, R), dtype=rd, device=device),
        field=torch.empty((nf, T, R), dtype=cd, device=device),
        comp_power=torch.empty((SLOT_COUNT, nf, T, R), dtype=rd, device=device),
        comp_field=torch.empty((SLOT_COUNT, nf, T, R), dtype=cd, device=device),
        diff_vec_power=torch.empty((nf, T, R), dtype=rd, device=device),
    )


def run_solve(compiled: CompiledScene, ep: Endpoints, mats: MaterialTables, frequencies: list[float], *,
              components: int, max_depth: int, coherent: bool, precision: int = _native.PRECISION_MIXED,
              cells: CellOutputs | None = None, want_rows: bool = False, row_capacity: int | None = None,
              discovery_rays: int = 0, check_status: bool = True, workspace: Workspace | None = None,
              retry: bool = True, stack_entries: int = 0) -> dict:
    """One ``wcb_solve``.  With ``want_rows`` a row buffer shorter than the
    solve needs returns ``WCB_ERR_CAPACITY``; the solve then runs again with
    the reported count (``retry``) or the error is raised.  ``stack_entries``
    overrides the traversal stack size (0: the scene's BVH depth + 2)."""
    lib = _native.load()
    device = ep.tx_pos.device
    desc, keep = make_desc(ep, frequencies, components, max_depth, coherent, precision, discovery_rays, stack_entries)
    nbytes = ctypes.c_int64()
    _native.check(lib.wcb_solve_workspace_size(compiled.native.handle, ctypes.byref(desc), ctypes.byref(nbytes)),
                  "wcb_solve_workspace_size")
    ws = (workspace or _WORKSPACE).get(nbytes.value, device)
    status = torch.zeros(1, dtype=torch.int32, device=device)
    row_count = torch.zeros(1, dtype=torch.int64, device=device)
    trans_overflow = torch.zeros(1, dtype=torch.int64, device=device)
    # row capacity: the caller's, else the last count seen on this scene (with
    # headroom), else 8 records per cell; a short buffer makes the solve run again
    hint = compiled.row_count_hint
    capacity = row_capacity if row_capacity is not None else max(1024, ep.num_tx * ep.num_rx * 8, int(hint * 1.25))
    while True:
        rows = torch.empty((capacity, _native.ROW_WORDS), dtype=torch.int32, device=device) if want_rows else None
        out = _native.Outputs()
        if cells is not None:
            out.path_gain = _native.ptr(cells.path_gain)
            out.field = _native.ptr(cells.field)
            out.comp_power = _native.ptr(cells.comp_power)
            out.comp_field = _native.ptr(cells.comp_field)
            out.diff_vec_power = _native.ptr(cells.diff_vec_power)
        out.rows = _native.ptr(rows)
        out.row_capacity = capacity if want_rows else 0
        out.row_count = _native.ptr(row_count)
        out.status = _native.ptr(status)
        out.transmission_overflow = _native.ptr(trans_overflow)
        rc = lib.wcb_solve(compiled.native.handle, ctypes.byref(desc), ctypes.byref(mats_struct := mats.as_struct()),
                           ctypes.byref(out), _native.ptr(ws), ws.numel(), _native.stream_handle(device))
        del mats_struct
        if rc == _native.WCB_ERR_CAPACITY and want_rows and retry:
            capacity = int(int(row_count.item()) * 1.25) + 1024
            continue
        _native.check(rc, "wcb_solve")
        break
    if check_status:
        check_device_status(status)
    result = {"desc": desc, "keep": keep, "status": status, "workspace": ws, "transmission_overflow": trans_overflow}
    if want_rows:
        n = int(row_count.item())
        result["rows"] = rows[:n]
        compiled.row_count_hint = max(n, compiled.row_count_hint)
    return result


def select_rows(rows: torch.Tensor, width: int, max_paths: int | None, scope: str) -> torch.Tensor:
    lib = _native.load()
    n = int(rows.shape[0])
    device = rows.device
    nbytes = ctypes.c_int64()
    _native.check(lib.wcb_rows_select_workspace_size(n, ctypes.byref(nbytes)), "wcb_rows_select_workspace_size")
    ws = _SELECT_WORKSPACE.get(nbytes.value, device)
    selected = torch.empty(max(n, 1), dtype=torch.int64, device=device)
    count = ctypes.c_int64()
    mp = -1 if max_paths is None else int(max_paths)
    _native.check(
        lib.wcb_rows_select(_native.ptr(rows) if n else None, n, int(width), mp, 0 if scope == "global" else 1,
                            _native.ptr(selected), ctypes.byref(count), _native.ptr(ws), ws.numel(),
                            _native.stream_handle(device)),
        "wcb_rows_select",
    )
    return selected[: count.value]


def evaluate_rows(compiled: CompiledScene, ep: Endpoints, mats: MaterialTables, frequencies: list[float], freq_index: int,
                  rows: torch.Tensor, selected: torch.Tensor, width: int, *, components: int, max_depth: int,
                  coherent: bool) -> dict:
    lib = _native.load()
    device = rows.device
    K = int(selected.shape[0])
    W = max(int(width), 1)
    out = {
        "path_length_m": torch.zeros(K, dtype=torch.float32, device=device),
        "delay_s": torch.zeros(K, dtype=torch.float32, device=device),
        "path_gain": torch.zeros(K, dtype=torch.float32, device=device),
        "path_field": torch.zeros(K, dtype=torch.complex64, device=device),
        "coefficient": torch.zeros(K, dtype=torch.complex64, device=device),
        "field_xyz": torch.zeros((K, 3), dtype=torch.complex64, device=device),
        "field_direction": torch.zeros((K, 3), dtype=torch.float32, device=device),
        "interaction_positions": torch.zeros((K, W, 3), dtype=torch.float32, device=device),
        "interaction_normals": torch.zeros((K, W, 3), dtype=torch.float32, device=device),
        "phase_rad": torch.zeros(K, dtype=torch.float32, device=device),
    }
    if K == 0:
        return out
    desc, keep = make_desc(ep, frequencies, components, max_depth, coherent)
    rf = _native.RowFields()
    for name in out:
        setattr(rf, name, _native.ptr(out[name]))
    _native.check(
        lib.wcb_rows_evaluate(compiled.native.handle, ctypes.byref(desc), ctypes.byref(ms := mats.as_struct()), int(freq_index),
                              _native.ptr(rows), _native.ptr(selected), K, W, ctypes.byref(rf),
                              _native.stream_handle(device)),
        "wcb_rows_evaluate",
    )
    del ms, keep
    return out


def accumulate_rows(rows: torch.Tensor, selected: torch.Tensor, path_gain: torch.Tensor, path_field: torch.Tensor,
                    field_xyz: torch.Tensor | None, tx_power: torch.Tensor, T: int, R: int, coherent: bool) -> CellOutputs:
    lib = _native.load()
    device = rows.device
    cells = alloc_cells(1, T, R, device)
    out = _native.Outputs()
    out.path_gain = _native.ptr(cells.path_gain)
    out.field = _native.ptr(cells.field)
    out.comp_power = _native.ptr(cells.comp_power)
    out.comp_field = _native.ptr(cells.comp_field)
    out.diff_vec_power = _native.ptr(cells.diff_vec_power)
    K = int(selected.shape[0])
    _native.check(
        lib.wcb_rows_accumulate(_native.ptr(rows) if K else None, _native.ptr(selected) if K else None, K,
                                _native.ptr(path_gain) if K else None, _native.ptr(path_field) if K else None,
                                _native.ptr(field_xyz) if (K and field_xyz is not None) else None, _native.ptr(tx_power), T, R,
                                int(bool(coherent)), ctypes.byref(out), _native.stream_handle(device)),
        "wcb_rows_accumulate",
    )
    return cells


def decode_rows(rows: torch.Tensor, selected: torch.Tensor) -> dict:
    """Integer columns of the selected path records (canonical order), in one
    pass over the records (``wcb_rows_decode``)."""

    device = rows.device
    K = int(selected.shape[0])
    out = {name: torch.empty(K, dtype=torch.int32, device=device)
           for name in ("tx_id", "rx_id", "component_id", "depth", "edge_id")}
    out["seq"] = torch.empty((K, 5), dtype=torch.int32, device=device)
    out["length"] = torch.empty(K, dtype=torch.float32, device=device)
    if K:
        sel = selected.to(torch.int64).contiguous()
        _native.check(_native.load().wcb_rows_decode(
            _native.ptr(rows), _native.ptr(sel), K, _native.ptr(out["tx_id"]), _native.ptr(out["rx_id"]),
            _native.ptr(out["component_id"]), _native.ptr(out["depth"]), _native.ptr(out["seq"]),
            _native.ptr(out["edge_id"]), _native.ptr(out["length"]), _native.stream_handle(device)), "wcb_rows_decode")
    return out
