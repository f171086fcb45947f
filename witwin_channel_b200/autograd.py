"""Reverse-mode differentiation of the deterministic solve (``ad_mode="vjp"``).

Mirrors the reference's deterministic AD contract (``deterministic.py`` with
``ad_mode="vjp"``; ``kernels/deterministic.py:186-367`` for the accumulation,
``kernels/fields.py:1087-2140`` for the fields, ``propagation/geometry.py:
214-286`` for the frozen-winner geometry): the forward solve runs once in
row mode and freezes every path's interaction sequence; the backward pass

1. maps the cotangents of the cell outputs to per-path cotangents of gain and
   field with the adjoint of the flat accumulation (``wcb_accumulate_flat_backward``),
2. re-evaluates every frozen path from the raw scene values in FP64 dual
   numbers and reduces the per-parameter contributions deterministically
   (``wcb_rows_vjp``),

giving gradients for mesh vertices, per-material eps_r / sigma_e (and layer
values), the carrier frequency, Tx positions and point-receiver positions.
Material values that depend on the frequency or on other tensors chain
through torch autograd as usual.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import Any

import torch

from . import _native, engine
from .compiler import compile_scene
from .kernels import ACCUM_FIELDS, _forward, deterministic_accumulate_flat_backward

WANT_TX, WANT_RX, WANT_FREQ, WANT_VERTICES, WANT_MATERIALS = 1, 2, 4, 8, 16


@dataclass
class _State:
    compiled: Any
    ep: engine.Endpoints
    mats: Any
    frequency: float
    components: int
    max_depth: int
    coherent: bool
    rows: torch.Tensor
    selected: torch.Tensor
    flat: dict          # valid, tx, rx, cid (int32), per-row gain/field f64
    saved64: dict       # FP64 accumulation outputs (linearisation point)
    outputs32: dict     # FP32 accumulation outputs (the returned values)
    layer_counts: list
    vertex_mask: torch.Tensor | None = None


def _as_f64(x, device) -> torch.Tensor:
    if isinstance(x, torch.Tensor):
        return x.to(device=device, dtype=torch.float64).reshape(())
    return torch.tensor(float(x), dtype=torch.float64, device=device)


def _differentiable_inputs(scene, compiled, freq_t: torch.Tensor, device) -> dict:
    verts = [st.vertices.reshape(-1, 3).to(device=device, dtype=torch.float64) for st in scene.structures]
    V = torch.cat(verts) if verts else torch.zeros((0, 3), dtype=torch.float64, device=device)
    mv = compiled.material_values(freq_t, keep_graph=True)
    eps = torch.stack([_as_f64(x, device) for x in mv["eps_r"]]) if mv["eps_r"] else torch.zeros(0, dtype=torch.float64, device=device)
    sig = torch.stack([_as_f64(x, device) for x in mv["sigma_e"]]) if mv["sigma_e"] else torch.zeros(0, dtype=torch.float64, device=device)
    flat = [row for rows in mv["layers"] for row in rows]
    leps = torch.stack([_as_f64(r[1], device) for r in flat]) if flat else torch.zeros(0, dtype=torch.float64, device=device)
    lsig = torch.stack([_as_f64(r[2], device) for r in flat]) if flat else torch.zeros(0, dtype=torch.float64, device=device)
    txs = scene.transmitters
    tx = torch.stack([t.position.reshape(3).to(device=device, dtype=torch.float64) for t in txs]) if txs else \
        torch.zeros((0, 3), dtype=torch.float64, device=device)
    rxs = scene.receivers
    if len(rxs) == 1 and hasattr(rxs[0], "shape") and hasattr(rxs[0], "spacing"):
        rx = torch.zeros((0, 3), dtype=torch.float64, device=device)
    else:
        rx = torch.stack([r.position.reshape(3).to(device=device, dtype=torch.float64) for r in rxs]) if rxs else \
            torch.zeros((0, 3), dtype=torch.float64, device=device)
    # differentiate only the vertices of structures whose vertex tensor takes gradients
    mask = torch.cat([torch.full((st.vertices.reshape(-1, 3).shape[0],), int(bool(st.vertices.requires_grad)),
                                 dtype=torch.uint8) for st in scene.structures]).to(device) if verts else None
    return {"vertices": V, "vertex_mask": mask, "eps_r": eps, "sigma_e": sig, "layer_eps_r": leps, "layer_sigma_e": lsig,
            "frequency": freq_t.reshape(()).to(dtype=torch.float64), "tx": tx, "rx": rx,
            "layer_counts": [len(rows) for rows in mv["layers"]]}


def rows_vjp(state: _State, g_gain: torch.Tensor | None, g_re: torch.Tensor | None, g_im: torch.Tensor | None,
             want: int, row_field: torch.Tensor | None = None,
             vertex_mask: torch.Tensor | None = None) -> tuple[torch.Tensor, list[int]]:
    """Dense FP64 gradient over the native parameter layout (see ``wcb_rows_vjp``)."""
    lib = _native.load()
    device = state.rows.device
    desc, keep = engine.make_desc(state.ep, [state.frequency], state.components, state.max_depth, state.coherent)
    ms = state.mats.as_struct()
    layout = (ctypes.c_int64 * 9)()
    _native.check(lib.wcb_rows_vjp_layout(state.compiled.native.handle, ctypes.byref(desc), ctypes.byref(ms), layout),
                  "wcb_rows_vjp_layout")
    total = int(layout[8])
    K = int(state.selected.shape[0])
    nbytes = ctypes.c_int64()
    max_layers = max(state.layer_counts) if state.layer_counts else 1
    _native.check(lib.wcb_rows_vjp_workspace_size(K, int(state.max_depth), int(max_layers), ctypes.byref(nbytes)),
                  "wcb_rows_vjp_workspace_size")
    ws = torch.empty(max(nbytes.value, 256), dtype=torch.uint8, device=device)
    grad = torch.zeros(max(total, 1), dtype=torch.float64, device=device)
    _native.check(
        lib.wcb_rows_vjp(state.compiled.native.handle, ctypes.byref(desc), ctypes.byref(ms), 0,
                         _native.ptr(state.rows) if K else None, _native.ptr(state.selected) if K else None, K,
                         _native.ptr(g_gain), _native.ptr(g_re), _native.ptr(g_im), int(want),
                         _native.ptr(vertex_mask), _native.ptr(grad),
                         grad.numel(), _native.ptr(row_field), _native.ptr(ws), ws.numel(),
                         _native.stream_handle(device)),
        "wcb_rows_vjp",
    )
    del keep
    return grad[:total], [int(layout[i]) for i in range(9)]


class _SolveFunction(torch.autograd.Function):
    """Cell outputs of the frozen-topology solve as a function of the scene values."""

    @staticmethod
    def forward(ctx, state: _State, vertices, eps_r, sigma_e, layer_eps_r, layer_sigma_e, frequency, tx, rx):
        ctx.state = state
        ctx.shapes = [tuple(t.shape) for t in (vertices, eps_r, sigma_e, layer_eps_r, layer_sigma_e, frequency, tx, rx)]
        o = state.outputs32
        return tuple(o[k].clone() for k in ACCUM_FIELDS)

    @staticmethod
    def backward(ctx, *grads):
        state: _State = ctx.state
        needs = ctx.needs_input_grad
        want = 0
        if needs[1]:
            want |= WANT_VERTICES
        if any(needs[2:6]):
            want |= WANT_MATERIALS
        if needs[6]:
            want |= WANT_FREQ
        if needs[7]:
            want |= WANT_TX
        if needs[8]:
            want |= WANT_RX
        none = (None,) * 9
        if want == 0 or all(g is None for g in grads):
            return none
        T, R = state.ep.num_tx, state.ep.num_rx
        g64 = [None if g is None else g.to(torch.float64).contiguous() for g in grads]
        s = state.saved64
        f = state.flat
        per_row = deterministic_accumulate_flat_backward(
            f["valid"], f["tx"], f["rx"], f["cid"], s["component_field_real"], s["component_field_imag"],
            s["field_total_real"], s["field_total_imag"], s["power_total"], grad_power_total=g64[0],
            grad_field_total_real=g64[1], grad_field_total_imag=g64[2], grad_component_power=g64[3],
            grad_component_field_real=g64[4], grad_component_field_imag=g64[5], num_tx=T, num_rx=R,
            coherent=state.coherent)
        grad, lay = rows_vjp(state, per_row["grad_path_gain"], per_row["grad_field_real"],
                             per_row["grad_field_imag"], want, vertex_mask=state.vertex_mask)
        parts = [grad[lay[i]:lay[i + 1]] for i in range(8)]
        out = [None]
        for i, shape in enumerate(ctx.shapes):
            out.append(parts[i].reshape(shape) if needs[i + 1] else None)
        return tuple(out)


def solve_vjp(scene: Any, config, reference_frequency_hz):
    """The deterministic solve with ``ad_mode="vjp"``: same outputs as the
    row-mode forward, differentiable in the scene values."""
    from .deterministic import (
        _BASE_COMPONENTS,
        _OPTIONAL_COMPONENTS,
        _SLOTS,
        Result,
        _endpoints,
        _layout,
        _metadata,
        _path_table,
    )

    if not config.coherent and "diffraction" in config.components:
        raise NotImplementedError("ad_mode='vjp' with incoherent accumulation and diffraction is not provided")
    device = torch.device("cuda", torch.cuda.current_device())
    if isinstance(reference_frequency_hz, torch.Tensor):
        freq_t = reference_frequency_hz.to(device=device)
    else:
        freq_t = torch.tensor(float(reference_frequency_hz), dtype=torch.float64, device=device)
    frequency = float(freq_t.detach())
    compiled = compile_scene(scene, device)
    ep = _endpoints(scene, device)
    mats = compiled.material_tables([frequency], device)
    bits = engine.component_bits(config.components)
    T, R = ep.num_tx, ep.num_rx
    launches0 = _native.launch_count()
    res = engine.run_solve(compiled, ep, mats, [frequency], components=bits, max_depth=config.max_depth,
                           coherent=config.coherent, want_rows=True)
    rows = res["rows"]
    width = max(int(config.max_depth), 0)
    selected = engine.select_rows(rows, width, config.max_paths, config.max_paths_scope)
    ev = engine.evaluate_rows(compiled, ep, mats, [frequency], 0, rows, selected, width, components=bits,
                              max_depth=config.max_depth, coherent=config.coherent)
    dec = engine.decode_rows(rows, selected)
    K = int(selected.shape[0])
    flat = {"valid": torch.ones(K, dtype=torch.bool, device=device), "tx": dec["tx_id"], "rx": dec["rx_id"],
            "cid": dec["component_id"].contiguous()}
    pf = ev["path_field"]
    g32, r32, i32 = ev["path_gain"].contiguous(), pf.real.contiguous(), pf.imag.contiguous()
    outputs32 = _forward(flat["valid"], flat["tx"], flat["rx"], flat["cid"], g32, r32, i32, T, R, config.coherent, 0)
    saved64 = _forward(flat["valid"], flat["tx"], flat["rx"], flat["cid"], g32.double(), r32.double(), i32.double(),
                       T, R, config.coherent, 0)
    inputs = _differentiable_inputs(scene, compiled, freq_t, device)
    state = _State(compiled=compiled, ep=ep, mats=mats, frequency=frequency, components=bits,
                   max_depth=config.max_depth, coherent=config.coherent, rows=rows, selected=selected, flat=flat,
                   saved64=saved64, outputs32=outputs32, layer_counts=inputs["layer_counts"],
                   vertex_mask=inputs["vertex_mask"])
    pt, ftr, fti, cp, cfr, cfi = _SolveFunction.apply(
        state, inputs["vertices"], inputs["eps_r"], inputs["sigma_e"], inputs["layer_eps_r"], inputs["layer_sigma_e"],
        inputs["frequency"], inputs["tx"], inputs["rx"])
    rx = ep.rx
    names = _BASE_COMPONENTS + tuple(n for n in _OPTIONAL_COMPONENTS if n in config.components)
    comp_power = {n: _layout(cp[_SLOTS[n]], rx) for n in names}
    comp_fields = {n: _layout(torch.complex(cfr[_SLOTS[n]], cfi[_SLOTS[n]]), rx) for n in names} \
        if config.return_field else {n: torch.empty((0,), dtype=torch.complex64, device=device) for n in names}
    counts = {name: int((dec["component_id"] == c).sum().item())
              for name, c in (("los", 0), ("reflection", 1), ("diffraction", 2), ("transmission", 5))}
    paths = _path_table(dec, ev, width, compiled, config.return_field) if config.export_paths else None
    meta = _metadata(config, counts, K, _native.launch_count() - launches0, {"ad": "fixed-topology vjp"})
    return Result(
        path_gain=_layout(pt, rx),
        field=_layout(torch.complex(ftr, fti), rx) if config.return_field
        else torch.empty((0,), dtype=torch.complex64, device=device),
        component_power=comp_power,
        component_fields=comp_fields,
        paths=paths,
        metadata=meta,
        diagnostics=None,
    )
