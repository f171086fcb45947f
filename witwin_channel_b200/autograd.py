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

Forward mode (``ad_mode="jvp"``; the reference runs its dual companions
inside the forward, ``deterministic.py:733-742``) uses the same frozen
forward: when the scene values are ``torch.autograd.forward_ad`` dual
tensors, the autograd Function's ``jvp`` packs their tangents into the same
parameter layout, re-evaluates every record once with one FP64 dual lane
seeded by it (``wcb_rows_jvp``) and scatters the records' field and gain
tangents to the cells with the accumulation's pushforward.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass, replace
from typing import Any

import numpy as np
import torch

from . import _native, engine
from .compiler import compile_scene
from .kernels import ACCUM_FIELDS, _forward, deterministic_accumulate_flat_backward, deterministic_accumulate_flat_jvp

WANT_TX, WANT_RX, WANT_FREQ, WANT_VERTICES, WANT_MATERIALS = 1, 2, 4, 8, 16


@dataclass
class _State:
    compiled: Any
    ep: engine.Endpoints
    mats: Any
    frequencies: list       # solve frequencies (Hz)
    components: int
    max_depth: int
    coherent: bool
    rows: torch.Tensor
    selected: torch.Tensor
    flat: dict              # valid, tx, rx, cid (int32) of the selected records
    saved64: list           # per frequency: FP64 accumulation outputs (linearisation point), made on first use
    outputs32: list         # per frequency: FP32 accumulation outputs (the returned values)
    layer_counts: list
    vertex_mask: torch.Tensor | None = None
    param_total: int = 0    # length of the native parameter layout
    order: Any = None       # execution order of the records (wcb_rows_order), made on first use
    comp_counts: Any = None  # its four group sizes (ctypes int64 array)


def _record_order(state: _State):
    """The records' execution order for the derivative kernels (grouped by
    component, depth and diffraction edge), computed once per record set and
    shared by every frequency's linearisation and VJP."""
    if state.order is None:
        lib = _native.load()
        device = state.rows.device
        K = int(state.selected.shape[0])
        order = torch.zeros(max(K, 1), dtype=torch.int32, device=device)
        counts = (ctypes.c_int64 * 4)()
        nbytes = ctypes.c_int64()
        _native.check(lib.wcb_rows_order_workspace_size(K, ctypes.byref(nbytes)), "wcb_rows_order_workspace_size")
        ws = _ORDER_WORKSPACE.get(nbytes.value, device)
        _native.check(lib.wcb_rows_order(state.compiled.native.handle, _native.ptr(state.rows) if K else None,
                                         _native.ptr(state.selected) if K else None, K, _native.ptr(order), counts,
                                         _native.ptr(ws), ws.numel(), _native.stream_handle(device)),
                      "wcb_rows_order")
        state.order, state.comp_counts = order, counts
    return state.order, state.comp_counts


def _linearisation(state: _State, fi: int) -> dict:
    """FP64 cell accumulation of the records' FP64 re-evaluated fields at
    frequency ``fi``: the point the derivatives of |sum field|^2 are taken at.
    (The FP32 forward values would do for most losses, but a loss whose cell
    terms cancel amplifies their rounding into the gradient.)  Computed once
    per frequency by one plain FP64 ``wcb_rows_jvp`` pass (no tangent) and cached."""
    if state.saved64[fi] is None:
        # every frequency in one pass (diffraction records share their UTD
        # geometry across the frequencies), each accumulated in FP64
        fields = rows_field64_all(state) if len(state.frequencies) > 1 else rows_jvp(state, fi, None)[0][None]
        f_ = state.flat
        for fj in range(len(state.frequencies)):
            if state.saved64[fj] is not None:
                continue
            field = fields[fj]
            re, im = field[:, 0].contiguous(), field[:, 1].contiguous()
            gain = (re * re + im * im).contiguous()
            state.saved64[fj] = _forward(f_["valid"], f_["tx"], f_["rx"], f_["cid"], gain, re, im, state.ep.num_tx,
                                         state.ep.num_rx, state.coherent, 0)
    return state.saved64[fi]


def rows_field64_all(state: _State) -> torch.Tensor:
    """The records' FP64 path fields at every solve frequency, (NF, K, 2), in
    one ``wcb_rows_jvp`` call (``freq_index=-1``)."""
    lib = _native.load()
    device = state.rows.device
    desc, keep = engine.make_desc(state.ep, state.frequencies, state.components, state.max_depth, state.coherent)
    ms = state.mats.as_struct()
    K = int(state.selected.shape[0])
    NF = len(state.frequencies)
    field = torch.zeros((NF, max(K, 1), 2), dtype=torch.float64, device=device)
    order, counts = _record_order(state)
    _native.check(
        lib.wcb_rows_jvp(state.compiled.native.handle, ctypes.byref(desc), ctypes.byref(ms), -1,
                         _native.ptr(state.rows) if K else None, _native.ptr(state.selected) if K else None, K,
                         None, 0, _native.ptr(field), None, _native.ptr(order), counts,
                         _native.stream_handle(device)),
        "wcb_rows_jvp",
    )
    del keep
    return field[:, :K]


def _as_f64(x, device) -> torch.Tensor:
    if isinstance(x, torch.Tensor):
        return x.to(device=device, dtype=torch.float64).reshape(())
    return torch.tensor(float(x), dtype=torch.float64, device=device)


def _stack0(values: list, device) -> torch.Tensor:
    return torch.stack(values) if values else torch.zeros(0, dtype=torch.float64, device=device)


def _differentiable_inputs(scene, compiled, freqs_t: torch.Tensor, device) -> dict:
    """The scene values the solve is differentiated in: vertices (V,3), per
    frequency material and layer eps_r / sigma_e (NF,M) and (NF,L), the
    frequencies (NF,), Tx positions (T,3) and point-receiver positions (R,3)."""
    verts = [st.vertices.reshape(-1, 3).to(device=device, dtype=torch.float64) for st in scene.structures]
    V = torch.cat(verts) if verts else torch.zeros((0, 3), dtype=torch.float64, device=device)
    eps, sig, leps, lsig = [], [], [], []
    layer_counts = []
    for f in range(freqs_t.shape[0]):
        mv = compiled.material_values(freqs_t[f], keep_graph=True)
        eps.append(_stack0([_as_f64(x, device) for x in mv["eps_r"]], device))
        sig.append(_stack0([_as_f64(x, device) for x in mv["sigma_e"]], device))
        flat = [row for rows in mv["layers"] for row in rows]
        leps.append(_stack0([_as_f64(r[1], device) for r in flat], device))
        lsig.append(_stack0([_as_f64(r[2], device) for r in flat], device))
        layer_counts = [len(rows) for rows in mv["layers"]]
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
    return {"vertices": V, "vertex_mask": mask, "eps_r": torch.stack(eps), "sigma_e": torch.stack(sig),
            "layer_eps_r": torch.stack(leps), "layer_sigma_e": torch.stack(lsig),
            "frequency": freqs_t.to(dtype=torch.float64), "tx": tx, "rx": rx, "layer_counts": layer_counts}


def rows_vjp(state: _State, freq_index: int, g_gain: torch.Tensor | None, g_re: torch.Tensor | None,
             g_im: torch.Tensor | None, want: int, row_field: torch.Tensor | None = None,
             vertex_mask: torch.Tensor | None = None) -> tuple[torch.Tensor, list[int]]:
    """Dense FP64 gradient over the native parameter layout (see ``wcb_rows_vjp``)
    for the records' fields at frequency ``freq_index``."""
    lib = _native.load()
    device = state.rows.device
    desc, keep = engine.make_desc(state.ep, state.frequencies, state.components, state.max_depth, state.coherent)
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
    ws = _VJP_WORKSPACE.get(nbytes.value, device)
    order, counts = _record_order(state)
    grad = torch.zeros(max(total, 1), dtype=torch.float64, device=device)
    _native.check(
        lib.wcb_rows_vjp(state.compiled.native.handle, ctypes.byref(desc), ctypes.byref(ms), int(freq_index),
                         _native.ptr(state.rows) if K else None, _native.ptr(state.selected) if K else None, K,
                         _native.ptr(g_gain), _native.ptr(g_re), _native.ptr(g_im), int(want),
                         _native.ptr(vertex_mask), _native.ptr(grad),
                         grad.numel(), _native.ptr(row_field), _native.ptr(order), counts, _native.ptr(ws),
                         ws.numel(), _native.stream_handle(device)),
        "wcb_rows_vjp",
    )
    del keep
    return grad[:total], [int(layout[i]) for i in range(9)]


_VJP_WORKSPACE = engine.Workspace()
_ORDER_WORKSPACE = engine.Workspace()


def _param_total(compiled, ep, mats, frequencies, bits, config) -> int:
    lib = _native.load()
    desc, keep = engine.make_desc(ep, frequencies, bits, config.max_depth, config.coherent)
    ms = mats.as_struct()
    layout = (ctypes.c_int64 * 9)()
    _native.check(lib.wcb_rows_vjp_layout(compiled.native.handle, ctypes.byref(desc), ctypes.byref(ms), layout),
                  "wcb_rows_vjp_layout")
    del keep
    return int(layout[8])


def rows_jvp(state: _State, freq_index: int, tangent: torch.Tensor | None) -> tuple[torch.Tensor, torch.Tensor]:
    """Per-record FP64 path field and its directional derivative ((K,2) each)
    for a dense FP64 tangent over the native parameter layout (``wcb_rows_jvp``);
    with ``tangent`` None the fields alone (the derivative is returned as zeros)."""
    lib = _native.load()
    device = state.rows.device
    desc, keep = engine.make_desc(state.ep, state.frequencies, state.components, state.max_depth, state.coherent)
    ms = state.mats.as_struct()
    K = int(state.selected.shape[0])
    field = torch.zeros((max(K, 1), 2), dtype=torch.float64, device=device)
    dfield = torch.zeros((max(K, 1), 2), dtype=torch.float64, device=device)
    if tangent is not None:
        tangent = tangent.to(device=device, dtype=torch.float64).contiguous()
    order, counts = _record_order(state)
    _native.check(
        lib.wcb_rows_jvp(state.compiled.native.handle, ctypes.byref(desc), ctypes.byref(ms), int(freq_index),
                         _native.ptr(state.rows) if K else None, _native.ptr(state.selected) if K else None, K,
                         _native.ptr(tangent), 0 if tangent is None else tangent.numel(), _native.ptr(field),
                         None if tangent is None else _native.ptr(dfield), _native.ptr(order), counts,
                         _native.stream_handle(device)),
        "wcb_rows_jvp",
    )
    del keep
    return field[:K], dfield[:K]


class _SolveFunction(torch.autograd.Function):
    """Cell outputs (NF,T,R) / (NF,6,T,R) of the frozen-topology solve as a
    function of the scene values."""

    @staticmethod
    def forward(ctx, state: _State, vertices, eps_r, sigma_e, layer_eps_r, layer_sigma_e, frequency, tx, rx):
        ctx.state = state
        ctx.shapes = [tuple(t.shape) for t in (vertices, eps_r, sigma_e, layer_eps_r, layer_sigma_e, frequency, tx, rx)]
        return tuple(torch.stack([o[k] for o in state.outputs32]) for k in ACCUM_FIELDS)

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
        dev = state.rows.device
        acc = [torch.zeros(shape, dtype=torch.float64, device=dev) for shape in ctx.shapes]
        f_ = state.flat
        for fi in range(len(state.frequencies)):
            gf = [None if g is None else g[fi].to(torch.float64).contiguous() for g in grads]
            if all(g is None for g in gf):
                continue
            s = _linearisation(state, fi)
            per_row = deterministic_accumulate_flat_backward(
                f_["valid"], f_["tx"], f_["rx"], f_["cid"], s["component_field_real"], s["component_field_imag"],
                s["field_total_real"], s["field_total_imag"], s["power_total"], grad_power_total=gf[0],
                grad_field_total_real=gf[1], grad_field_total_imag=gf[2], grad_component_power=gf[3],
                grad_component_field_real=gf[4], grad_component_field_imag=gf[5], num_tx=T, num_rx=R,
                coherent=state.coherent)
            grad, lay = rows_vjp(state, fi, per_row["grad_path_gain"], per_row["grad_field_real"],
                                 per_row["grad_field_imag"], want, vertex_mask=state.vertex_mask)
            parts = [grad[lay[i]:lay[i + 1]] for i in range(8)]
            acc[0] += parts[0].reshape(ctx.shapes[0])
            for i in (1, 2, 3, 4):
                acc[i][fi] += parts[i]
            acc[5][fi] += parts[5][0] if parts[5].numel() else 0.0
            acc[6] += parts[6].reshape(ctx.shapes[6])
            acc[7] += parts[7].reshape(ctx.shapes[7])
        return (None,) + tuple(a if needs[i + 1] else None for i, a in enumerate(acc))

    @staticmethod
    def jvp(ctx, _t_state, *tangents):
        """Forward mode: the inputs' tangents, laid out like the VJP gradient,
        seed one FP64 dual lane per record (``wcb_rows_jvp``); the records'
        field and gain tangents are scattered to the cells by the flat
        accumulation's pushforward."""
        state: _State = ctx.state
        if all(t is None for t in tangents):
            return (None,) * len(ACCUM_FIELDS)
        dev = state.rows.device
        T, R = state.ep.num_tx, state.ep.num_rx
        shapes = ctx.shapes

        def part(i, fi=None):
            shape = shapes[i] if fi is None else shapes[i][1:]
            t = tangents[i]
            if t is None:
                return torch.zeros(int(np.prod(shape)), dtype=torch.float64, device=dev)
            t = t if fi is None else t[fi]
            return t.reshape(-1).to(device=dev, dtype=torch.float64)

        f_ = state.flat
        per_freq = []
        for fi in range(len(state.frequencies)):
            tf = tangents[5]
            t_freq = torch.zeros(1, dtype=torch.float64, device=dev) if tf is None else \
                tf[fi:fi + 1].to(device=dev, dtype=torch.float64)
            tangent = torch.cat([part(0), part(1, fi), part(2, fi), part(3, fi), part(4, fi), t_freq, part(6),
                                 part(7)])
            field, dfield = rows_jvp(state, fi, tangent)
            t_re, t_im = dfield[:, 0].contiguous(), dfield[:, 1].contiguous()
            t_gain = (2.0 * (field[:, 0] * t_re + field[:, 1] * t_im)).contiguous()
            s = _linearisation(state, fi)
            out = deterministic_accumulate_flat_jvp(
                f_["valid"], f_["tx"], f_["rx"], f_["cid"], s["component_field_real"], s["component_field_imag"],
                s["power_total"], tangent_path_gain=t_gain, tangent_field_real=t_re, tangent_field_imag=t_im,
                num_tx=T, num_rx=R, coherent=state.coherent)
            per_freq.append(out)
        return tuple(torch.stack([o[k] for o in per_freq]).to(torch.float32) for k in ACCUM_FIELDS)


class RowFieldFunction(torch.autograd.Function):
    """Per-row powered path fields (K,) complex as a function of the Tx and
    point-Rx positions, the scene's vertices and material values and the
    frequency, with the rows' records frozen (one frequency: ``state``'s
    first).  ``live`` (int64) are the rows that carry derivatives, one for one
    with ``state.selected``; the others are constants (replayed rows that
    stopped existing).  Backward runs the native fixed-topology VJP
    (``wcb_rows_vjp``: FP64 re-evaluation of every live row, reverse mode for
    diffraction), forward mode the native JVP (``wcb_rows_jvp``).  Used by the
    consumer's scalar coefficient, the deterministic path table and the path
    solver's coefficients."""

    @staticmethod
    def forward(ctx, state, coefficient, live, src, snk, vertices, eps_r, sigma_e, layer_eps_r, layer_sigma_e,
                frequency):
        ctx.state = state
        ctx.live = live
        ctx.count = int(coefficient.shape[0])
        ctx.shapes = [tuple(t.shape) for t in (vertices, eps_r, sigma_e, layer_eps_r, layer_sigma_e, frequency, src,
                                               snk)]
        ctx.dtypes = [t.dtype for t in (src, snk)]
        return coefficient.clone()

    @staticmethod
    def backward(ctx, grad):
        state = ctx.state
        needs = ctx.needs_input_grad
        want = 0
        if needs[5]:
            want |= WANT_VERTICES
        if any(needs[6:10]):
            want |= WANT_MATERIALS
        if needs[10]:
            want |= WANT_FREQ
        if needs[3]:
            want |= WANT_TX
        if needs[4]:
            want |= WANT_RX
        none = (None,) * 11
        if want == 0 or grad is None or int(state.selected.shape[0]) == 0:
            return none
        g = grad.index_select(0, ctx.live)
        g_re = g.real.to(torch.float64).contiguous()
        g_im = g.imag.to(torch.float64).contiguous()
        dense, lay = rows_vjp(state, 0, None, g_re, g_im, want, vertex_mask=state.vertex_mask)
        parts = [dense[lay[i]:lay[i + 1]] for i in range(8)]
        s = ctx.shapes
        vert = parts[0].reshape(s[0])
        mats = [parts[i].reshape(s[i]) for i in (1, 2, 3, 4)]
        freq = parts[5].reshape(s[5]) if parts[5].numel() else torch.zeros(s[5], dtype=torch.float64,
                                                                            device=dense.device)
        src = parts[6].reshape(s[6]).to(ctx.dtypes[0])
        snk = parts[7].reshape(s[7]).to(ctx.dtypes[1])
        grads = (src, snk, vert, *mats, freq)
        return (None, None, None) + tuple(x if needs[i + 3] else None for i, x in enumerate(grads))

    @staticmethod
    def jvp(ctx, _t_state, _t_coefficient, _t_live, t_src, t_snk, t_vertices, t_eps, t_sig, t_leps, t_lsig, t_freq):
        state = ctx.state
        dev = state.rows.device
        s = ctx.shapes

        def flat(t, shape):
            if t is None:
                return torch.zeros(int(np.prod(shape)), dtype=torch.float64, device=dev)
            return t.reshape(-1).to(device=dev, dtype=torch.float64)

        out = torch.zeros(ctx.count, dtype=torch.complex64, device=dev)
        if int(state.selected.shape[0]) == 0:
            return out
        tangent = torch.cat([flat(t_vertices, s[0]), flat(t_eps, s[1]), flat(t_sig, s[2]), flat(t_leps, s[3]),
                             flat(t_lsig, s[4]), flat(t_freq, s[5]), flat(t_src, s[6]), flat(t_snk, s[7])])
        _field, dfield = rows_jvp(state, 0, tangent)
        out.index_copy_(0, ctx.live, torch.complex(dfield[:, 0], dfield[:, 1]).to(torch.complex64))
        return out



def differentiable_row_fields(scene: Any, compiled: Any, ep: engine.Endpoints, mats: Any, frequency: float,
                              frequency_input: Any, components: int, max_depth: int, rows: torch.Tensor,
                              selected: torch.Tensor, field: torch.Tensor, tx: torch.Tensor | None = None,
                              rx: torch.Tensor | None = None) -> torch.Tensor:
    """``field`` ((K,) complex64, the records ``selected`` of ``rows`` at
    ``frequency``) made differentiable in the scene's vertices and material
    values, the frequency (when ``frequency_input`` is a tensor) and the Tx /
    point-Rx positions (the scene's endpoints, or ``tx`` / ``rx`` when given),
    through :class:`RowFieldFunction`."""
    device = field.device
    if isinstance(frequency_input, torch.Tensor):
        freqs_t = frequency_input.reshape(1).to(device=device, dtype=torch.float64)
    else:
        freqs_t = torch.tensor([float(frequency)], dtype=torch.float64, device=device)
    inputs = _differentiable_inputs(scene, compiled, freqs_t, device)
    state = _State(compiled=compiled, ep=ep, mats=mats, frequencies=[float(frequency)], components=components,
                   max_depth=max_depth, coherent=True, rows=rows, selected=selected, flat={}, saved64=[None],
                   outputs32=[], layer_counts=inputs["layer_counts"], vertex_mask=inputs["vertex_mask"])
    live = torch.arange(int(selected.shape[0]), device=device, dtype=torch.int64)
    return RowFieldFunction.apply(state, field, live, inputs["tx"] if tx is None else tx,
                                  inputs["rx"] if rx is None else rx, inputs["vertices"], inputs["eps_r"],
                                  inputs["sigma_e"], inputs["layer_eps_r"], inputs["layer_sigma_e"],
                                  inputs["frequency"])


def unit_coefficient(coefficient: torch.Tensor, path_field: torch.Tensor, tx_power: torch.Tensor) -> torch.Tensor:
    """The unit-excitation coefficients with the derivatives of the powered
    ``path_field`` divided by sqrt(power) (rows of a non-positive power carry
    none); the values are ``coefficient``'s."""
    amp = torch.sqrt(torch.clamp(tx_power.to(torch.float32), min=0.0))
    inv = torch.where(amp > 0, 1.0 / torch.clamp(amp, min=1e-30), torch.zeros_like(amp))
    return coefficient + (path_field - path_field.detach()) * inv


def vjp_forward(scene: Any, config, frequencies_hz, evaluate_rows: bool | None = None,
                precision: str = "mixed") -> dict:
    """Row-mode forward at every frequency (geometry and records frozen once)
    with autograd-connected cell outputs: ``path_gain``/``field_total_*`` (NF,T,R),
    ``component_*`` (NF,6,T,R) in the flat (tx, rx) order, plus the records.
    ``evaluate_rows`` (default: ``config.export_paths``) adds the FP32 row
    evaluations a path table is built from.  ``precision="fp64"`` runs the
    record search (traversal, candidate tests) in FP64 as well; the values and
    derivatives are FP64 in both forms."""
    if not config.coherent and "diffraction" in config.components:
        raise NotImplementedError("ad_mode='vjp' with incoherent accumulation and diffraction is not provided")
    device = torch.device("cuda", torch.cuda.current_device())
    if isinstance(frequencies_hz, torch.Tensor):
        freqs_t = frequencies_hz.to(device=device).reshape(-1)
    else:
        freqs_t = torch.tensor([float(f) for f in frequencies_hz], dtype=torch.float64, device=device)
    frequencies = [float(f) for f in freqs_t.detach().cpu()]
    compiled = compile_scene(scene, device)
    from .deterministic import _endpoints

    ep = _endpoints(scene, device)
    mats = compiled.material_tables(frequencies, device)
    bits = engine.component_bits(config.components)
    T, R = ep.num_tx, ep.num_rx
    prec = _native.PRECISION_FP64 if precision == "fp64" else _native.PRECISION_MIXED
    res = engine.run_solve(compiled, ep, mats, frequencies, components=bits, max_depth=config.max_depth,
                           coherent=config.coherent, want_rows=True, precision=prec)
    rows = res["rows"]
    width = max(int(config.max_depth), 0)
    selected = engine.select_rows(rows, width, config.max_paths, config.max_paths_scope)
    dec = engine.decode_rows(rows, selected)
    K = int(selected.shape[0])
    flat = {"valid": torch.ones(K, dtype=torch.bool, device=device), "tx": dec["tx_id"], "rx": dec["rx_id"],
            "cid": dec["component_id"].contiguous()}
    if evaluate_rows is None:
        evaluate_rows = bool(config.export_paths)
    evs = [engine.evaluate_rows(compiled, ep, mats, frequencies, fi, rows, selected, width, components=bits,
                                max_depth=config.max_depth, coherent=config.coherent)
           for fi in range(len(frequencies))] if evaluate_rows else None
    inputs = _differentiable_inputs(scene, compiled, freqs_t, device)
    state = _State(compiled=compiled, ep=ep, mats=mats, frequencies=frequencies, components=bits,
                   max_depth=config.max_depth, coherent=config.coherent, rows=rows, selected=selected, flat=flat,
                   saved64=[None] * len(frequencies), outputs32=[], layer_counts=inputs["layer_counts"],
                   vertex_mask=inputs["vertex_mask"], param_total=_param_total(compiled, ep, mats, frequencies,
                                                                               bits, config))
    # the returned cell values are the FP64 records' sums (the function the
    # derivatives are taken of), rounded to FP32
    for fi in range(len(frequencies)):
        s64 = _linearisation(state, fi)
        state.outputs32.append({k: v.to(torch.float32) for k, v in s64.items()})
    out = _SolveFunction.apply(state, inputs["vertices"], inputs["eps_r"], inputs["sigma_e"], inputs["layer_eps_r"],
                               inputs["layer_sigma_e"], inputs["frequency"], inputs["tx"], inputs["rx"])
    result = dict(zip(ACCUM_FIELDS, out))
    result.update(compiled=compiled, ep=ep, dec=dec, evaluations=evs, count=K, width=width, rows=rows,
                  selected=selected, mats=mats, components=bits, ep_frequency=frequencies[0])
    return result


def solve_vjp(scene: Any, config, reference_frequency_hz, precision: str = "mixed"):
    """The deterministic solve with ``ad_mode="vjp"``: same outputs as the
    row-mode forward, differentiable in the scene values."""
    from .deterministic import (
        _BASE_COMPONENTS,
        _OPTIONAL_COMPONENTS,
        _SLOTS,
        Result,
        _component_counts,
        _layout,
        _metadata,
        _path_table,
    )

    launches0 = _native.launch_count()
    freq = reference_frequency_hz.reshape(1) if isinstance(reference_frequency_hz, torch.Tensor) else \
        [float(reference_frequency_hz)]
    v = vjp_forward(scene, config, freq, precision=precision)
    device = v["power_total"].device
    pt, ftr, fti = v["power_total"][0], v["field_total_real"][0], v["field_total_imag"][0]
    cp, cfr, cfi = v["component_power"][0], v["component_field_real"][0], v["component_field_imag"][0]
    rx = v["ep"].rx
    names = _BASE_COMPONENTS + tuple(n for n in _OPTIONAL_COMPONENTS if n in config.components)
    comp_power = {n: _layout(cp[_SLOTS[n]], rx) for n in names}
    comp_fields = {n: _layout(torch.complex(cfr[_SLOTS[n]], cfi[_SLOTS[n]]), rx) for n in names} \
        if config.return_field else {n: torch.empty((0,), dtype=torch.complex64, device=device) for n in names}
    dec = v["dec"]
    counts = _component_counts(dec["component_id"])
    paths = _path_table(dec, v["evaluations"][0], v["width"], v["compiled"], config.return_field) \
        if config.export_paths else None
    if paths is not None and v["count"] > 0:
        # the table's per-path field, gain and coefficient carry the records'
        # fixed-topology derivatives too
        ev = v["evaluations"][0]
        pf = differentiable_row_fields(scene, v["compiled"], v["ep"], v["mats"], float(v["ep_frequency"]),
                                       reference_frequency_hz, v["components"], config.max_depth, v["rows"],
                                       v["selected"], ev["path_field"])
        gain = ev["path_gain"] + (pf.abs() ** 2 - (pf.abs() ** 2).detach())
        coef = unit_coefficient(ev["coefficient"], pf, v["ep"].tx_power.index_select(0, dec["tx_id"].long()))
        fields = dict(field_real=pf.real, field_imag=pf.imag) if config.return_field else {}
        paths = replace(paths, path_gain=gain, coefficient=coef, **fields)
    meta = _metadata(config, counts, v["count"], _native.launch_count() - launches0,
                     {"ad": f"fixed-topology {config.ad_mode}"})
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
