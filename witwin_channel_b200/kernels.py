"""Flat accumulation operators (mirror of ``witwin/channel/kernels/deterministic.py``).

``deterministic_accumulate_flat`` and its backward/JVP companions keep the
reference's names, argument meaning, validation errors and output dict; the
work runs in ``libwcb200.so`` (``wcb_accumulate_flat*``).  The accumulation is
deterministic: every output slot sums its paths in path index order, so the
FP32 and FP64 results are reproducible bit for bit.
"""

from __future__ import annotations

import ctypes

import torch

from . import _native

ACCUM_FIELDS = (
    "power_total",
    "field_total_real",
    "field_total_imag",
    "component_power",
    "component_field_real",
    "component_field_imag",
)


def _validate(name: str, tensor, *, dtype, ndim: int) -> torch.Tensor:
    """Same checks and errors as the reference's ``validate_cuda_tensor`` (runtime.py:86-102)."""
    if not isinstance(tensor, torch.Tensor):
        raise TypeError(f"{name} must be a torch.Tensor")
    if tensor.dtype != dtype:
        raise TypeError(f"{name} must have dtype {dtype}")
    if not tensor.is_cuda:
        raise ValueError(f"{name} must be a CUDA tensor")
    if tensor.ndim != ndim:
        raise ValueError(f"{name} must have {ndim} dimensions")
    if not tensor.is_contiguous():
        raise ValueError(f"{name} must be contiguous")
    return tensor


def _check_inputs(valid, tx_id, rx_id, component_id, values, float_dtype, num_tx, num_rx, domain):
    if int(domain) not in (0, 1):
        raise ValueError("scattering_combine_domain must be 0 (power) or 1 (coherent)")
    _validate("valid", valid, dtype=torch.bool, ndim=1)
    _validate("tx_id", tx_id, dtype=torch.int32, ndim=1)
    _validate("rx_id", rx_id, dtype=torch.int32, ndim=1)
    _validate("component_id", component_id, dtype=torch.int32, ndim=1)
    for name, value in values.items():
        if value is not None:
            _validate(name, value, dtype=float_dtype, ndim=1)
    for name, tensor in {"valid": valid, "rx_id": rx_id, "component_id": component_id, **values}.items():
        if tensor is not None and tensor.shape != tx_id.shape:
            raise ValueError(f"{name} must match tx_id shape")
    if num_tx < 0 or num_rx < 0:
        raise ValueError("num_tx and num_rx must be non-negative")


def _dtype_code(dtype: torch.dtype) -> int:
    if dtype == torch.float32:
        return _native.DTYPE_F32
    if dtype == torch.float64:
        return _native.DTYPE_F64
    raise TypeError(f"unsupported dtype {dtype}")


def _outputs(num_tx: int, num_rx: int, dtype, device) -> dict[str, torch.Tensor]:
    out = {}
    for name in ACCUM_FIELDS:
        shape = (6, num_tx, num_rx) if name.startswith("component") else (num_tx, num_rx)
        out[name] = torch.empty(shape, dtype=dtype, device=device)
    return out


def _struct(d: dict | None) -> _native.AccumulateOutputs:
    d = d or {}
    return _native.AccumulateOutputs(*[_native.ptr(d.get(name)) for name in ACCUM_FIELDS])


def _workspace(nbytes: int, device) -> torch.Tensor:
    return torch.empty(max(int(nbytes), 1), dtype=torch.uint8, device=device)


def _forward(valid, tx_id, rx_id, component_id, path_gain, field_real, field_imag, num_tx, num_rx, coherent,
             domain) -> dict[str, torch.Tensor]:
    lib = _native.load()
    device = tx_id.device
    n = int(tx_id.numel())
    out = _outputs(int(num_tx), int(num_rx), path_gain.dtype, device)
    nbytes = ctypes.c_int64()
    _native.check(lib.wcb_accumulate_flat_workspace_size(n, ctypes.byref(nbytes)), "wcb_accumulate_flat_workspace_size")
    ws = _workspace(nbytes.value, device)
    s = _struct(out)
    _native.check(
        lib.wcb_accumulate_flat(_native.ptr(valid), _native.ptr(tx_id), _native.ptr(rx_id), _native.ptr(component_id),
                                _native.ptr(path_gain), _native.ptr(field_real), _native.ptr(field_imag), n,
                                int(num_tx), int(num_rx), int(bool(coherent)), int(domain),
                                _dtype_code(path_gain.dtype), ctypes.byref(s), _native.ptr(ws), ws.numel(),
                                _native.stream_handle(device)),
        "wcb_accumulate_flat",
    )
    return out


def deterministic_accumulate_flat(valid: torch.Tensor, tx_id: torch.Tensor, rx_id: torch.Tensor,
                                  component_id: torch.Tensor, path_gain: torch.Tensor, field_real: torch.Tensor,
                                  field_imag: torch.Tensor, *, num_tx: int, num_rx: int, coherent: bool,
                                  scattering_combine_domain: int = 0) -> dict[str, torch.Tensor]:
    """Six-slot per-cell accumulation (``kernels/deterministic.py:23-102``); float32 in and out."""
    _check_inputs(valid, tx_id, rx_id, component_id,
                  {"path_gain": path_gain, "field_real": field_real, "field_imag": field_imag}, torch.float32,
                  num_tx, num_rx, scattering_combine_domain)
    return _forward(valid, tx_id, rx_id, component_id, path_gain, field_real, field_imag, num_tx, num_rx, coherent,
                    scattering_combine_domain)


def deterministic_accumulate_flat_backward(
    valid, tx_id, rx_id, component_id, component_field_real, component_field_imag, field_total_real,
    field_total_imag, power_total, *, grad_power_total=None, grad_field_total_real=None,
    grad_field_total_imag=None, grad_component_power=None, grad_component_field_real=None,
    grad_component_field_imag=None, num_tx: int, num_rx: int, coherent: bool, scattering_combine_domain: int = 0,
) -> dict[str, torch.Tensor]:
    """Adjoint gather (``kernels/deterministic.py:115-152``)."""
    lib = _native.load()
    device = tx_id.device
    n = int(tx_id.numel())
    dtype = power_total.dtype
    grads = {k: (None if v is None else v.contiguous()) for k, v in zip(ACCUM_FIELDS, (
        grad_power_total, grad_field_total_real, grad_field_total_imag, grad_component_power,
        grad_component_field_real, grad_component_field_imag))}
    saved = {"power_total": power_total, "field_total_real": field_total_real, "field_total_imag": field_total_imag,
             "component_field_real": component_field_real, "component_field_imag": component_field_imag}
    out = {k: torch.empty(n, dtype=dtype, device=device) for k in ("grad_path_gain", "grad_field_real",
                                                                      "grad_field_imag")}
    sv, gv = _struct(saved), _struct(grads)
    _native.check(
        lib.wcb_accumulate_flat_backward(_native.ptr(valid), _native.ptr(tx_id), _native.ptr(rx_id),
                                         _native.ptr(component_id), n, int(num_tx), int(num_rx), int(bool(coherent)),
                                         int(scattering_combine_domain), _dtype_code(dtype), ctypes.byref(sv),
                                         ctypes.byref(gv), _native.ptr(out["grad_path_gain"]),
                                         _native.ptr(out["grad_field_real"]), _native.ptr(out["grad_field_imag"]),
                                         _native.stream_handle(device)),
        "wcb_accumulate_flat_backward",
    )
    return out


def deterministic_accumulate_flat_jvp(
    valid, tx_id, rx_id, component_id, component_field_real, component_field_imag, power_total, *,
    tangent_path_gain=None, tangent_field_real=None, tangent_field_imag=None, num_tx: int, num_rx: int,
    coherent: bool, scattering_combine_domain: int = 0,
) -> dict[str, torch.Tensor]:
    """Pushforward scatter (``kernels/deterministic.py:155-185``)."""
    lib = _native.load()
    device = tx_id.device
    n = int(tx_id.numel())
    dtype = power_total.dtype
    out = _outputs(int(num_tx), int(num_rx), dtype, device)
    saved = {"power_total": power_total, "component_field_real": component_field_real,
             "component_field_imag": component_field_imag}
    nbytes = ctypes.c_int64()
    _native.check(lib.wcb_accumulate_flat_jvp_workspace_size(n, _dtype_code(dtype), ctypes.byref(nbytes)),
                  "wcb_accumulate_flat_jvp_workspace_size")
    ws = _workspace(nbytes.value, device)
    sv, ov = _struct(saved), _struct(out)
    t = [None if v is None else v.contiguous() for v in (tangent_path_gain, tangent_field_real, tangent_field_imag)]
    _native.check(
        lib.wcb_accumulate_flat_jvp(_native.ptr(valid), _native.ptr(tx_id), _native.ptr(rx_id),
                                    _native.ptr(component_id), _native.ptr(t[0]), _native.ptr(t[1]),
                                    _native.ptr(t[2]), n, int(num_tx), int(num_rx), int(bool(coherent)),
                                    int(scattering_combine_domain), _dtype_code(dtype), ctypes.byref(sv),
                                    ctypes.byref(ov), _native.ptr(ws), ws.numel(), _native.stream_handle(device)),
        "wcb_accumulate_flat_jvp",
    )
    return out


class _AccumulateFlatFunction(torch.autograd.Function):
    """Differentiable flat accumulation (``kernels/deterministic.py:188-367``).

    Forward: the native accumulation (float32, or float64 for gradcheck).
    Backward: one adjoint gather per path.  Forward mode: the pushforward
    scatter.  The slot/tx/rx ids are frozen discrete inputs."""

    @staticmethod
    def forward(valid, tx_id, rx_id, component_id, path_gain, field_real, field_imag, num_tx, num_rx, coherent,
                domain):
        out = _forward(valid, tx_id, rx_id, component_id, path_gain, field_real, field_imag, num_tx, num_rx,
                       coherent, domain)
        return tuple(out[name] for name in ACCUM_FIELDS)

    @staticmethod
    def setup_context(ctx, inputs, output):
        ctx.set_materialize_grads(False)
        valid, tx_id, rx_id, component_id = (torch.autograd.forward_ad.unpack_dual(v).primal for v in inputs[:4])
        ctx.num_tx, ctx.num_rx = int(inputs[7]), int(inputs[8])
        ctx.coherent, ctx.domain = bool(inputs[9]), int(inputs[10])
        power_total, field_total_real, field_total_imag, _cp, cfr, cfi = output
        saved = (valid, tx_id, rx_id, component_id, cfr, cfi, field_total_real, field_total_imag, power_total)
        ctx.save_for_backward(*saved)
        ctx.save_for_forward(*saved)

    @staticmethod
    def backward(ctx, g_pt, g_ftr, g_fti, g_cp, g_cfr, g_cfi):
        none = (None,) * 11
        if not any(ctx.needs_input_grad[4:7]) or all(g is None for g in (g_pt, g_ftr, g_fti, g_cp, g_cfr, g_cfi)):
            return none
        valid, tx_id, rx_id, component_id, cfr, cfi, ftr, fti, pt = ctx.saved_tensors
        out = deterministic_accumulate_flat_backward(
            valid, tx_id, rx_id, component_id, cfr, cfi, ftr, fti, pt, grad_power_total=g_pt,
            grad_field_total_real=g_ftr, grad_field_total_imag=g_fti, grad_component_power=g_cp,
            grad_component_field_real=g_cfr, grad_component_field_imag=g_cfi, num_tx=ctx.num_tx,
            num_rx=ctx.num_rx, coherent=ctx.coherent, scattering_combine_domain=ctx.domain)
        return (None, None, None, None,
                out["grad_path_gain"] if ctx.needs_input_grad[4] else None,
                out["grad_field_real"] if ctx.needs_input_grad[5] else None,
                out["grad_field_imag"] if ctx.needs_input_grad[6] else None,
                None, None, None, None)

    @staticmethod
    def jvp(ctx, _tv, _tt, _tr, _tc, t_gain, t_real, t_imag, _a, _b, _c, _d):
        if t_gain is None and t_real is None and t_imag is None:
            return (None,) * len(ACCUM_FIELDS)
        valid, tx_id, rx_id, component_id, cfr, cfi, _ftr, _fti, pt = ctx.saved_tensors
        out = deterministic_accumulate_flat_jvp(
            valid, tx_id, rx_id, component_id, cfr, cfi, pt, tangent_path_gain=t_gain, tangent_field_real=t_real,
            tangent_field_imag=t_imag, num_tx=ctx.num_tx, num_rx=ctx.num_rx, coherent=ctx.coherent,
            scattering_combine_domain=ctx.domain)
        return tuple(out[name] for name in ACCUM_FIELDS)


def deterministic_accumulate_flat_ad(valid: torch.Tensor, tx_id: torch.Tensor, rx_id: torch.Tensor,
                                     component_id: torch.Tensor, path_gain: torch.Tensor, field_real: torch.Tensor,
                                     field_imag: torch.Tensor, *, num_tx: int, num_rx: int, coherent: bool,
                                     scattering_combine_domain: int = 0) -> dict[str, torch.Tensor]:
    """Differentiable accumulation; float32 or float64 (strict gradcheck) inputs."""
    dtype = path_gain.dtype if isinstance(path_gain, torch.Tensor) else None
    if dtype not in (torch.float32, torch.float64):
        raise TypeError("path_gain must have dtype torch.float32 or torch.float64")
    _check_inputs(valid, tx_id, rx_id, component_id,
                  {"path_gain": path_gain, "field_real": field_real, "field_imag": field_imag}, dtype,
                  num_tx, num_rx, scattering_combine_domain)
    out = _AccumulateFlatFunction.apply(valid, tx_id, rx_id, component_id, path_gain, field_real, field_imag,
                                        int(num_tx), int(num_rx), bool(coherent), int(scattering_combine_domain))
    return dict(zip(ACCUM_FIELDS, out))
