"""Standalone field operators (mirror of the forward ops in ``witwin/channel/kernels/fields.py``).

Same names, argument meaning, validation errors and result dict as the
reference's ``field_free_space`` (:110-146), ``field_project_complex3``
(:149-177), ``field_reflection_sequence`` (:180-242) and
``field_transmission_sequence`` (:245-330); the arithmetic runs in
``libwcb200.so`` (``wcb_field_*``), FP32 fields with the k*d phase reduced
in FP64.
"""

from __future__ import annotations

import ctypes

import torch

from . import _native
from .kernels import _validate


def _validate3(name, value, ndim=2):
    _validate(name, value, dtype=torch.float32, ndim=ndim)
    if value.shape[-1] != 3:
        raise ValueError(f"{name} must end with shape (3,)")


def _result(count: int, device) -> dict[str, torch.Tensor]:
    return {
        "field_vector": torch.zeros((count, 3), dtype=torch.complex64, device=device),
        "coefficient": torch.zeros((count,), dtype=torch.complex64, device=device),
        "path_field": torch.zeros((count,), dtype=torch.complex64, device=device),
        "path_gain": torch.zeros((count,), dtype=torch.float32, device=device),
        "path_length_m": torch.zeros((count,), dtype=torch.float32, device=device),
        "delay_s": torch.zeros((count,), dtype=torch.float32, device=device),
        "direction": torch.zeros((count, 3), dtype=torch.float32, device=device),
    }


def _out_ptrs(out):
    return [_native.ptr(out[k]) for k in ("field_vector", "coefficient", "path_field", "path_gain", "path_length_m",
                                           "delay_s", "direction")]


def field_free_space(source: torch.Tensor, target: torch.Tensor, tx_power: torch.Tensor,
                     tx_polarization: torch.Tensor, rx_polarization: torch.Tensor, *,
                     frequency_hz: float) -> dict[str, torch.Tensor]:
    for name, value in (("source", source), ("target", target), ("tx_polarization", tx_polarization),
                        ("rx_polarization", rx_polarization)):
        _validate3(name, value)
    _validate("tx_power", tx_power, dtype=torch.float32, ndim=1)
    count = int(source.shape[0])
    if any(int(v.shape[0]) != count for v in (target, tx_power, tx_polarization, rx_polarization)):
        raise ValueError("free-space field tensors must have matching rows")
    if frequency_hz <= 0.0:
        raise ValueError("frequency_hz must be positive")
    out = _result(count, source.device)
    lib = _native.load()
    _native.check(lib.wcb_field_free_space(count, *(_native.ptr(t) for t in (source, target, tx_power,
                                                                             tx_polarization, rx_polarization)),
                                           float(frequency_hz), *_out_ptrs(out), _native.stream_handle(source.device)),
                  "wcb_field_free_space")
    return out


def field_project_complex3(field_vector: torch.Tensor, direction: torch.Tensor,
                           rx_polarization: torch.Tensor) -> dict[str, torch.Tensor]:
    _validate("field_vector", field_vector, dtype=torch.complex64, ndim=2)
    _validate3("direction", direction)
    _validate3("rx_polarization", rx_polarization)
    count = int(field_vector.shape[0])
    if field_vector.shape != (count, 3):
        raise ValueError("field_vector must have shape (N, 3)")
    if direction.shape != (count, 3) or rx_polarization.shape != (count, 3):
        raise ValueError("direction and rx_polarization must match field_vector rows")
    out = {"coefficient": torch.zeros((count,), dtype=torch.complex64, device=field_vector.device),
           "path_gain": torch.zeros((count,), dtype=torch.float32, device=field_vector.device)}
    lib = _native.load()
    _native.check(lib.wcb_field_project_complex3(count, _native.ptr(field_vector), _native.ptr(direction),
                                                 _native.ptr(rx_polarization), _native.ptr(out["coefficient"]),
                                                 _native.ptr(out["path_gain"]),
                                                 _native.stream_handle(field_vector.device)),
                  "wcb_field_project_complex3")
    return out


def field_reflection_sequence(source, target, interaction_positions, interaction_normals, tx_power,
                              tx_polarization, rx_polarization, eps_r, sigma_e, mu_r, gain, thickness, *,
                              frequency_hz: float) -> dict[str, torch.Tensor]:
    for name, value in (("source", source), ("target", target), ("tx_polarization", tx_polarization),
                        ("rx_polarization", rx_polarization)):
        _validate3(name, value)
    for name, value in (("interaction_positions", interaction_positions),
                        ("interaction_normals", interaction_normals)):
        _validate3(name, value, ndim=3)
    _validate("tx_power", tx_power, dtype=torch.float32, ndim=1)
    count = int(source.shape[0])
    depth = int(interaction_positions.shape[1])
    if interaction_positions.shape != (count, depth, 3) or depth <= 0:
        raise ValueError("interaction_positions must have shape (N, D, 3), D > 0")
    if interaction_normals.shape != interaction_positions.shape:
        raise ValueError("interaction_normals must match interaction_positions")
    for name, value in (("eps_r", eps_r), ("sigma_e", sigma_e), ("mu_r", mu_r), ("gain", gain),
                        ("thickness", thickness)):
        _validate(name, value, dtype=torch.float32, ndim=2)
        if value.shape != (count, depth):
            raise ValueError(f"{name} must have shape (N, D)")
    if frequency_hz <= 0.0:
        raise ValueError("frequency_hz must be positive")
    if depth > 5:
        raise ValueError("reflection chains deeper than 5 bounces are not supported")
    out = _result(count, source.device)
    lib = _native.load()
    args = (source, target, interaction_positions, interaction_normals, tx_power, tx_polarization, rx_polarization,
            eps_r, sigma_e, mu_r, gain, thickness)
    _native.check(lib.wcb_field_reflection_sequence(count, depth, *(_native.ptr(t) for t in args),
                                                    float(frequency_hz), *_out_ptrs(out),
                                                    _native.stream_handle(source.device)),
                  "wcb_field_reflection_sequence")
    return out


def field_transmission_sequence(path_valid, source, target, interaction_positions, interaction_normals,
                                interaction_material_id, interaction_valid, tx_power, tx_polarization,
                                rx_polarization, layer_offset, layer_count, layer_thickness_m, layer_eps_r,
                                layer_sigma_e, layer_mu_r, *, frequency_hz: float) -> dict[str, torch.Tensor]:
    """Straight thin-sheet chain.  Walls whose ``interaction_valid`` is False are
    skipped (the native op takes the valid walls packed first, in order); rows
    whose ``path_valid`` is False return zeros."""
    _validate("path_valid", path_valid, dtype=torch.bool, ndim=1)
    for name, value in (("source", source), ("target", target), ("tx_polarization", tx_polarization),
                        ("rx_polarization", rx_polarization)):
        _validate3(name, value)
    for name, value in (("interaction_positions", interaction_positions),
                        ("interaction_normals", interaction_normals)):
        _validate3(name, value, ndim=3)
    _validate("interaction_material_id", interaction_material_id, dtype=torch.int32, ndim=2)
    _validate("interaction_valid", interaction_valid, dtype=torch.bool, ndim=2)
    _validate("tx_power", tx_power, dtype=torch.float32, ndim=1)
    count = int(source.shape[0])
    if path_valid.shape != (count,):
        raise ValueError("path_valid must have shape (N,)")
    depth = int(interaction_positions.shape[1])
    if interaction_positions.shape != (count, depth, 3) or depth <= 0:
        raise ValueError("interaction_positions must have shape (N, D, 3), D > 0")
    if interaction_normals.shape != interaction_positions.shape:
        raise ValueError("interaction_normals must match interaction_positions")
    if interaction_material_id.shape != (count, depth):
        raise ValueError("interaction_material_id must have shape (N, D)")
    if interaction_valid.shape != (count, depth):
        raise ValueError("interaction_valid must have shape (N, D)")
    if any(int(v.shape[0]) != count for v in (target, tx_power, tx_polarization, rx_polarization)):
        raise ValueError("transmission endpoint tensors must have matching rows")
    _validate("layer_offset", layer_offset, dtype=torch.int32, ndim=1)
    _validate("layer_count", layer_count, dtype=torch.int32, ndim=1)
    for name, value in (("layer_thickness_m", layer_thickness_m), ("layer_eps_r", layer_eps_r),
                        ("layer_sigma_e", layer_sigma_e), ("layer_mu_r", layer_mu_r)):
        _validate(name, value, dtype=torch.float32, ndim=1)
    if layer_offset.shape != layer_count.shape:
        raise ValueError("layer_offset and layer_count must have the same shape")
    if frequency_hz <= 0.0:
        raise ValueError("frequency_hz must be positive")
    if depth > 5:
        raise ValueError("transmission chains through more than 5 walls are not supported")
    # pack the valid walls first, keeping their order
    order = torch.sort((~interaction_valid).to(torch.int8), dim=1, stable=True).indices
    normals = torch.gather(interaction_normals, 1, order[..., None].expand(-1, -1, 3)).contiguous()
    mids = torch.gather(interaction_material_id, 1, order).contiguous()
    walls = torch.where(path_valid, interaction_valid.sum(dim=1), 0).to(torch.int32).contiguous()
    m = _native.Materials()
    m.num_materials = int(layer_offset.shape[0])
    m.num_layers = int(layer_thickness_m.shape[0])
    for name, t in (("layer_offset", layer_offset), ("layer_count", layer_count),
                    ("layer_thickness", layer_thickness_m), ("layer_eps_r", layer_eps_r),
                    ("layer_sigma_e", layer_sigma_e), ("layer_mu_r", layer_mu_r)):
        setattr(m, name, _native.ptr(t))
    out = _result(count, source.device)
    lib = _native.load()
    _native.check(lib.wcb_field_transmission_sequence(
        count, depth, _native.ptr(source), _native.ptr(target), _native.ptr(normals), _native.ptr(mids),
        _native.ptr(walls), _native.ptr(tx_power), _native.ptr(tx_polarization), _native.ptr(rx_polarization),
        ctypes.byref(m), float(frequency_hz), *_out_ptrs(out), _native.stream_handle(source.device)),
        "wcb_field_transmission_sequence")
    if not bool(path_valid.all()):
        keep = path_valid
        for k, v in out.items():
            out[k] = torch.where(keep.view(-1, *([1] * (v.dim() - 1))), v, torch.zeros_like(v))
    return out
