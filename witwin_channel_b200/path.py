"""Explicit path solver: per-link path export (``witwin.channel.path``).

Restates the reference's point-to-point path API (``witwin/channel/path.py``):
``Config`` (``:74-151``), ``RaggedPathSoA`` (``:164-337``: stable per-pair
ragged storage with the per-pair limit), ``InteractionType`` (``:344-349``),
``PathResult`` (``:354-793``: the padded (rx, rx_ant, tx, tx_ant, path, time)
result with its CIR, CFR and tap views and ``filter_by_type``),
``BeamformedPathResult`` (``:796-876``), ``endpoint_angles`` (``:879-884``),
the packing of evaluated rows (``from_evaluated_paths``, ``:887-975``) and
``solve`` (``:1707-1721``).

The paths come from the same native engine as the deterministic solve (row
mode: candidate kernels, canonical selection with a per-pair limit, row
field evaluation in ``libwcb200.so``); the packing is index arithmetic on
device tensors, and the CFR views run the native ``wcb_cfr`` kernel.
Antenna arrays (``path.py:1079-1486``): synthetic arrays expand the centre
endpoints' paths by far-field steering and element patterns; explicit
arrays trace every element as its own endpoint in the same native solve.
Endpoint weights (precoding / combining) ride on the result for
``beamform``.  With ``ad_mode`` "vjp" / "jvp" the coefficients ``a`` carry the
records' fixed-topology derivatives (native VJP / JVP).  Results have one time
step.
"""

from __future__ import annotations

import ctypes
import enum
import math
from dataclasses import dataclass, replace
from typing import Any

import torch

from . import _native, engine
from .compiler import compile_scene
from .constants import PHASE_CONVENTION
from .deterministic import AD_MODES, DEFAULT_COMPONENTS, DEPTH_CAPPED_COMPONENTS, VALID_COMPONENTS
from .deterministic import _endpoints, _frequency_value
from .scene import AntennaPattern, AntennaState, ReceiverGrid, orientation_matrix

_LIGHT_SPEED_M_PER_S = 299_792_458.0
_VALID_MAX_PATHS_SCOPES = frozenset({"per_pair"})


@dataclass(frozen=True, slots=True)
class Config:
    """Path solver configuration (reference ``path.py:74-151``)."""

    max_depth: int = 1
    components: frozenset[str] | set[str] | tuple[str, ...] | list[str] = DEFAULT_COMPONENTS
    max_paths: int | None = None
    max_paths_scope: str = "per_pair"
    ad_mode: str = "none"
    coupled_paths: bool = False
    coupled_candidate_limit: int = 1_000_000
    scattering_samples_per_m2: float = 8.0
    scattering_max_paths_per_pair: int = 4096
    scattering_power_threshold: float = 0.0
    scattering_chain_max_depth: int = 0
    scattering_chain_samples_per_m2: float = 2.0
    scattering_chain_max_rows: int = 256
    isb_boundary_taper: bool = False
    isb_boundary_taper_width: float = 0.5

    def __post_init__(self) -> None:
        if self.max_depth < 0:
            raise ValueError("max_depth must be non-negative")
        if not (self.isb_boundary_taper_width > 0.0):
            raise ValueError("isb_boundary_taper_width must be positive")
        if self.scattering_samples_per_m2 <= 0.0:
            raise ValueError("scattering_samples_per_m2 must be positive")
        if self.scattering_max_paths_per_pair <= 0:
            raise ValueError("scattering_max_paths_per_pair must be positive")
        if self.scattering_power_threshold < 0.0:
            raise ValueError("scattering_power_threshold must be non-negative")
        components = frozenset(self.components)
        if not components or not components.issubset(VALID_COMPONENTS):
            raise ValueError(f"components must be a subset of {sorted(VALID_COMPONENTS)}")
        if self.scattering_chain_max_depth < 0:
            raise ValueError("scattering_chain_max_depth must be non-negative")
        if self.scattering_chain_max_depth > 0 and "scattering" not in components:
            raise RuntimeError("scattering_chain_max_depth requires the 'scattering' component")
        if self.max_depth > 5 and components & DEPTH_CAPPED_COMPONENTS:
            raise RuntimeError("path reflection/transmission support max_depth <= 5")
        if self.max_paths is not None and self.max_paths <= 0:
            raise ValueError("max_paths must be positive when set")
        if self.max_paths_scope not in _VALID_MAX_PATHS_SCOPES:
            raise ValueError("path max_paths_scope must be 'per_pair'")
        if self.coupled_candidate_limit <= 0:
            raise ValueError("coupled_candidate_limit must be positive")
        if self.ad_mode not in AD_MODES:
            raise ValueError(f"path ad_mode must be one of {sorted(AD_MODES)}")
        object.__setattr__(self, "components", components)


class InteractionType(enum.IntFlag):
    NONE = 0
    REFLECTION = 1
    DIFFRACTION = 2
    TRANSMISSION = 4
    SCATTERING = 8


def _check(predicate: torch.Tensor, message: str) -> None:
    if not bool(predicate):
        raise ValueError(message)


@dataclass(frozen=True, slots=True)
class RaggedPathSoA:
    """Per-link ragged path storage: paths sorted stably by their pair index
    ((rx, rx_ant, tx, tx_ant) row-major) with ``pair_offsets`` delimiting each
    pair (reference ``path.py:164-337``)."""

    num_rx: int
    num_rx_ant: int
    num_tx: int
    num_tx_ant: int
    num_time_steps: int
    pair_offsets: torch.Tensor
    rx_id: torch.Tensor
    rx_ant_id: torch.Tensor
    tx_id: torch.Tensor
    tx_ant_id: torch.Tensor
    field: torch.Tensor
    delay_s: torch.Tensor
    theta_t: torch.Tensor
    phi_t: torch.Tensor
    theta_r: torch.Tensor
    phi_r: torch.Tensor
    interaction_type: torch.Tensor
    primitive_id: torch.Tensor
    material_id: torch.Tensor
    position: torch.Tensor
    normal: torch.Tensor

    @property
    def path_count(self) -> int:
        return int(self.delay_s.shape[0])

    @property
    def pair_count(self) -> int:
        return self.num_rx * self.num_rx_ant * self.num_tx * self.num_tx_ant

    @property
    def max_depth(self) -> int:
        return int(self.interaction_type.shape[1])

    @classmethod
    def from_flat(cls, *, num_rx: int, num_rx_ant: int, num_tx: int, num_tx_ant: int, rx_id: torch.Tensor,
                  tx_id: torch.Tensor, field: torch.Tensor, delay_s: torch.Tensor, theta_t: torch.Tensor,
                  phi_t: torch.Tensor, theta_r: torch.Tensor, phi_r: torch.Tensor, interaction_type: torch.Tensor,
                  primitive_id: torch.Tensor, material_id: torch.Tensor, position: torch.Tensor,
                  normal: torch.Tensor, rx_ant_id: torch.Tensor | None = None, tx_ant_id: torch.Tensor | None = None,
                  max_paths_per_pair: int | None = None) -> "RaggedPathSoA":
        count = int(delay_s.shape[0])
        device = delay_s.device
        if field.ndim == 1:
            field = field.unsqueeze(-1)
        if field.ndim != 2 or field.shape[0] != count:
            raise ValueError("field must have shape (path, time)")
        if field.dtype != torch.complex64:
            raise ValueError("field must use complex64")
        if max_paths_per_pair is not None and max_paths_per_pair <= 0:
            raise ValueError("max_paths_per_pair must be positive when set")
        zeros = torch.zeros((count,), device=device, dtype=torch.int32)
        rx_ant_id = zeros if rx_ant_id is None else rx_ant_id.to(device=device, dtype=torch.int32)
        tx_ant_id = zeros if tx_ant_id is None else tx_ant_id.to(device=device, dtype=torch.int32)
        rx_id = rx_id.to(device=device, dtype=torch.int32)
        tx_id = tx_id.to(device=device, dtype=torch.int32)
        per_path = {"rx_id": rx_id, "rx_ant_id": rx_ant_id, "tx_id": tx_id, "tx_ant_id": tx_ant_id,
                    "delay_s": delay_s, "theta_t": theta_t, "phi_t": phi_t, "theta_r": theta_r, "phi_r": phi_r}
        for name, value in per_path.items():
            if value.shape != (count,):
                raise ValueError(f"{name} must have shape (path,)")
        if interaction_type.ndim != 2:
            raise ValueError("interaction_type must have shape (path, depth)")
        depth = int(interaction_type.shape[1])
        for name, value in {"interaction_type": interaction_type, "primitive_id": primitive_id,
                            "material_id": material_id}.items():
            if value.shape != (count, depth):
                raise ValueError(f"{name} must have shape (path, depth)")
        for name, value in {"position": position, "normal": normal}.items():
            if value.shape != (count, depth, 3):
                raise ValueError(f"{name} must have shape (path, depth, 3)")
        pair_count = int(num_rx) * int(num_rx_ant) * int(num_tx) * int(num_tx_ant)
        if count and pair_count <= 0:
            raise ValueError("non-empty paths require non-empty endpoint dimensions")
        for ids, dim, name in ((rx_id, num_rx, "rx_id"), (rx_ant_id, num_rx_ant, "rx_ant_id"),
                               (tx_id, num_tx, "tx_id"), (tx_ant_id, num_tx_ant, "tx_ant_id")):
            _check(((ids >= 0) & (ids < int(dim))).all(), f"{name} is outside the declared endpoint dimension")
        pair_index = ((rx_id.to(torch.int64) * int(num_rx_ant) + rx_ant_id) * int(num_tx) + tx_id) * int(num_tx_ant) \
            + tx_ant_id
        order = torch.argsort(pair_index, stable=True)
        pair_index = pair_index[order]
        counts = torch.bincount(pair_index, minlength=pair_count)
        if max_paths_per_pair is not None and count:
            starts = torch.cumsum(counts, dim=0) - counts
            ranks = torch.arange(count, device=device, dtype=torch.int64) - torch.repeat_interleave(starts, counts)
            keep = ranks < int(max_paths_per_pair)
            order = order[keep]
            pair_index = pair_index[keep]
            counts = torch.bincount(pair_index, minlength=pair_count)
        offsets = torch.cat((torch.zeros((1,), device=device, dtype=torch.int64), torch.cumsum(counts, dim=0)))

        def take(value: torch.Tensor, dtype: torch.dtype) -> torch.Tensor:
            return value.to(device=device, dtype=dtype)[order].contiguous()

        return cls(num_rx=int(num_rx), num_rx_ant=int(num_rx_ant), num_tx=int(num_tx), num_tx_ant=int(num_tx_ant),
                   num_time_steps=int(field.shape[1]), pair_offsets=offsets.contiguous(),
                   rx_id=take(rx_id, torch.int32), rx_ant_id=take(rx_ant_id, torch.int32),
                   tx_id=take(tx_id, torch.int32), tx_ant_id=take(tx_ant_id, torch.int32),
                   field=take(field, torch.complex64), delay_s=take(delay_s, torch.float32),
                   theta_t=take(theta_t, torch.float32), phi_t=take(phi_t, torch.float32),
                   theta_r=take(theta_r, torch.float32), phi_r=take(phi_r, torch.float32),
                   interaction_type=take(interaction_type, torch.int32), primitive_id=take(primitive_id, torch.int32),
                   material_id=take(material_id, torch.int32), position=take(position, torch.float32),
                   normal=take(normal, torch.float32))


def _masked_min(values: torch.Tensor, valid: torch.Tensor) -> torch.Tensor:
    if values.shape[-1] == 0:
        return torch.zeros((*values.shape[:-1], 1), device=values.device, dtype=values.dtype)
    minima = torch.where(valid, values, torch.full_like(values, float("inf"))).min(dim=-1, keepdim=True).values
    return torch.where(torch.isfinite(minima), minima, torch.zeros_like(minima))


_CFR_WORKSPACE = engine.Workspace()


def _native_cfr(rx_flat: torch.Tensor, tx_flat: torch.Tensor, coeff: torch.Tensor, tau: torch.Tensor, num_rx: int,
                num_tx: int, frequencies: torch.Tensor, normalize: bool) -> torch.Tensor:
    """(num_rx, num_tx, K) complex64 spectra of records given in ascending
    (rx, tx) order, through ``wcb_cfr`` (one CFR per link; delays normalised
    per link by their minimum when ``normalize``)."""
    device = coeff.device
    if device.type != "cuda":
        raise RuntimeError("the CFR view runs on the GPU: move the PathResult to CUDA")
    freqs = frequencies.to(device=device, dtype=torch.float64).contiguous()
    K = int(freqs.shape[0])
    f_host = freqs.cpu()
    df = 0.0
    if K > 1:
        steps = f_host[1:] - f_host[:-1]
        if float((steps - steps[0]).abs().max()) <= 1e-9 * max(float(steps[0].abs()), 1.0):
            df = float(steps[0])
    elif K == 1:
        df = 1.0
    n = int(coeff.shape[0])
    out = torch.empty((num_tx, num_rx, K), dtype=torch.complex64, device=device)
    if num_rx * num_tx == 0 or K == 0:
        return out.permute(1, 0, 2)
    lib = _native.load()
    nbytes = ctypes.c_int64()
    _native.check(lib.wcb_cfr_workspace_size(int(num_tx), int(num_rx), ctypes.byref(nbytes)), "wcb_cfr_workspace_size")
    ws = _CFR_WORKSPACE.get(nbytes.value, device)
    tx_i = tx_flat.to(torch.int32).contiguous()
    rx_i = rx_flat.to(torch.int32).contiguous()
    d = tau.to(torch.float32).contiguous()
    a = torch.view_as_real(coeff.to(torch.complex64).contiguous())
    _native.check(
        lib.wcb_cfr(_native.ptr(tx_i) if n else None, _native.ptr(rx_i) if n else None, _native.ptr(d) if n else None,
                    _native.ptr(a) if n else None, n, int(num_tx), int(num_rx), K, float(f_host[0]), df,
                    _native.ptr(freqs), int(bool(normalize)), _native.ptr(out), _native.ptr(ws), ws.numel(),
                    _native.stream_handle(device)),
        "wcb_cfr",
    )
    return out.permute(1, 0, 2)


@dataclass(frozen=True, slots=True)
class PathResult:
    """Padded path result, shape (rx, rx_ant, tx, tx_ant, path[, time])
    (reference ``path.py:354-793``)."""

    a: torch.Tensor
    tau: torch.Tensor
    theta_t: torch.Tensor
    phi_t: torch.Tensor
    theta_r: torch.Tensor
    phi_r: torch.Tensor
    valid: torch.Tensor
    interaction_type: torch.Tensor
    primitive_id: torch.Tensor
    material_id: torch.Tensor
    position: torch.Tensor
    normal: torch.Tensor
    num_paths: torch.Tensor
    metadata: dict[str, Any]
    field_xyz: torch.Tensor | None = None
    field_direction: torch.Tensor | None = None
    tx_weights: torch.Tensor | None = None
    rx_weights: torch.Tensor | None = None

    def __post_init__(self) -> None:
        if self.a.ndim != 6 or self.a.dtype != torch.complex64:
            raise ValueError("a must be complex64 with shape (rx, rx_ant, tx, tx_ant, path, time)")
        path_shape = self.a.shape[:-1]
        for name in ("tau", "theta_t", "phi_t", "theta_r", "phi_r", "valid"):
            if getattr(self, name).shape != path_shape:
                raise ValueError(f"{name} must match the path shape")
        depth_shape = (*path_shape, self.max_depth)
        for name in ("interaction_type", "primitive_id", "material_id"):
            if getattr(self, name).shape != depth_shape:
                raise ValueError(f"{name} must match the depth shape")
        for name in ("position", "normal"):
            if getattr(self, name).shape != (*depth_shape, 3):
                raise ValueError(f"{name} must match the vector depth shape")
        if self.num_paths.shape != self.path_count_shape:
            raise ValueError("num_paths must match the endpoint-pair shape")
        field_xyz = self.field_xyz
        if field_xyz is None:
            field_xyz = torch.zeros((*path_shape, 3), device=self.a.device, dtype=torch.complex64)
            object.__setattr__(self, "field_xyz", field_xyz)
        field_direction = self.field_direction
        if field_direction is None:
            field_direction = torch.zeros((*path_shape, 3), device=self.a.device, dtype=torch.float32)
            object.__setattr__(self, "field_direction", field_direction)
        if field_xyz.shape != (*path_shape, 3):
            raise ValueError("field_xyz must match the path shape with a complex3 tail")
        if field_direction.shape != (*path_shape, 3):
            raise ValueError("field_direction must match the path shape with a vec3 tail")
        if field_xyz.dtype != torch.complex64:
            raise ValueError("field_xyz must use complex64")
        if field_direction.dtype != torch.float32:
            raise ValueError("field_direction must use float32")
        if self.tx_weights is not None and self.tx_weights.shape != (self.num_tx, self.num_tx_ant):
            raise ValueError("tx_weights must match the transmitter antenna shape")
        if self.rx_weights is not None and self.rx_weights.shape != (self.num_rx, self.num_rx_ant):
            raise ValueError("rx_weights must match the receiver antenna shape")
        if self.valid.dtype != torch.bool:
            raise ValueError("valid must use bool")
        if any(getattr(self, n).dtype != torch.float32
               for n in ("tau", "theta_t", "phi_t", "theta_r", "phi_r", "position", "normal")):
            raise ValueError("path geometry tensors must use float32")
        if any(getattr(self, n).dtype != torch.int32
               for n in ("interaction_type", "primitive_id", "material_id", "num_paths")):
            raise ValueError("interaction and path-count tensors must use int32")
        tensors = (self.a, self.tau, self.theta_t, self.phi_t, self.theta_r, self.phi_r, self.valid,
                   self.interaction_type, self.primitive_id, self.material_id, self.position, self.normal,
                   self.num_paths, field_xyz, field_direction)
        if any(t.device != self.a.device for t in tensors):
            raise ValueError("all PathResult tensors must share one device")

    # -- shape --------------------------------------------------------------
    @property
    def num_rx(self) -> int:
        return int(self.a.shape[0])

    @property
    def num_rx_ant(self) -> int:
        return int(self.a.shape[1])

    @property
    def num_tx(self) -> int:
        return int(self.a.shape[2])

    @property
    def num_tx_ant(self) -> int:
        return int(self.a.shape[3])

    @property
    def max_num_paths(self) -> int:
        return int(self.a.shape[4])

    @property
    def num_time_steps(self) -> int:
        return int(self.a.shape[5])

    @property
    def max_depth(self) -> int:
        return int(self.interaction_type.shape[-1])

    @property
    def path_shape(self) -> tuple[int, int, int, int, int]:
        return tuple(int(v) for v in self.a.shape[:-1])  # type: ignore[return-value]

    @property
    def path_count_shape(self) -> tuple[int, int, int, int]:
        return tuple(int(v) for v in self.a.shape[:4])  # type: ignore[return-value]

    @property
    def rx_id(self) -> torch.Tensor:
        ids = torch.arange(self.num_rx, device=self.a.device, dtype=torch.int32)
        return ids.reshape(-1, 1, 1, 1, 1).expand(self.path_shape).contiguous()

    @property
    def tx_id(self) -> torch.Tensor:
        ids = torch.arange(self.num_tx, device=self.a.device, dtype=torch.int32)
        return ids.reshape(1, 1, -1, 1, 1).expand(self.path_shape).contiguous()

    @property
    def path_length_m(self) -> torch.Tensor:
        length = self.tau * _LIGHT_SPEED_M_PER_S
        return torch.where(self.valid, length, torch.full_like(length, -1.0))

    @property
    def types(self) -> torch.Tensor:
        return self.interaction_type

    @property
    def vertices(self) -> torch.Tensor:
        return self.position

    @property
    def normals(self) -> torch.Tensor:
        return self.normal

    @property
    def objects(self) -> torch.Tensor:
        return self.primitive_id

    # -- packing ------------------------------------------------------------
    @classmethod
    def from_ragged(cls, ragged: RaggedPathSoA, *, max_paths_per_pair: int | None = None, minimum_path_width: int = 0,
                    metadata: dict[str, Any] | None = None) -> "PathResult":
        counts = ragged.pair_offsets[1:] - ragged.pair_offsets[:-1]
        if max_paths_per_pair is None:
            max_paths_per_pair = int(counts.max().item()) if counts.numel() else 0
        width = max(int(max_paths_per_pair), int(minimum_path_width))
        if width < 0:
            raise ValueError("max_paths_per_pair must be non-negative")
        _check((counts <= width).all(), "ragged input exceeds max_paths_per_pair")
        base = (ragged.num_rx, ragged.num_rx_ant, ragged.num_tx, ragged.num_tx_ant)
        shape = (*base, width)
        device = ragged.delay_s.device
        ranks = torch.arange(ragged.path_count, device=device, dtype=torch.int64) - torch.repeat_interleave(
            ragged.pair_offsets[:-1], counts)
        pair = torch.repeat_interleave(torch.arange(ragged.pair_count, device=device, dtype=torch.int64), counts)
        linear = pair * width + ranks
        slots = ragged.pair_count * width

        def padded(source: torch.Tensor, tail: tuple[int, ...], fill: float | int) -> torch.Tensor:
            out = torch.full((slots, *tail), fill, device=device, dtype=source.dtype)
            out[linear] = source
            return out.reshape(*shape, *tail)

        valid = torch.zeros((slots,), device=device, dtype=torch.bool)
        valid[linear] = True
        meta = dict(metadata or {})
        meta.update({"schema": "PathResult", "schema_version": 1, "max_paths_scope": "per_pair",
                     "stable_order": "input_order_within_receiver_antenna_transmitter_antenna_pair"})
        d = ragged.max_depth
        return cls(a=padded(ragged.field, (ragged.num_time_steps,), 0.0), tau=padded(ragged.delay_s, (), -1.0),
                   theta_t=padded(ragged.theta_t, (), 0.0), phi_t=padded(ragged.phi_t, (), 0.0),
                   theta_r=padded(ragged.theta_r, (), 0.0), phi_r=padded(ragged.phi_r, (), 0.0),
                   valid=valid.reshape(shape),
                   interaction_type=padded(ragged.interaction_type, (d,), int(InteractionType.NONE)),
                   primitive_id=padded(ragged.primitive_id, (d,), -1),
                   material_id=padded(ragged.material_id, (d,), -1),
                   position=padded(ragged.position, (d, 3), 0.0), normal=padded(ragged.normal, (d, 3), 0.0),
                   num_paths=counts.to(torch.int32).reshape(base), metadata=meta)

    # -- signal views -------------------------------------------------------
    def cir(self, *, normalize_delays: bool = True) -> tuple[torch.Tensor, torch.Tensor]:
        tau = self.tau
        if normalize_delays:
            tau = tau - _masked_min(tau, self.valid)
        tau = torch.where(self.valid, tau, torch.full_like(tau, -1.0))
        return torch.where(self.valid.unsqueeze(-1), self.a, torch.zeros_like(self.a)), tau

    def cfr(self, frequencies: torch.Tensor, *, normalize_delays: bool = True) -> torch.Tensor:
        """(rx, rx_ant, tx, tx_ant, time, frequency) complex64: each antenna
        pair's paths summed as a_p exp(-j 2 pi tau_p f), delays normalised per
        pair by their minimum.  Runs ``wcb_cfr`` on the GPU."""
        if not isinstance(frequencies, torch.Tensor):
            frequencies = torch.as_tensor(frequencies, dtype=torch.float64)
        if frequencies.ndim != 1:
            raise ValueError("frequencies must have shape (frequency,)")
        rxp = self.num_rx * self.num_rx_ant
        txp = self.num_tx * self.num_tx_ant
        flat_valid = self.valid.reshape(-1)
        pair = torch.arange(rxp * txp, device=self.a.device, dtype=torch.int64).repeat_interleave(self.max_num_paths)
        pair = pair[flat_valid]
        rx_flat, tx_flat = pair // max(txp, 1), pair % max(txp, 1)
        tau = self.tau.reshape(-1)[flat_valid]
        coeff = self.a.reshape(-1, self.num_time_steps)[flat_valid]
        out = [_native_cfr(rx_flat, tx_flat, coeff[:, t], tau, rxp, txp, frequencies, normalize_delays)
               for t in range(self.num_time_steps)]
        spectra = torch.stack(out, dim=2)  # (rx', tx', time, K)
        return spectra.reshape(self.num_rx, self.num_rx_ant, self.num_tx, self.num_tx_ant, self.num_time_steps, -1)

    def taps(self, bandwidth: float, num_taps: int, *, normalize_delays: bool = True) -> torch.Tensor:
        if bandwidth <= 0.0:
            raise ValueError("bandwidth must be > 0")
        if num_taps <= 0:
            raise ValueError("num_taps must be > 0")
        tau = self.tau
        if normalize_delays:
            tau = tau - _masked_min(tau, self.valid)
        tap_index = torch.round(tau * float(bandwidth)).to(torch.int64)
        out = torch.zeros((*self.path_count_shape, self.num_time_steps, int(num_taps)), device=self.a.device,
                          dtype=torch.complex64)
        if self.max_num_paths == 0:
            return out
        base_count = self.num_rx * self.num_rx_ant * self.num_tx * self.num_tx_ant
        coeff = self.a.reshape(base_count, self.max_num_paths, self.num_time_steps)
        tap_index = tap_index.reshape(base_count, self.max_num_paths)
        keep = self.valid.reshape(base_count, self.max_num_paths) & (tap_index >= 0) & (tap_index < num_taps)
        base = torch.arange(base_count, device=self.a.device).view(-1, 1, 1).expand_as(coeff.real)
        time = torch.arange(self.num_time_steps, device=self.a.device).view(1, 1, -1).expand_as(coeff.real)
        tap = tap_index.unsqueeze(-1).expand_as(coeff.real)
        keep = keep.unsqueeze(-1).expand_as(coeff.real)
        out.reshape(base_count, self.num_time_steps, num_taps).index_put_((base[keep], time[keep], tap[keep]),
                                                                         coeff[keep], accumulate=True)
        return out

    def beamform(self, *, tx_weights: torch.Tensor | None = None,
                 rx_weights: torch.Tensor | None = None) -> "BeamformedPathResult":
        tx = self.tx_weights if tx_weights is None else tx_weights
        rx = self.rx_weights if rx_weights is None else rx_weights
        if tx is None or rx is None:
            raise ValueError("beamform requires tx_weights and rx_weights, either explicitly or on every solved "
                             "endpoint")
        tx = tx.to(device=self.a.device, dtype=torch.complex64)
        rx = rx.to(device=self.a.device, dtype=torch.complex64)
        if tx.ndim == 1 and self.num_tx == 1:
            tx = tx.unsqueeze(0)
        if rx.ndim == 1 and self.num_rx == 1:
            rx = rx.unsqueeze(0)
        if tx.shape != (self.num_tx, self.num_tx_ant):
            raise ValueError(f"tx_weights must have shape {(self.num_tx, self.num_tx_ant)}")
        if rx.shape != (self.num_rx, self.num_rx_ant):
            raise ValueError(f"rx_weights must have shape {(self.num_rx, self.num_rx_ant)}")
        return BeamformedPathResult(source=self, tx_weights=tx, rx_weights=rx)

    def filter_by_type(self, *interaction_types: int) -> "PathResult":
        if not interaction_types:
            return self
        requested = {int(v) for v in interaction_types}
        nonempty = self.interaction_type != int(InteractionType.NONE)
        keep = self.valid & (~nonempty.any(dim=-1) if 0 in requested else torch.zeros_like(self.valid))
        for value in requested - {0}:
            keep = keep | (self.valid & (self.interaction_type == value).any(dim=-1))
        per_tx = self.num_tx * self.num_tx_ant
        pair = torch.arange(self.num_rx * self.num_rx_ant * per_tx, device=self.a.device).view(-1, 1).expand(
            -1, self.max_num_paths).reshape(-1)[keep.reshape(-1)]
        rx_id = pair // (self.num_rx_ant * per_tx)
        rem = pair % (self.num_rx_ant * per_tx)
        rx_ant_id = rem // per_tx
        rem = rem % per_tx
        ragged = RaggedPathSoA.from_flat(
            num_rx=self.num_rx, num_rx_ant=self.num_rx_ant, num_tx=self.num_tx, num_tx_ant=self.num_tx_ant,
            rx_id=rx_id, rx_ant_id=rx_ant_id, tx_id=rem // self.num_tx_ant, tx_ant_id=rem % self.num_tx_ant,
            field=self.a[keep], delay_s=self.tau[keep], theta_t=self.theta_t[keep], phi_t=self.phi_t[keep],
            theta_r=self.theta_r[keep], phi_r=self.phi_r[keep], interaction_type=self.interaction_type[keep],
            primitive_id=self.primitive_id[keep], material_id=self.material_id[keep], position=self.position[keep],
            normal=self.normal[keep])
        meta = dict(self.metadata)
        meta["filtered_interaction_types"] = sorted(requested)
        filtered = PathResult.from_ragged(ragged, minimum_path_width=1, metadata=meta)
        return replace(filtered, tx_weights=self.tx_weights, rx_weights=self.rx_weights)


@dataclass(frozen=True, slots=True)
class BeamformedPathResult:
    """Beamformed signal views over a raw :class:`PathResult` (reference
    ``path.py:796-876``): coefficients weighted by conj(rx_w) * tx_w and
    merged per (rx, tx) link."""

    source: PathResult
    tx_weights: torch.Tensor
    rx_weights: torch.Tensor

    def cir(self, *, normalize_delays: bool = True) -> tuple[torch.Tensor, torch.Tensor]:
        s = self.source
        factor = (self.rx_weights.conj().reshape(s.num_rx, s.num_rx_ant, 1, 1, 1, 1)
                  * self.tx_weights.reshape(1, 1, s.num_tx, s.num_tx_ant, 1, 1))
        coeff = torch.where(s.valid.unsqueeze(-1), s.a * factor, torch.zeros_like(s.a))
        coeff = coeff.permute(0, 2, 1, 3, 4, 5).reshape(s.num_rx, s.num_tx, s.num_rx_ant * s.num_tx_ant * s.max_num_paths,
                                                        s.num_time_steps)
        valid = s.valid.permute(0, 2, 1, 3, 4).reshape(s.num_rx, s.num_tx, -1)
        tau = s.tau.permute(0, 2, 1, 3, 4).reshape(s.num_rx, s.num_tx, -1)
        if normalize_delays:
            tau = tau - _masked_min(tau, valid)
        tau = torch.where(valid, tau, torch.full_like(tau, -1.0))
        return coeff, tau

    def cfr(self, frequencies: torch.Tensor, *, normalize_delays: bool = True) -> torch.Tensor:
        """(rx, tx, time, frequency) complex64 through ``wcb_cfr``."""
        if not isinstance(frequencies, torch.Tensor):
            frequencies = torch.as_tensor(frequencies, dtype=torch.float64)
        if frequencies.ndim != 1:
            raise ValueError("frequencies must have shape (frequency,)")
        s = self.source
        coeff, tau = self.cir(normalize_delays=False)
        valid = tau >= 0.0
        n_per = int(tau.shape[2])
        link = torch.arange(s.num_rx * s.num_tx, device=tau.device, dtype=torch.int64).repeat_interleave(n_per)
        flat = valid.reshape(-1)
        link = link[flat]
        rx_flat, tx_flat = link // max(s.num_tx, 1), link % max(s.num_tx, 1)
        t = tau.reshape(-1)[flat]
        c = coeff.reshape(-1, s.num_time_steps)[flat]
        out = [_native_cfr(rx_flat, tx_flat, c[:, k], t, s.num_rx, s.num_tx, frequencies, normalize_delays)
               for k in range(s.num_time_steps)]
        return torch.stack(out, dim=2)

    def taps(self, bandwidth: float, num_taps: int, *, normalize_delays: bool = True) -> torch.Tensor:
        if bandwidth <= 0.0:
            raise ValueError("bandwidth must be > 0")
        if num_taps <= 0:
            raise ValueError("num_taps must be > 0")
        s = self.source
        coeff, tau = self.cir(normalize_delays=normalize_delays)
        tap_index = torch.round(tau * float(bandwidth)).to(torch.int64)
        out = torch.zeros((s.num_rx, s.num_tx, s.num_time_steps, int(num_taps)), device=coeff.device,
                          dtype=torch.complex64)
        if coeff.shape[2] == 0:
            return out
        base_count = s.num_rx * s.num_tx
        coeff = coeff.reshape(base_count, coeff.shape[2], s.num_time_steps)
        tap_index = tap_index.reshape(base_count, tap_index.shape[2])
        keep = (tap_index >= 0) & (tap_index < num_taps)
        base = torch.arange(base_count, device=coeff.device).view(-1, 1, 1).expand_as(coeff.real)
        time = torch.arange(s.num_time_steps, device=coeff.device).view(1, 1, -1).expand_as(coeff.real)
        tap = tap_index.unsqueeze(-1).expand_as(coeff.real)
        keep = keep.unsqueeze(-1).expand_as(coeff.real)
        out.reshape(base_count, s.num_time_steps, num_taps).index_put_((base[keep], time[keep], tap[keep]),
                                                                      coeff[keep], accumulate=True)
        return out


def endpoint_angles(direction: torch.Tensor) -> tuple[torch.Tensor, torch.Tensor]:
    """Zenith and azimuth of a direction (reference ``path.py:879-884``)."""
    norm = torch.linalg.vector_norm(direction, dim=-1)
    safe = torch.clamp(norm, min=torch.finfo(direction.dtype).tiny)
    theta = torch.acos(torch.clamp(direction[..., 2] / safe, -1.0, 1.0))
    phi = torch.atan2(direction[..., 1], direction[..., 0])
    return theta.to(torch.float32), phi.to(torch.float32)


_INTERACTION_OF_COMPONENT = {1: int(InteractionType.REFLECTION), 2: int(InteractionType.DIFFRACTION),
                             5: int(InteractionType.TRANSMISSION)}


def _receiver_positions(scene: Any, rx: dict, device: torch.device) -> torch.Tensor:
    if rx["kind"] == "grid":
        return rx["grid"].points().to(device=device, dtype=torch.float32)
    return rx["positions"]


def _validate(scene: Any, config: Config) -> None:
    if config.coupled_paths:
        raise NotImplementedError("coupled reflection-diffraction paths are outside this engine")
    if "scattering" in config.components:
        raise NotImplementedError("rough-surface scattering is outside this engine")
    if config.isb_boundary_taper:
        raise NotImplementedError("the ISB boundary taper is outside this engine")
    if config.max_depth < 1 and ("reflection" in config.components or "diffraction" in config.components):
        raise RuntimeError("requested reflection/diffraction paths require max_depth >= 1")
    if not torch.cuda.is_available():
        raise RuntimeError("witwin_channel_b200.path solver requires CUDA")


# --- antenna arrays (reference path.py:1079-1486, scene/endpoints.py:66-125) ---

_ARRAY_PHASE_CONVENTION = "exp(+j*k*element_position_dot_endpoint_direction)"


def _unit_vector(theta: torch.Tensor, phi: torch.Tensor) -> torch.Tensor:
    sin_theta = torch.sin(theta)
    return torch.stack((sin_theta * torch.cos(phi), sin_theta * torch.sin(phi), torch.cos(theta)), dim=-1)


def _rotation(endpoint: Any, device: torch.device) -> torch.Tensor:
    orientation = getattr(endpoint, "orientation", None)
    if orientation is None:
        return torch.eye(3, device=device)
    return orientation_matrix(orientation).to(device)


def _local_direction(direction: torch.Tensor, endpoint: Any) -> torch.Tensor:
    return direction @ _rotation(endpoint, direction.device)


def pattern_field_response(pattern: AntennaPattern, local_direction: torch.Tensor) -> torch.Tensor:
    """Element field response at endpoint-local directions (reference
    ``scene/endpoints.py:66-95``): isotropic 1, vertical sqrt(1 - z^2),
    horizontal sqrt(1 - x^2) of the unit direction, or the custom callable."""

    direction = local_direction.to(torch.float32)
    direction = direction / torch.linalg.vector_norm(direction, dim=-1, keepdim=True).clamp_min(
        torch.finfo(torch.float32).tiny)
    if pattern.kind == "custom":
        response = pattern.custom(direction)
        if response.shape != direction.shape[:-1]:
            raise ValueError("custom pattern response must match direction batch shape")
        return response.to(device=direction.device, dtype=torch.complex64)
    if pattern.kind == "vertical":
        response = torch.sqrt(torch.clamp(1.0 - direction[..., 2].square(), min=0.0))
    elif pattern.kind == "horizontal":
        response = torch.sqrt(torch.clamp(1.0 - direction[..., 0].square(), min=0.0))
    else:
        response = torch.ones(direction.shape[:-1], device=direction.device)
    return response.to(torch.complex64)


def steering_vector(endpoint: Any, direction: torch.Tensor, *, frequency_hz: float) -> torch.Tensor:
    """``exp(+j k r . u)`` per element (reference ``scene/endpoints.py:98-125``)
    under the ``exp(-j k d)`` phase convention: the element positions turned
    by the endpoint orientation, ``u`` the unit direction.  (..., A)."""

    if frequency_hz <= 0.0:
        raise ValueError("frequency_hz must be positive")
    device = direction.device
    positions = endpoint.element_positions.to(device) @ _rotation(endpoint, device).T
    unit = direction.to(torch.float32)
    unit = unit / torch.linalg.vector_norm(unit, dim=-1, keepdim=True).clamp_min(torch.finfo(torch.float32).tiny)
    phase = (2.0 * math.pi * float(frequency_hz) / _LIGHT_SPEED_M_PER_S) * torch.einsum("...c,ac->...a", unit,
                                                                                         positions)
    return torch.exp(1.0j * phase).to(torch.complex64)


def apply_endpoint_weights(coefficients: torch.Tensor, *, tx_weights: torch.Tensor,
                           rx_weights: torch.Tensor) -> torch.Tensor:
    """Combine ``(rx, rx_ant, tx, tx_ant, ...)`` channels with per-endpoint
    weights (reference ``scene/endpoints.py:143-170``): transmit weights as
    given, receive weights conjugated; trailing dimensions kept."""

    if coefficients.ndim < 4:
        raise ValueError("coefficients must have (rx, rx_ant, tx, tx_ant, ...) dimensions")
    expected_tx = (coefficients.shape[2], coefficients.shape[3])
    expected_rx = (coefficients.shape[0], coefficients.shape[1])
    if tx_weights.shape != expected_tx:
        raise ValueError(f"tx_weights must have shape {expected_tx}")
    if rx_weights.shape != expected_rx:
        raise ValueError(f"rx_weights must have shape {expected_rx}")
    tx = tx_weights.to(device=coefficients.device, dtype=torch.complex64)
    rx = rx_weights.to(device=coefficients.device, dtype=torch.complex64)
    tail = (1,) * (coefficients.ndim - 4)
    weighted = coefficients * tx.reshape(1, 1, *expected_tx, *tail)
    weighted = weighted * rx.conj().reshape(*expected_rx, 1, 1, *tail)
    return weighted.sum(dim=3).sum(dim=1)


def _flatten_receivers(receivers: list) -> list:
    out: list = []
    for receiver in receivers:
        out.extend([receiver] * (receiver.count if isinstance(receiver, ReceiverGrid) else 1))
    return out


def _weight_coverage(endpoints: list, attribute: str) -> None:
    values = [getattr(endpoint, attribute, None) for endpoint in endpoints]
    if any(v is None for v in values) and any(v is not None for v in values):
        raise ValueError(f"{attribute} must be configured on every endpoint or none")


def _stack_weights(endpoints: list, attribute: str, device: torch.device) -> torch.Tensor | None:
    values = [getattr(endpoint, attribute, None) for endpoint in endpoints]
    if not values or all(v is None for v in values):
        return None
    _weight_coverage(endpoints, attribute)
    return torch.stack(values).to(device=device, dtype=torch.complex64)


def _antenna_counts(transmitters: list, receivers: list) -> tuple[int, int]:
    tx_counts = {int(getattr(t, "num_antennas", 1)) for t in transmitters}
    rx_counts = {int(getattr(r, "num_antennas", 1)) for r in receivers}
    if len(tx_counts) > 1 or len(rx_counts) > 1:
        raise ValueError("all endpoints on each side must use the same antenna count")
    return next(iter(rx_counts), 1), next(iter(tx_counts), 1)


def validate_synthetic_array_scene(transmitters: list, receivers: list) -> None:
    """Preflight of a synthetic-array solve (reference ``path.py:1200-1212``)."""

    flat = _flatten_receivers(receivers)
    if any(not getattr(e, "synthetic_array", True) for e in (*transmitters, *flat)):
        raise ValueError("explicit arrays require per-element topology tracing")
    _antenna_counts(transmitters, flat)
    _weight_coverage(transmitters, "precoding")
    _weight_coverage(flat, "combining")


def _endpoint_factor(endpoints: list, directions: torch.Tensor, *, frequency_hz: float,
                     conjugate_pattern: bool) -> torch.Tensor:
    """Steering x pattern weights of each endpoint over its own directions
    (``directions[i]`` for ``endpoints[i]``): (endpoint, *batch, A).  Endpoints
    sharing one object (a grid's points) are evaluated in one batch."""

    groups: dict[int, list[int]] = {}
    for index, endpoint in enumerate(endpoints):
        groups.setdefault(id(endpoint), []).append(index)

    def weights(endpoint: Any, sub: torch.Tensor) -> torch.Tensor:
        pattern = pattern_field_response(endpoint.pattern, _local_direction(sub, endpoint))
        if conjugate_pattern:
            pattern = pattern.conj()
        return steering_vector(endpoint, sub, frequency_hz=frequency_hz) * pattern.unsqueeze(-1)

    if len(groups) == 1:
        return weights(endpoints[0], directions)
    num_ant = int(endpoints[0].num_antennas)
    out = torch.empty((len(endpoints), *directions.shape[1:-1], num_ant), dtype=torch.complex64,
                      device=directions.device)
    for indices in groups.values():
        idx = torch.tensor(indices, device=directions.device, dtype=torch.long)
        out.index_copy_(0, idx, weights(endpoints[indices[0]], directions.index_select(0, idx)))
    return out


def _array_metadata(result: PathResult, semantics: str, num_rx_ant: int, num_tx_ant: int) -> dict:
    meta = dict(result.metadata)
    meta.update({"array_semantics": semantics, "num_rx_ant": num_rx_ant, "num_tx_ant": num_tx_ant})
    if semantics.startswith("synthetic"):
        meta["array_phase_convention"] = _ARRAY_PHASE_CONVENTION
    return meta


def pack_synthetic_arrays(result: PathResult, *, frequency_hz: float, transmitters: list,
                          receivers: list) -> PathResult:
    """Expand a centre-endpoint result over synthetic arrays by far-field
    phase weighting (reference ``path.py:1215-1337``): every element shares the
    centre's paths; each path is weighted by the transmit steering and
    pattern at its departure direction and the receive steering and
    conjugate pattern at its arrival (source) direction."""

    if frequency_hz <= 0.0:
        raise ValueError("frequency_hz must be positive")
    flat = _flatten_receivers(receivers)
    if len(transmitters) != result.num_tx or len(flat) != result.num_rx:
        raise ValueError("endpoint counts must match the centre-reference result")
    if result.num_tx_ant != 1 or result.num_rx_ant != 1:
        raise ValueError("synthetic packing requires a single-antenna centre result")
    validate_synthetic_array_scene(transmitters, receivers)
    num_rx_ant, num_tx_ant = _antenna_counts(transmitters, flat)
    device = result.a.device
    tx_weights = _stack_weights(transmitters, "precoding", device)
    rx_weights = _stack_weights(flat, "combining", device)
    meta = _array_metadata(result, "synthetic_far_field_phase_weighting", num_rx_ant, num_tx_ant)
    if result.num_tx == 0 or result.num_rx == 0:
        return replace(result, metadata=meta, tx_weights=tx_weights, rx_weights=rx_weights)
    departure = _unit_vector(result.theta_t[:, 0, :, 0], result.phi_t[:, 0, :, 0])            # (rx, tx, path, 3)
    arrival = _unit_vector(result.theta_r[:, 0, :, 0], result.phi_r[:, 0, :, 0])
    # (tx, rx, path, A_tx) -> (rx, tx, A_tx, path)
    tx_factor = _endpoint_factor(transmitters, departure.transpose(0, 1), frequency_hz=frequency_hz,
                                 conjugate_pattern=False).permute(1, 0, 3, 2)
    # (rx, tx, path, A_rx) -> (rx, A_rx, tx, path)
    rx_factor = _endpoint_factor(flat, arrival, frequency_hz=frequency_hz, conjugate_pattern=True).permute(0, 3, 1, 2)
    factor = rx_factor[:, :, :, None, :] * tx_factor[:, None, :, :, :]

    def expand(value: torch.Tensor) -> torch.Tensor:
        base = value[:, 0, :, 0]
        return base[:, None, :, None].expand(result.num_rx, num_rx_ant, result.num_tx, num_tx_ant,
                                             *base.shape[2:]).contiguous()

    return replace(
        result, a=(expand(result.a) * factor.unsqueeze(-1)).to(torch.complex64), tau=expand(result.tau),
        theta_t=expand(result.theta_t), phi_t=expand(result.phi_t), theta_r=expand(result.theta_r),
        phi_r=expand(result.phi_r), valid=expand(result.valid), interaction_type=expand(result.interaction_type),
        primitive_id=expand(result.primitive_id), material_id=expand(result.material_id),
        position=expand(result.position), normal=expand(result.normal), num_paths=expand(result.num_paths),
        metadata=meta, field_xyz=(expand(result.field_xyz) * factor.unsqueeze(-1)).to(torch.complex64),
        field_direction=expand(result.field_direction), tx_weights=tx_weights, rx_weights=rx_weights)


class _ElementEndpoints:
    """The endpoints of an explicit-array solve: one single-element endpoint
    per array element, at its world position, keeping the endpoint's world
    polarization and power (reference ``path.py:1340-1387``)."""

    def __init__(self, transmitters: list, receivers: list) -> None:
        if any(isinstance(r, ReceiverGrid) for r in receivers):
            raise ValueError("explicit arrays currently require point receivers")

        def expand(endpoint: Any, role: str) -> list:
            return [AntennaState(endpoint.id, role, p, polarization=endpoint.polarization,
                                 power_w=getattr(endpoint, "power_w", 1.0))
                    for p in endpoint.element_world_positions(endpoint.position)]

        self.transmitters = [e for t in transmitters for e in expand(t, "tx")]
        self.receivers = [e for r in receivers for e in expand(r, "rx")]


def pack_explicit_arrays(result: PathResult, *, transmitters: list, receivers: list, num_rx_ant: int,
                         num_tx_ant: int) -> PathResult:
    """Fold per-element endpoints back into antenna dimensions and apply the
    element patterns at each element's own departure / arrival directions
    (reference ``path.py:1390-1454``)."""

    num_rx, num_tx = len(receivers), len(transmitters)
    if result.num_rx != num_rx * num_rx_ant or result.num_tx != num_tx * num_tx_ant:
        raise ValueError("expanded explicit result does not match endpoint array layout")

    def fold(value: torch.Tensor) -> torch.Tensor:
        base = value[:, 0, :, 0]
        return base.reshape(num_rx, num_rx_ant, num_tx, num_tx_ant, *base.shape[2:])

    theta_t, phi_t, theta_r, phi_r = (fold(result.theta_t), fold(result.phi_t), fold(result.theta_r),
                                      fold(result.phi_r))
    factor = torch.ones_like(theta_t, dtype=torch.complex64)
    departure = _unit_vector(theta_t, phi_t)
    arrival = _unit_vector(theta_r, phi_r)
    for tx_id, transmitter in enumerate(transmitters):
        factor[:, :, tx_id] *= pattern_field_response(transmitter.pattern,
                                                      _local_direction(departure[:, :, tx_id], transmitter))
    for rx_id, receiver in enumerate(receivers):
        factor[rx_id] *= pattern_field_response(receiver.pattern, _local_direction(arrival[rx_id], receiver)).conj()
    device = result.a.device
    return replace(
        result, a=(fold(result.a) * factor.unsqueeze(-1)).contiguous(), tau=fold(result.tau), theta_t=theta_t,
        phi_t=phi_t, theta_r=theta_r, phi_r=phi_r, valid=fold(result.valid),
        interaction_type=fold(result.interaction_type), primitive_id=fold(result.primitive_id),
        material_id=fold(result.material_id), position=fold(result.position), normal=fold(result.normal),
        num_paths=fold(result.num_paths),
        metadata=_array_metadata(result, "explicit_per_element_topology", num_rx_ant, num_tx_ant),
        field_xyz=(fold(result.field_xyz) * factor.unsqueeze(-1)).contiguous(),
        field_direction=fold(result.field_direction),
        tx_weights=_stack_weights(transmitters, "precoding", device),
        rx_weights=_stack_weights(receivers, "combining", device))


def solve(scene: Any, config: Config, *, reference_frequency_hz) -> PathResult:
    """Canonical paths of every (rx, tx) pair packed per pair (reference
    ``path.py:1551-1721``): the native row-mode solve, selection with the
    per-pair limit, row field evaluation, then the ragged and padded
    packing of ``from_evaluated_paths`` (``path.py:887-975``).  Antenna
    arrays (reference ``_pipeline_solve``, ``path.py:1654-1681``): synthetic
    arrays share the centre endpoints' paths and are expanded by far-field
    phase weighting; if any endpoint's array is explicit, every element is
    traced as its own endpoint."""
    if not isinstance(config, Config):
        raise TypeError("config must be a witwin_channel_b200.path.Config")
    frequency = _frequency_value(reference_frequency_hz)
    transmitters, receivers = list(scene.transmitters), list(scene.receivers)
    # array preflight before any device work
    explicit = any(not getattr(e, "synthetic_array", True) for e in (*transmitters, *receivers))
    if explicit:
        if any(isinstance(r, ReceiverGrid) for r in receivers):
            raise ValueError("explicit arrays currently require point receivers")
        num_rx_ant, num_tx_ant = _antenna_counts(transmitters, receivers)
        _weight_coverage(transmitters, "precoding")
        _weight_coverage(receivers, "combining")
    else:
        validate_synthetic_array_scene(transmitters, receivers)
    _validate(scene, config)
    if explicit:
        elements = _ElementEndpoints(transmitters, receivers)
        base = _solve_base(scene, config, frequency, elements, reference_frequency_hz)
        return pack_explicit_arrays(base, transmitters=transmitters, receivers=receivers, num_rx_ant=num_rx_ant,
                                    num_tx_ant=num_tx_ant)
    base = _solve_base(scene, config, frequency, scene, reference_frequency_hz)
    return pack_synthetic_arrays(base, frequency_hz=frequency, transmitters=transmitters, receivers=receivers)


def _solve_base(scene: Any, config: Config, frequency: float, endpoints: Any, frequency_input: Any = None) -> PathResult:
    """One centre-endpoint solve of ``scene``'s geometry between the
    endpoints of ``endpoints`` (``.transmitters`` / ``.receivers``).  With
    ``config.ad_mode`` "vjp" / "jvp" the coefficients carry the records'
    fixed-topology derivatives (vertices, materials, a tensor frequency, the
    endpoint positions)."""
    device = torch.device("cuda", torch.cuda.current_device())
    compiled = compile_scene(scene, device)
    ep = _endpoints(endpoints, device)
    mats = compiled.material_tables([frequency], device)
    bits = engine.component_bits(config.components)
    width = max(int(config.max_depth), 0)
    launches0 = _native.launch_count()
    res = engine.run_solve(compiled, ep, mats, [frequency], components=bits, max_depth=config.max_depth,
                           coherent=True, want_rows=True)
    rows = res["rows"]
    selected = engine.select_rows(rows, width, config.max_paths, "per_pair")
    ev = engine.evaluate_rows(compiled, ep, mats, [frequency], 0, rows, selected, width, components=bits,
                              max_depth=config.max_depth, coherent=True)
    dec = engine.decode_rows(rows, selected)
    K = int(selected.shape[0])
    cid = dec["component_id"].to(torch.int64)
    depth = dec["depth"].to(torch.int64)
    tx_id = dec["tx_id"].to(torch.int64)
    rx_id = dec["rx_id"].to(torch.int64)
    # interaction types: one event per bounce of the row's component
    kind = torch.zeros_like(cid)
    for c, v in _INTERACTION_OF_COMPONENT.items():
        kind = torch.where(cid == c, torch.full_like(cid, v), kind)
    step = torch.arange(width, device=device, dtype=torch.int64).view(1, -1)
    types = torch.where(step < depth.view(-1, 1), kind.view(-1, 1), torch.zeros_like(step)).to(torch.int32)
    faces = dec["seq"][:, :width].to(torch.int64)
    # materials of the face events (reflection, transmission); an index is
    # formed only for real face ids, so no lookup leaves the table
    fm = compiled.face_material.to(device=device, dtype=torch.int32)
    is_face = (types != 0) & (types != int(InteractionType.DIFFRACTION)) & (faces >= 0) & (faces < fm.numel())
    if fm.numel() and width:
        mat_seq = torch.where(is_face, fm[torch.where(is_face, faces, torch.zeros_like(faces))],
                              torch.full_like(types, -1))
    else:
        mat_seq = torch.full_like(types, -1)
    seq = faces.to(torch.int32).clone()
    if width:
        diff = (cid == 2) & (depth > 0)
        seq[diff, 0] = dec["edge_id"].to(torch.int32)[diff]
    pos = ev["interaction_positions"][:, :width].contiguous()
    nrm = ev["interaction_normals"][:, :width].contiguous()
    nrm = torch.where(torch.isfinite(nrm), nrm, torch.zeros_like(nrm))
    # departure / arrival angles from the endpoints and the first / last event
    tx_pos = ep.tx_pos
    rx_pos = _receiver_positions(endpoints, ep.rx, device)
    tp = tx_pos[tx_id] if K else torch.zeros((0, 3), device=device)
    rp = rx_pos[rx_id] if K else torch.zeros((0, 3), device=device)
    direct = rp - tp
    if width and K:
        first = pos[:, 0]
        last = pos[torch.arange(K, device=device), (depth - 1).clamp_min(0)]
        has = (depth > 0).view(-1, 1)
        departure = torch.where(has, first - tp, direct)
        arrival = torch.where(has, rp - last, direct)
    else:
        departure, arrival = direct, direct
    theta_t, phi_t = endpoint_angles(departure)
    theta_r, phi_r = endpoint_angles(-arrival)
    num_tx, num_rx = int(ep.num_tx), int(ep.num_rx)
    coefficient = ev["coefficient"]
    if config.ad_mode != "none" and K:
        from .autograd import differentiable_row_fields, unit_coefficient

        def stack(items: list) -> torch.Tensor:
            return torch.stack([e.position.reshape(3).to(device=device, dtype=torch.float64) for e in items]) \
                if items else torch.zeros((0, 3), dtype=torch.float64, device=device)

        rx_input = stack(list(endpoints.receivers)) if ep.rx["kind"] != "grid" else None
        pf = differentiable_row_fields(scene, compiled, ep, mats, frequency, frequency_input, bits,
                                       config.max_depth, rows, selected, ev["path_field"],
                                       tx=stack(list(endpoints.transmitters)), rx=rx_input)
        coefficient = unit_coefficient(coefficient, pf, ep.tx_power.index_select(0, tx_id))
    ragged = RaggedPathSoA.from_flat(
        num_rx=num_rx, num_rx_ant=1, num_tx=num_tx, num_tx_ant=1, rx_id=rx_id, tx_id=tx_id,
        field=coefficient.unsqueeze(-1), delay_s=ev["delay_s"], theta_t=theta_t, phi_t=phi_t,
        theta_r=theta_r, phi_r=phi_r, interaction_type=types, primitive_id=seq, material_id=mat_seq, position=pos,
        normal=nrm)
    counts = {name: int((cid == c).sum().item()) for name, c in
              (("los", 0), ("reflection", 1), ("diffraction", 2), ("transmission", 5))}
    meta = {
        "solver": "path",
        "device": "cuda",
        "path_count": K,
        "effective_max_depth": width,
        "max_paths_per_pair": config.max_paths,
        "components": {c: ("enabled" if c in config.components else "not_requested") for c in sorted(VALID_COMPONENTS)},
        "component_counts": counts,
        "kernel": {"primitive": "path_solver", "forward_launch_count": _native.launch_count() - launches0,
                   "scheduling_strategy": "native_cuda", "ad_status": config.ad_mode},
        "field_abi": "complex3_v1",
        "phase_convention": dict(PHASE_CONVENTION),
        "coefficient_semantics": "unit_excitation_dimensionless_receiver_projection",
        "interaction_geometry": "canonical_topology",
        "array_semantics": "single_antenna_endpoints",
        "num_rx_ant": 1,
        "num_tx_ant": 1,
    }
    if "transmission" in config.components:
        meta["transmission"] = {"thin_sheet_straight_path_approximation": True, "group_delay": "geometric"}
    result = PathResult.from_ragged(ragged, metadata=meta)
    field_xyz = torch.zeros((*result.path_shape, 3), device=device, dtype=torch.complex64)
    field_direction = torch.zeros((*result.path_shape, 3), device=device, dtype=torch.float32)
    if K:
        # from_flat sorted the records by pair; the same stable order maps the row fields
        order = torch.argsort(rx_id * max(num_tx, 1) + tx_id, stable=True)
        field_xyz[result.valid] = ev["field_xyz"][order]
        field_direction[result.valid] = ev["field_direction"][order]
    return replace(result, field_xyz=field_xyz, field_direction=field_direction)


__all__ = ["Config", "InteractionType", "PathResult", "RaggedPathSoA", "apply_endpoint_weights",
           "pack_explicit_arrays", "pack_synthetic_arrays", "pattern_field_response", "solve", "steering_vector",
           "validate_synthetic_array_scene"]
