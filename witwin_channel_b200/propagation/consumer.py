"""Propagation consumer boundary (``witwin.channel.propagation.consumer``).

Restates the reference's solver-neutral consumer contract
(``witwin/channel/propagation/consumer.py``): the vocabulary (``:415-439``),
``EndpointBatch`` (``:515-588``), ``PropagationRequest`` (``:623-654``), the
compact row records ``PropagationTopology``, ``PropagationGeometry``,
``ScalarTransport``, ``Complex3Transport``, ``JonesTransport`` and
``PropagationPathBatch`` (``:656-960``), ``PropagationConvention``
(``:963-1006``), ``PropagationCapabilities`` with ``capabilities()``
(``:1008-1190``), ``PropagationDiagnostics`` and ``PropagationEvaluation``
(``:1192-1225``), and discovery ``evaluate`` (``:3478-3520``).

Rows come from the native engine in ``libwcb200.so``: row-mode discovery of
every (source, sink) pair, canonical selection with the request's global path
limit, and row field evaluation.  They are published in the sink-major,
source-minor pair order (``pair_index = sink_index * source_count +
source_index``), and rows of one pair keep the canonical order.  The packing
is index arithmetic on device tensors.

What this engine advertises is what it does: components LoS, reflection,
transmission and diffraction; the scalar and complex3 responses, and the
polarimetric (LoS Jones) response through the native ``wcb_los_jones``
(``consumer_los_jones``, ``:2037-2093``).

Fixed-topology replay (``prepare_fixed_topology``, ``replicate_over_slots``,
``reevaluate``, ``rediscovery_required``, ``evaluate_time_varying``;
reference ``:1228-1784, 3523-4342``) re-evaluates frozen LoS and reflection
rows at new endpoint positions through one native ``wcb_rows_replay``
launch: every row and every wideband frequency column in one pass, the
contract validation folded into the same launch, one 8-byte status read per
call.

AD: ``ad_mode`` "vjp" and "jvp" differentiate the scalar coefficient and the
complex3 field on both routes (source and sink positions, vertices, eps_r /
sigma_e and a tensor frequency) through the native fixed-topology VJP / JVP
of the rows' records; the Jones operator, the wideband columns and the
geometry outputs are primal-only, and requests that need them differentiated
fail before any native work.
"""

from __future__ import annotations

import math
from dataclasses import dataclass
from typing import Any, Literal, TypeAlias, get_args

import torch

from .. import _native, engine
from .. import autograd as _ad
from ..compiler import CompiledScene
from ..constants import (
    NARROWBAND_FREQUENCY_OFFSET_ERROR_LAW,
    NARROWBAND_FREQUENCY_OFFSET_LAW,
    PHASOR,
    TIME_DEPENDENCE,
)
from ..deterministic import _frequency_value, _path_table

# --- The published vocabulary (reference consumer.py:415-455) ---------------

CONTRACT_VERSION = 6

PropagationComponent: TypeAlias = Literal["los", "reflection", "transmission", "diffraction"]
PropagationResponse: TypeAlias = Literal["scalar_transport", "complex3_transport", "polarimetric_transport"]
PropagationTopologyMode: TypeAlias = Literal["discover"]
PropagationAdMode: TypeAlias = Literal["none", "jvp", "vjp"]
PropagationWorldMotion: TypeAlias = Literal["frozen_world", "fixed_winner_replay"]

COMPONENTS: frozenset[str] = frozenset(get_args(PropagationComponent))
RESPONSES: frozenset[str] = frozenset(get_args(PropagationResponse))
TOPOLOGY_MODES: frozenset[str] = frozenset(get_args(PropagationTopologyMode))
AD_MODES: frozenset[str] = frozenset(get_args(PropagationAdMode))
WORLD_MOTIONS: frozenset[str] = frozenset(get_args(PropagationWorldMotion))

MAX_DEPTH = 5

WORLD_VERSION_DOMAINS: tuple[str, ...] = (
    "topology_version",
    "material_version",
    "assignment_version",
    "geometry_version",
)

# What this engine produces (a subset of the vocabulary above); the
# polarimetric (Jones) response is line-of-sight only, as in the reference.
_SUPPORTED_RESPONSES: frozenset[str] = RESPONSES
_RESPONSE_COMPONENTS: tuple[tuple[str, frozenset[str]], ...] = (
    ("complex3_transport", COMPONENTS),
    ("polarimetric_transport", frozenset({"los"})),
    ("scalar_transport", COMPONENTS),
)
_SUPPORTED_AD_MODES: frozenset[str] = frozenset({"none"})

# The material values the native derivative kernels differentiate; the
# others (permeabilities, thicknesses, gains) are primal-only here.
_DIFFERENTIABLE_MATERIAL_LEAVES: frozenset[str] = frozenset(
    {"materials.eps_r", "materials.sigma_e", "materials.layer_eps_r", "materials.layer_sigma_e"})

# Components a frozen topology may carry into replay, with the discovery
# encoding of their component id (reference consumer.py:211-214).
_FIXED_TOPOLOGY_COMPONENT_IDS: tuple[tuple[str, int], ...] = (("los", 0), ("reflection", 1))

_COMPONENT_MATERIAL_LEAVES: tuple[tuple[str, tuple[str, ...]], ...] = (
    ("diffraction", ("eps_r", "sigma_e", "thickness_m", "gain")),
    ("los", ()),
    ("reflection", ("eps_r", "sigma_e", "thickness_m", "gain")),
    ("transmission", ("layer_eps_r", "layer_sigma_e", "layer_thickness_m")),
)

_PRIMAL_ONLY_AD_INPUTS: tuple[str, ...] = (
    "materials.gain",
    "materials.layer_mu_r",
    "materials.layer_thickness_m",
    "materials.mu_r",
    "materials.thickness_m",
    "sinks.polarization_basis",
    "sinks.polarizations",
    "sources.polarization_basis",
    "sources.polarizations",
    "sources.powers_w",
)

# The kernels take each frequency as a float64 (C ABI ``frequency_hz``), so
# two absolute frequencies are the same launch only inside one float64 ULP.
NATIVE_FREQUENCY_RESOLUTION_LAW = "resolution_hz = ulp_float64(reference_frequency_hz)"

WIDEBAND_OFFSET_LAYOUT = (
    "frequency_minor:"
    "payload[row, j] = response(row) at"
    " reference_frequency_hz+frequency_offsets_hz[j];"
    "row axis and pair segmentation unchanged;"
    "row_valid stays [K] and broadcasts over j;"
    "geometry published once from the reference evaluation;"
    "slot composition gives [slot_count*frozen_row_count, F]"
)
WIDEBAND_FREQUENCY_QUANTIZATION_LAW = (
    "launch_grid=float64;"
    " resolution_hz=ulp_float64(reference_frequency_hz);"
    " abs_phase_error_rad <= pi*resolution_hz*delay_s"
)


def require_frequency_offsets(value: object) -> tuple[float, ...] | None:
    """Structural check of a wideband offset grid (reference ``consumer.py:94-135``):
    ``None`` or a non-empty tuple of distinct finite host floats."""

    if value is None:
        return None
    if isinstance(value, torch.Tensor):
        raise TypeError("frequency_offsets_hz must be a tuple of host floats, not a torch.Tensor: the offset grid "
                        "declares which absolute frequencies to evaluate and is not a differentiable input")
    if not isinstance(value, tuple):
        raise TypeError("frequency_offsets_hz must be a tuple of floats or None")
    if not value:
        raise ValueError("frequency_offsets_hz must be a non-empty tuple; pass None for a single-frequency request")
    offsets = []
    for entry in value:
        if isinstance(entry, bool) or not isinstance(entry, (int, float)):
            raise TypeError("frequency_offsets_hz entries must be floats")
        offset = float(entry)
        if not math.isfinite(offset):
            raise ValueError(f"frequency_offsets_hz entries must be finite, got {entry!r}")
        offsets.append(offset)
    if len(set(offsets)) != len(offsets):
        raise ValueError("frequency_offsets_hz must not repeat an offset; duplicate entries produce bit-identical "
                         "columns and hide a caller bug")
    return tuple(offsets)


def require_wideband_payload(name: str, payload: object, offsets: object, reference: torch.Tensor) -> None:
    """Paired presence and shape of a wideband payload (reference ``consumer.py:138-173``):
    the payload and its offset grid are both present or both absent, and the
    payload is the reference tensor with a frequency axis after the row axis."""

    if payload is None and offsets is None:
        return
    if payload is None or offsets is None:
        raise ValueError(f"{name} and frequency_offsets_hz are paired: publish both or neither")
    if not isinstance(offsets, tuple) or not offsets:
        raise TypeError("frequency_offsets_hz must be a non-empty tuple of floats")
    if not isinstance(payload, torch.Tensor):
        raise TypeError(f"{name} must be a torch.Tensor")
    if payload.dtype != reference.dtype:
        raise TypeError(f"{name} must use {reference.dtype}, got {payload.dtype}")
    expected = (int(reference.shape[0]), len(offsets), *reference.shape[1:])
    if tuple(payload.shape) != expected:
        raise ValueError(f"{name} must have shape {expected}, got {tuple(payload.shape)}")
    if payload.device != reference.device:
        raise ValueError(f"{name} must be on {reference.device}, got {payload.device}")


def native_frequency_resolution_hz(reference_frequency_hz: float) -> float:
    """The smallest frequency step the native launches resolve at ``reference_frequency_hz``."""

    value = float(reference_frequency_hz)
    if not (value > 0.0 and math.isfinite(value)):
        raise ValueError("reference_frequency_hz must be a positive finite float")
    return math.ulp(value)


# --- Structural checks --------------------------------------------------------


def _require_tensor(name: str, value: object, *, dtype: torch.dtype, ndim: int | None = None,
                    shape: tuple[int, ...] | None = None, device: torch.device | None = None) -> torch.Tensor:
    """The consumer boundary's tensor check: a wrong type or dtype is a
    TypeError, a wrong rank, shape or device a ValueError."""

    if not isinstance(value, torch.Tensor):
        raise TypeError(f"{name} must be a torch.Tensor")
    if value.dtype != dtype:
        raise TypeError(f"{name} must have dtype {dtype}, got {value.dtype}")
    if ndim is not None and value.ndim != ndim:
        raise ValueError(f"{name} must have {ndim} dimensions, got {value.ndim}")
    if shape is not None and tuple(value.shape) != tuple(shape):
        raise ValueError(f"{name} must have shape {tuple(shape)}, got {tuple(value.shape)}")
    if device is not None and value.device != device:
        raise ValueError(f"{name} must be on {device}, got {value.device}")
    return value


def _require_vocabulary(name: str, value: object, allowed: frozenset[str]) -> str:
    if not isinstance(value, str):
        raise TypeError(f"{name} must be a string")
    if value not in allowed:
        raise NotImplementedError(f"unsupported {name} {value!r}; supported values are {sorted(allowed)}")
    return value


def _require_components(value: object) -> frozenset[str]:
    if type(value) is not frozenset or not value:
        raise TypeError("components must be a non-empty frozenset")
    unsupported = value - COMPONENTS
    if unsupported:
        raise NotImplementedError(f"unsupported propagation components: {sorted(unsupported)}")
    return value


# --- Request records ------------------------------------------------------------


@dataclass(frozen=True, slots=True, eq=False)
class EndpointBatch:
    """Explicit point endpoints of one request (reference ``consumer.py:515-588``).

    ``powers_w`` is required on a source batch and absent on a sink batch;
    ``polarization_basis`` holds two world-Cartesian reference vectors per
    endpoint (used by the polarimetric response only)."""

    stable_ids: torch.Tensor
    positions_m: torch.Tensor
    polarizations: torch.Tensor
    polarization_basis: torch.Tensor | None = None
    powers_w: torch.Tensor | None = None

    def __post_init__(self) -> None:
        positions = _require_tensor("positions_m", self.positions_m, dtype=torch.float32, ndim=2)
        if positions.shape[1:] != (3,):
            raise ValueError("positions_m must have shape (N, 3)")
        if positions.device.type != "cuda":
            raise ValueError("endpoint tensors must be CUDA tensors")
        rows = int(positions.shape[0])
        device = positions.device
        _require_tensor("stable_ids", self.stable_ids, dtype=torch.int64, shape=(rows,), device=device)
        _require_tensor("polarizations", self.polarizations, dtype=torch.float32, shape=(rows, 3), device=device)
        if self.polarization_basis is not None:
            _require_tensor("polarization_basis", self.polarization_basis, dtype=torch.float32, shape=(rows, 2, 3),
                            device=device)
        if self.powers_w is not None:
            _require_tensor("powers_w", self.powers_w, dtype=torch.float32, shape=(rows,), device=device)
        for name in ("stable_ids", "positions_m", "polarizations", "polarization_basis", "powers_w"):
            value = getattr(self, name)
            if value is not None and not value.is_contiguous():
                raise ValueError(f"{name} must be contiguous")

    @property
    def count(self) -> int:
        return int(self.positions_m.shape[0])

    @property
    def device(self) -> torch.device:
        return self.positions_m.device


def _require_endpoints(sources: object, sinks: object) -> None:
    if not isinstance(sources, EndpointBatch) or not isinstance(sinks, EndpointBatch):
        raise TypeError("sources and sinks must be EndpointBatch instances")
    if sources.powers_w is None:
        raise ValueError("sources.powers_w is required")
    if sinks.powers_w is not None:
        raise ValueError("sinks.powers_w must be absent")
    if sources.device != sinks.device:
        raise ValueError("source and sink batches must share one CUDA device")


@dataclass(frozen=True, slots=True)
class PropagationRequest:
    """A discovery request against a compiled scene (reference
    ``consumer.py:623-654``).  Structure is checked here; what depends on the
    engine (response, AD mode) is checked by :func:`evaluate` before any
    native work."""

    sources: EndpointBatch
    sinks: EndpointBatch
    reference_frequency_hz: float | torch.Tensor
    components: frozenset[str]
    max_depth: int
    response: PropagationResponse
    topology_mode: PropagationTopologyMode
    ad_mode: PropagationAdMode
    max_paths: int | None = None

    def __post_init__(self) -> None:
        _require_endpoints(self.sources, self.sinks)
        _require_components(self.components)
        _require_vocabulary("response", self.response, RESPONSES)
        _require_vocabulary("topology_mode", self.topology_mode, TOPOLOGY_MODES)
        _require_vocabulary("ad_mode", self.ad_mode, AD_MODES)
        if type(self.max_depth) is not int or not 0 <= self.max_depth <= MAX_DEPTH:
            raise ValueError(f"max_depth must be an int in [0, {MAX_DEPTH}]")
        if self.max_paths is not None and (type(self.max_paths) is not int or self.max_paths <= 0):
            raise ValueError("max_paths must be a positive int when set")


# --- World provenance -------------------------------------------------------------


@dataclass(frozen=True, slots=True, eq=False)
class WorldProvenance:
    """Which world a discovered topology belongs to (reference ``consumer.py:466-512``).

    The four version domains the compiled scene recorded: ``topology_version``
    (face tables and structure layout), ``geometry_version`` (an epoch of the
    vertex positions, new at every compile and in-place refit),
    ``material_version`` (the material values) and ``assignment_version`` (the
    face -> material / surface assignment).  ``time_s`` is carried for
    reporting only and never compared."""

    topology_version: int
    geometry_version: int
    material_version: int
    assignment_version: int
    time_s: float | torch.Tensor | None = None

    @classmethod
    def of(cls, compiled: Any) -> WorldProvenance:
        """Read the four version domains of a compiled scene."""

        return cls(topology_version=int(compiled.topology_version), geometry_version=int(compiled.geometry_version),
                   material_version=int(compiled.material_version),
                   assignment_version=int(compiled.assignment_version), time_s=getattr(compiled, "time_s", None))

    def moved_domain(self, current: WorldProvenance, *, allow_geometry: bool = False) -> str | None:
        """Name the first version domain that differs from ``current``, or ``None``."""

        for name in WORLD_VERSION_DOMAINS:
            if allow_geometry and name == "geometry_version":
                continue
            if getattr(self, name) != getattr(current, name):
                return name
        return None


# --- Result records -------------------------------------------------------------


@dataclass(frozen=True, slots=True, eq=False)
class PropagationTopology:
    """Compact discrete rows in pair-major order (reference ``consumer.py:656-737``).

    ``provenance`` is the :class:`WorldProvenance` of the compiled scene the
    rows were discovered against; a hand-built topology leaves it ``None`` and
    has no world to be stale against."""

    source_index: torch.Tensor
    sink_index: torch.Tensor
    source_id: torch.Tensor
    sink_id: torch.Tensor
    depth: torch.Tensor
    component_id: torch.Tensor
    primitive_id: torch.Tensor
    edge_id: torch.Tensor
    material_id: torch.Tensor
    primitive_sequence: torch.Tensor
    material_sequence: torch.Tensor
    interaction_type: torch.Tensor
    provenance: Any = None

    def __post_init__(self) -> None:
        source_index = _require_tensor("source_index", self.source_index, dtype=torch.int32, ndim=1)
        rows = int(source_index.shape[0])
        device = source_index.device
        for name in ("sink_index", "depth", "component_id", "primitive_id", "edge_id", "material_id"):
            _require_tensor(name, getattr(self, name), dtype=torch.int32, shape=(rows,), device=device)
        for name in ("source_id", "sink_id"):
            _require_tensor(name, getattr(self, name), dtype=torch.int64, shape=(rows,), device=device)
        sequence = _require_tensor("primitive_sequence", self.primitive_sequence, dtype=torch.int32, ndim=2,
                                   device=device)
        shape = tuple(sequence.shape)
        if shape[0] != rows:
            raise ValueError("primitive_sequence must share compact rows")
        for name in ("material_sequence", "interaction_type"):
            _require_tensor(name, getattr(self, name), dtype=torch.int32, shape=shape, device=device)

    @property
    def row_count(self) -> int:
        return int(self.source_index.shape[0])

    @property
    def device(self) -> torch.device:
        return self.source_index.device


@dataclass(frozen=True, slots=True, eq=False)
class PropagationGeometry:
    """Continuous SI geometry of one compact topology (reference ``consumer.py:740-793``)."""

    path_length_m: torch.Tensor
    delay_s: torch.Tensor
    field_direction: torch.Tensor
    interaction_positions_m: torch.Tensor
    interaction_normals: torch.Tensor

    def __post_init__(self) -> None:
        length = _require_tensor("path_length_m", self.path_length_m, dtype=torch.float32, ndim=1)
        rows = int(length.shape[0])
        device = length.device
        _require_tensor("delay_s", self.delay_s, dtype=torch.float32, shape=(rows,), device=device)
        _require_tensor("field_direction", self.field_direction, dtype=torch.float32, shape=(rows, 3), device=device)
        positions = _require_tensor("interaction_positions_m", self.interaction_positions_m, dtype=torch.float32,
                                    ndim=3, device=device)
        if positions.shape[0] != rows or positions.shape[2] != 3:
            raise ValueError("interaction_positions_m must have shape (K, depth, 3)")
        _require_tensor("interaction_normals", self.interaction_normals, dtype=torch.float32,
                        shape=tuple(positions.shape), device=device)

    @property
    def row_count(self) -> int:
        return int(self.path_length_m.shape[0])

    @property
    def device(self) -> torch.device:
        return self.path_length_m.device


@dataclass(frozen=True, slots=True, eq=False)
class ScalarTransport:
    """Receiver-projected complex transport at the reference frequency,
    carrying the source amplitude ``sqrt(powers_w)`` (reference
    ``consumer.py:796-833``).  A fixed-topology replay with
    ``frequency_offsets_hz`` adds ``coefficient_offsets`` ``[K, F]``, column
    ``j`` at ``reference_frequency_hz + frequency_offsets_hz[j]``."""

    coefficient: torch.Tensor
    coefficient_offsets: torch.Tensor | None = None
    frequency_offsets_hz: tuple[float, ...] | None = None

    def __post_init__(self) -> None:
        _require_tensor("coefficient", self.coefficient, dtype=torch.complex64, ndim=1)
        require_wideband_payload("coefficient_offsets", self.coefficient_offsets, self.frequency_offsets_hz,
                                 self.coefficient)

    @property
    def row_count(self) -> int:
        return int(self.coefficient.shape[0])

    @property
    def device(self) -> torch.device:
        return self.coefficient.device


@dataclass(frozen=True, slots=True, eq=False)
class Complex3Transport:
    """World-Cartesian complex field at the sink, carrying ``sqrt(powers_w)``,
    and the arrival direction (reference ``consumer.py:836-875``).  Projecting
    ``field`` on the sink polarization gives :attr:`ScalarTransport.coefficient`.
    A wideband replay adds ``field_offsets`` ``[K, F, 3]``."""

    field: torch.Tensor
    direction: torch.Tensor
    field_offsets: torch.Tensor | None = None
    frequency_offsets_hz: tuple[float, ...] | None = None

    def __post_init__(self) -> None:
        field = _require_tensor("field", self.field, dtype=torch.complex64, ndim=2)
        if field.shape[1:] != (3,):
            raise ValueError("field must have shape (K, 3)")
        _require_tensor("direction", self.direction, dtype=torch.float32, shape=(int(field.shape[0]), 3),
                        device=field.device)
        require_wideband_payload("field_offsets", self.field_offsets, self.frequency_offsets_hz, self.field)

    @property
    def row_count(self) -> int:
        return int(self.field.shape[0])

    @property
    def device(self) -> torch.device:
        return self.field.device


@dataclass(frozen=True, slots=True, eq=False)
class JonesTransport:
    """Source-basis to sink-basis complex 2 x 2 operator (reference
    ``consumer.py:878-913``): ``matrix[k, i, j]`` is the response of sink
    basis vector ``i`` to source basis vector ``j`` at unit excitation (no
    transmitter power, no antenna pattern)."""

    matrix: torch.Tensor
    source_basis: torch.Tensor
    sink_basis: torch.Tensor

    def __post_init__(self) -> None:
        matrix = _require_tensor("matrix", self.matrix, dtype=torch.complex64, ndim=3)
        if matrix.shape[1:] != (2, 2):
            raise ValueError("matrix must have shape (K, 2, 2)")
        rows = int(matrix.shape[0])
        for name in ("source_basis", "sink_basis"):
            _require_tensor(name, getattr(self, name), dtype=torch.float32, shape=(rows, 2, 3), device=matrix.device)

    @property
    def row_count(self) -> int:
        return int(self.matrix.shape[0])

    @property
    def device(self) -> torch.device:
        return self.matrix.device


PropagationTransport: TypeAlias = ScalarTransport | Complex3Transport | JonesTransport


@dataclass(frozen=True, slots=True, eq=False)
class PropagationPathBatch:
    """The compact ``K`` rows with their pair segmentation (reference
    ``consumer.py:919-960``): rows of pair ``p`` are
    ``pair_offsets[p]:pair_offsets[p + 1]``."""

    pair_count: int
    path_count: int
    pair_index: torch.Tensor
    pair_offsets: torch.Tensor
    topology: PropagationTopology
    geometry: PropagationGeometry
    transport: PropagationTransport

    def __post_init__(self) -> None:
        if type(self.pair_count) is not int or self.pair_count < 0:
            raise ValueError("pair_count must be a non-negative int")
        if type(self.path_count) is not int or self.path_count < 0:
            raise ValueError("path_count must be a non-negative int")
        pair_index = _require_tensor("pair_index", self.pair_index, dtype=torch.int64, shape=(self.path_count,))
        _require_tensor("pair_offsets", self.pair_offsets, dtype=torch.int64, shape=(self.pair_count + 1,),
                        device=pair_index.device)
        for name in ("topology", "geometry", "transport"):
            part = getattr(self, name)
            if part.row_count != self.path_count:
                raise ValueError(f"{name} must have exactly path_count rows")
            if part.device != pair_index.device:
                raise ValueError("all path tensors must share one device")


@dataclass(frozen=True, slots=True)
class PropagationConvention:
    """Units, phase and layout conventions of the published rows (reference
    ``consumer.py:963-1006``)."""

    contract_version: int = CONTRACT_VERSION
    pair_layout: str = "sink_major_source_minor:pair_index=sink_index*source_count+source_index"
    slot_pair_layout: str = (
        "block_diagonal_slots:"
        "row=slot*frozen_row_count+frozen_row;"
        "source_index=slot*slot_source_count+slot_source_index;"
        "sink_index=slot*slot_sink_count+slot_sink_index;"
        "pair_index=slot*slot_source_count*slot_sink_count"
        "+slot_sink_index*slot_source_count+slot_source_index;"
        "pair_count=slot_count*slot_source_count*slot_sink_count"
    )
    distance_unit: str = "m"
    delay_unit: str = "s"
    phasor: str = PHASOR
    time_dependence: str = TIME_DEPENDENCE
    coefficient_reference: str = "includes_reference_frequency_phase"
    narrowband_frequency_offset_law: str = NARROWBAND_FREQUENCY_OFFSET_LAW
    narrowband_frequency_offset_error_law: str = NARROWBAND_FREQUENCY_OFFSET_ERROR_LAW
    wideband_offset_layout: str = WIDEBAND_OFFSET_LAYOUT
    wideband_frequency_quantization_law: str = WIDEBAND_FREQUENCY_QUANTIZATION_LAW
    complex3_basis: str = "world_cartesian"
    jones_mapping: str = "source_transverse_basis_to_sink_transverse_basis"


@dataclass(frozen=True, slots=True)
class PropagationCapabilities:
    """What this engine supports, discoverable before a request is built
    (reference ``consumer.py:1008-1116``; same fields)."""

    contract_version: int
    components: frozenset[str]
    responses: frozenset[str]
    topology_modes: frozenset[str]
    ad_modes: frozenset[str]
    world_motions: frozenset[str]
    world_version_domains: tuple[str, ...]
    response_components: tuple[tuple[str, frozenset[str]], ...]
    response_ad_modes: tuple[tuple[str, frozenset[str]], ...]
    component_ad_modes: tuple[tuple[str, frozenset[str]], ...]
    fixed_topology_components: frozenset[str]
    fixed_topology_responses: frozenset[str]
    supports_fixed_topology: bool
    supports_los_jones: bool
    fixed_topology_row_validity_components: frozenset[str]
    polarimetric_frozen_ad_inputs: tuple[str, ...]
    supports_slot_batching: bool
    max_slot_count: int | None
    supports_wideband_offsets: bool
    wideband_responses: frozenset[str]
    wideband_components: frozenset[str]
    wideband_dispersive_materials: bool
    wideband_rough_materials: bool
    max_frequency_offset_count: int | None
    native_frequency_resolution_law: str
    component_material_leaves: tuple[tuple[str, tuple[str, ...]], ...]
    differentiable_geometry_outputs: tuple[tuple[str, frozenset[str]], ...]
    direction_differentiable_components: frozenset[str]
    primal_only_ad_inputs: tuple[str, ...]
    supports_higher_order_ad: bool
    ad_accounting: bool

    def components_for(self, response: str) -> frozenset[str]:
        return dict(self.response_components)[response]

    def ad_modes_for(self, response: str) -> frozenset[str]:
        return dict(self.response_ad_modes)[response]

    def ad_modes_for_component(self, component: str) -> frozenset[str]:
        return dict(self.component_ad_modes)[component]

    def material_leaves_for(self, component: str) -> tuple[str, ...]:
        return dict(self.component_material_leaves)[component]

    def differentiable_geometry_for(self, route: str) -> frozenset[str]:
        return dict(self.differentiable_geometry_outputs)[route]


_CAPABILITIES = PropagationCapabilities(
    contract_version=CONTRACT_VERSION,
    components=COMPONENTS,
    responses=_SUPPORTED_RESPONSES,
    topology_modes=TOPOLOGY_MODES,
    ad_modes=AD_MODES,
    world_motions=WORLD_MOTIONS,
    world_version_domains=WORLD_VERSION_DOMAINS,
    response_components=_RESPONSE_COMPONENTS,
    # the scalar coefficient and the complex3 field are differentiated (native
    # fixed-topology VJP / JVP of every component); the Jones operator is not
    response_ad_modes=tuple((response, _SUPPORTED_AD_MODES if response == "polarimetric_transport" else AD_MODES)
                            for response in sorted(_SUPPORTED_RESPONSES)),
    component_ad_modes=tuple((component, AD_MODES) for component in sorted(COMPONENTS)),
    fixed_topology_components=frozenset(name for name, _ in _FIXED_TOPOLOGY_COMPONENT_IDS),
    fixed_topology_responses=RESPONSES,
    supports_fixed_topology=True,
    supports_los_jones=True,
    fixed_topology_row_validity_components=frozenset({"los", "reflection"}),
    polarimetric_frozen_ad_inputs=("tx_power", "mu_r", "source_basis", "sink_basis", "endpoint_polarizations"),
    supports_slot_batching=True,
    max_slot_count=None,
    supports_wideband_offsets=True,
    wideband_responses=frozenset({"scalar_transport", "complex3_transport"}),
    wideband_components=frozenset(name for name, _ in _FIXED_TOPOLOGY_COMPONENT_IDS),
    # every frequency column's material table is evaluated at that column's
    # own frequency (dispersion laws included), so an offset column of a
    # dispersive scene is exact
    wideband_dispersive_materials=True,
    wideband_rough_materials=False,
    max_frequency_offset_count=None,
    native_frequency_resolution_law=NATIVE_FREQUENCY_RESOLUTION_LAW,
    component_material_leaves=_COMPONENT_MATERIAL_LEAVES,
    differentiable_geometry_outputs=(("discovery", frozenset()),
                                     ("fixed_topology", frozenset({"path_length_m", "delay_s"}))),
    direction_differentiable_components=frozenset(),
    primal_only_ad_inputs=_PRIMAL_ONLY_AD_INPUTS,
    supports_higher_order_ad=False,
    ad_accounting=True,
)

_CONVENTION = PropagationConvention()


def capabilities() -> PropagationCapabilities:
    """The frozen capability record of this contract version (reference ``consumer.py:1181-1190``)."""

    return _CAPABILITIES


@dataclass(frozen=True, slots=True)
class PropagationDiagnostics:
    """Launch and host-observation counts of one call (reference ``consumer.py:1192-1217``).

    ``candidate_count`` is the number of path records discovery produced
    before the path limit; ``visibility_rejection_count`` is not counted by
    this engine (its kernels drop occluded candidates without a counter) and
    stays 0.  ``compact_count_*`` are the device-to-host reads of the record
    and selection counts and their stream synchronisations; ``validation_*``
    the read of the solve's status word."""

    discovery_launch_count: int
    candidate_count: int
    visibility_rejection_count: int
    compact_count_d2h_copies: int
    compact_count_d2h_bytes: int
    compact_sync_count: int
    validation_d2h_copies: int
    validation_d2h_bytes: int
    validation_sync_count: int
    frequency_column_count: int = 1
    ad_companion_launches: int = 0
    ad_tape_bytes: int = 0


@dataclass(frozen=True, slots=True, eq=False)
class PropagationEvaluation:
    paths: PropagationPathBatch
    convention: PropagationConvention
    capabilities: PropagationCapabilities
    diagnostics: PropagationDiagnostics


# --- LoS Jones operator -------------------------------------------------------------


@dataclass(frozen=True, slots=True)
class LoSJonesRows:
    """Output of :func:`consumer_los_jones` (reference ``consumer.py:1798-1803``)."""

    matrix: torch.Tensor
    source_basis: torch.Tensor
    sink_basis: torch.Tensor
    native_launch_count: int


def consumer_los_jones(*, pair_index: torch.Tensor, source_positions: torch.Tensor, sink_positions: torch.Tensor,
                       source_reference_basis: torch.Tensor, sink_reference_basis: torch.Tensor,
                       frequency_hz: float, _check_pairs: bool = True) -> LoSJonesRows:
    """Primal LoS transport between row-specific transverse bases (reference
    ``consumer.py:2037-2093``), one native ``wcb_los_jones`` launch.  Row ``k``
    takes ``pair_index[k] = sink * source_count + source``.  A pair index out of
    range raises ``IndexError`` after the launch (the kernel flags it; the
    check reads one status word)."""

    tensors = (pair_index, source_positions, sink_positions, source_reference_basis, sink_reference_basis)
    if any(not isinstance(value, torch.Tensor) for value in tensors):
        raise TypeError("LoS Jones inputs must be torch tensors")
    if any(value.requires_grad for value in tensors):
        raise RuntimeError("LoS Jones transport does not support AD")
    pair = _require_tensor("pair_index", pair_index, dtype=torch.int64, ndim=1)
    device = pair.device
    if device.type != "cuda":
        raise ValueError("LoS Jones inputs must be CUDA tensors")
    src = _require_tensor("source_positions", source_positions, dtype=torch.float32, ndim=2, device=device)
    snk = _require_tensor("sink_positions", sink_positions, dtype=torch.float32, ndim=2, device=device)
    if src.shape[1:] != (3,) or snk.shape[1:] != (3,):
        raise ValueError("source_positions and sink_positions must have shape (N, 3)")
    S, R = int(src.shape[0]), int(snk.shape[0])
    _require_tensor("source_reference_basis", source_reference_basis, dtype=torch.float32, shape=(S, 2, 3),
                    device=device)
    _require_tensor("sink_reference_basis", sink_reference_basis, dtype=torch.float32, shape=(R, 2, 3),
                    device=device)
    frequency = float(frequency_hz)
    if not (frequency > 0.0 and math.isfinite(frequency)):
        raise ValueError("frequency_hz must be a positive finite float")
    N = int(pair.shape[0])
    matrix = torch.empty((N, 2, 2), dtype=torch.complex64, device=device)
    source_basis = torch.empty((N, 2, 3), dtype=torch.float32, device=device)
    sink_basis = torch.empty((N, 2, 3), dtype=torch.float32, device=device)
    if N == 0:
        return LoSJonesRows(matrix=matrix, source_basis=source_basis, sink_basis=sink_basis, native_launch_count=0)
    if S == 0 or R == 0:
        raise IndexError("pair_index addresses an empty endpoint batch")
    lib = _native.load()
    status = torch.zeros(1, dtype=torch.int32, device=device)
    keep = [x.contiguous() for x in (pair, src, snk, source_reference_basis, sink_reference_basis)]
    with torch.cuda.device(device):
        _native.check(lib.wcb_los_jones(_native.ptr(keep[0]), N, _native.ptr(keep[1]), S, _native.ptr(keep[2]), R,
                                        _native.ptr(keep[3]), _native.ptr(keep[4]), frequency, _native.ptr(matrix),
                                        _native.ptr(source_basis), _native.ptr(sink_basis), _native.ptr(status),
                                        _native.stream_handle(device)), "wcb_los_jones")
    if _check_pairs and int(status.item()) != 0:
        raise IndexError(f"pair_index outside [0, {S * R})")
    return LoSJonesRows(matrix=matrix, source_basis=source_basis, sink_basis=sink_basis, native_launch_count=1)


def _require_polarimetric_inputs(request: PropagationRequest) -> None:
    """The polarimetric response needs both reference bases and takes them,
    the powers and the polarizations as primal-only (reference
    ``consumer.py:3186-3244``)."""

    if request.sources.polarization_basis is None or request.sinks.polarization_basis is None:
        raise ValueError("polarimetric_transport requires source and sink polarization_basis tensors")
    for name, value in (("sources.polarization_basis", request.sources.polarization_basis),
                        ("sinks.polarization_basis", request.sinks.polarization_basis),
                        ("sources.powers_w", request.sources.powers_w),
                        ("sources.polarizations", request.sources.polarizations),
                        ("sinks.polarizations", request.sinks.polarizations),
                        ("sources.positions_m", request.sources.positions_m),
                        ("sinks.positions_m", request.sinks.positions_m)):
        if value is not None and value.requires_grad:
            raise NotImplementedError(f"polarimetric_transport {name} is primal-only")


# --- evaluate ---------------------------------------------------------------------


def _preflight(compiled: object, request: object) -> float:
    """Refuse what this engine does not produce before any native work
    (reference ``consumer.py:3149-3183``)."""

    if not isinstance(compiled, CompiledScene):
        raise TypeError("evaluate requires a CompiledScene")
    if not isinstance(request, PropagationRequest):
        raise TypeError("request must be a PropagationRequest")
    if request.response not in _CAPABILITIES.responses:
        raise NotImplementedError(f"response {request.response!r} is not produced by this engine; supported "
                                  f"responses are {sorted(_CAPABILITIES.responses)}")
    response_components = _CAPABILITIES.components_for(request.response)
    if not request.components.issubset(response_components):
        raise NotImplementedError(f"{request.response} does not support components "
                                  f"{sorted(request.components - response_components)}")
    if request.ad_mode not in _CAPABILITIES.ad_modes_for(request.response):
        raise NotImplementedError(f"{request.response} does not support AD mode {request.ad_mode!r}")
    if request.response == "polarimetric_transport":
        _require_polarimetric_inputs(request)
    frequency = request.reference_frequency_hz
    if request.ad_mode == "none" and isinstance(frequency, torch.Tensor) and frequency.requires_grad:
        raise NotImplementedError("a differentiable reference frequency needs ad_mode 'vjp' or 'jvp'")
    _require_ad_request(compiled, request, request.response, request.ad_mode)
    if request.max_depth < 1 and request.components & {"reflection", "diffraction", "transmission"}:
        raise ValueError("reflection, diffraction and transmission rows require max_depth >= 1")
    if compiled.face_material.device != request.sources.device:
        raise ValueError("the compiled scene and the endpoint batches must share one CUDA device")
    return _frequency_value(frequency)


_C0_M_PER_S = 299_792_458.0

# Sources the canonical record key orders directly (its 11-bit source field).
_CANONICAL_SOURCE_LIMIT = 2048


def _interaction_types(component_id: torch.Tensor, depth: torch.Tensor, width: int) -> torch.Tensor:
    """Per-slot interaction flags of each row (reference ``propagation/topology.py:89-107``):
    reflection 1 on every active slot, diffraction 2 on slot 0, transmission 4 on
    every active slot, 0 elsewhere."""

    count = int(component_id.numel())
    result = torch.zeros((count, width), device=component_id.device, dtype=torch.int32)
    if count == 0 or width == 0:
        return result
    slots = torch.arange(width, device=component_id.device).view(1, -1)
    active = slots < depth.to(torch.int64).view(-1, 1)
    cid = component_id.view(-1, 1)
    result = torch.where(active & (cid == 1), torch.full_like(result, 1), result)
    result = torch.where(active & (cid == 5), torch.full_like(result, 4), result)
    first = (component_id == 2) & (depth > 0)
    result[:, 0] = torch.where(first, torch.full_like(result[:, 0], 2), result[:, 0])
    return result


def evaluate(compiled_scene: CompiledScene, request: PropagationRequest) -> PropagationEvaluation:
    """Discover and evaluate one compact propagation batch (reference
    ``consumer.py:3478-3520``): all pairs of ``request.sources`` x
    ``request.sinks``, at most ``max_paths`` rows in all."""

    frequency = _preflight(compiled_scene, request)
    compiled = compiled_scene
    sources, sinks = request.sources, request.sinks
    device = sources.device
    S, R = sources.count, sinks.count
    ep = engine.Endpoints(
        tx_pos=sources.positions_m, tx_power=sources.powers_w, tx_pol=sources.polarizations,
        rx={"kind": "point", "grid": None, "count": R, "shape": None, "pol": sinks.polarizations,
            "pol_stride": 3 if R > 0 else 0, "positions": sinks.positions_m},
    )
    width = int(request.max_depth)
    bits = engine.component_bits(request.components)
    launches0 = _native.launch_count()
    ad_tape = 0
    with torch.cuda.device(device):
        mats = compiled.material_tables([frequency], device)
        if S and R:
            res = engine.run_solve(compiled, ep, mats, [frequency], components=bits, max_depth=width, coherent=True,
                                   want_rows=True)
            rows = res["rows"]
        else:
            rows = torch.zeros((0, _native.ROW_WORDS), dtype=torch.int32, device=device)
        candidates = int(rows.shape[0])
        selected = engine.select_rows(rows, width, request.max_paths, "global")
        ev = engine.evaluate_rows(compiled, ep, mats, [frequency], 0, rows, selected, width, components=bits,
                                  max_depth=width, coherent=True)
        dec = engine.decode_rows(rows, selected)
        table = _path_table(dec, ev, width, compiled, include_fields=True)
        # sink-major, source-minor pair order.  The canonical selection key
        # leads with (sink, source) and holds the source in 11 bits, so up to
        # 2048 sources the selected rows (a global limit keeps a prefix)
        # already come in this order; beyond that a stable sort restores it
        # and keeps the canonical order of the rows inside each pair.
        pair = table.rx_id.to(torch.int64) * S + table.tx_id.to(torch.int64)
        order = None if S <= _CANONICAL_SOURCE_LIMIT else torch.argsort(pair, stable=True)
        pair_index = (pair if order is None else pair[order]).contiguous()
        # per-pair counts by a scatter (no host read of the largest pair)
        counts = torch.zeros(S * R, dtype=torch.int64, device=device)
        counts.index_add_(0, pair_index, torch.ones_like(pair_index))
        pair_offsets = torch.zeros(S * R + 1, dtype=torch.int64, device=device)
        pair_offsets[1:] = torch.cumsum(counts, 0)

        def take(x: torch.Tensor, dtype: torch.dtype) -> torch.Tensor:
            return (x if order is None else x.index_select(0, order)).to(dtype).contiguous()

        tx = take(table.tx_id, torch.int32)
        rx = take(table.rx_id, torch.int32)
        cid = take(table.component_id, torch.int32)
        depth = take(table.depth, torch.int32)
        seq = take(table.primitive_sequence, torch.int32)
        topology = PropagationTopology(
            source_index=tx, sink_index=rx,
            source_id=sources.stable_ids.index_select(0, tx.to(torch.int64)).contiguous(),
            sink_id=sinks.stable_ids.index_select(0, rx.to(torch.int64)).contiguous(),
            depth=depth, component_id=cid,
            primitive_id=take(table.primitive_id, torch.int32), edge_id=take(table.edge_id, torch.int32),
            material_id=take(table.material_id, torch.int32), primitive_sequence=seq,
            material_sequence=take(table.material_sequence, torch.int32),
            interaction_type=_interaction_types(cid, depth, width),
            provenance=WorldProvenance.of(compiled),
        )
        direction = take(table.field_direction, torch.float32)
        geometry = PropagationGeometry(
            path_length_m=take(table.path_length_m, torch.float32), delay_s=take(table.delay_s, torch.float32),
            field_direction=direction,
            interaction_positions_m=take(table.interaction_positions, torch.float32),
            interaction_normals=take(table.interaction_normals, torch.float32),
        )
        if request.response == "scalar_transport":
            coefficient = take(ev["path_field"], torch.complex64)
            if request.ad_mode != "none":
                pub = selected if order is None else selected.index_select(0, order)
                K = int(pub.shape[0])
                coefficient, ad_tape = _differentiable_coefficient(
                    compiled, request, coefficient, rows, pub.contiguous(),
                    torch.arange(K, device=device, dtype=torch.int64), ep, mats, frequency, bits, width)
            transport: PropagationTransport = ScalarTransport(coefficient=coefficient)
        elif request.response == "polarimetric_transport":
            # LoS rows only (preflighted): one fused launch over the compact pairs
            jones = consumer_los_jones(pair_index=pair_index, source_positions=sources.positions_m,
                                       sink_positions=sinks.positions_m,
                                       source_reference_basis=sources.polarization_basis,
                                       sink_reference_basis=sinks.polarization_basis, frequency_hz=frequency,
                                       _check_pairs=False)
            transport = JonesTransport(matrix=jones.matrix, source_basis=jones.source_basis,
                                       sink_basis=jones.sink_basis)
        else:
            # the row kernel's complex3 vector is at unit excitation; the
            # published field carries the source amplitude sqrt(powers_w)
            # (a negative power counts as zero, as in the row kernel)
            amplitude = torch.sqrt(torch.clamp(sources.powers_w.index_select(0, tx.to(torch.int64)), min=0.0))
            field = (take(ev["field_xyz"], torch.complex64) * amplitude.view(-1, 1)).contiguous()
            if request.ad_mode != "none":
                pub = selected if order is None else selected.index_select(0, order)
                K = int(pub.shape[0])
                field, ad_tape = _differentiable_field3(
                    compiled, request, field, rows, pub.contiguous(),
                    torch.arange(K, device=device, dtype=torch.int64), ep, mats, frequency, bits, width)
            transport = Complex3Transport(field=field, direction=direction)
    paths = PropagationPathBatch(pair_count=S * R, path_count=int(pair_index.numel()), pair_index=pair_index,
                                 pair_offsets=pair_offsets, topology=topology, geometry=geometry, transport=transport)
    # host observations: the solve's record count (8 bytes) and status word
    # (4 bytes); the selection's kept count (4 bytes, one read and two stream
    # syncs) when there were records to select from
    solved = bool(S and R)
    selecting = candidates > 0
    diagnostics = PropagationDiagnostics(
        discovery_launch_count=_native.launch_count() - launches0,
        candidate_count=candidates,
        visibility_rejection_count=0,
        compact_count_d2h_copies=int(solved) + int(selecting),
        compact_count_d2h_bytes=8 * int(solved) + 4 * int(selecting),
        compact_sync_count=int(solved) + 2 * int(selecting),
        validation_d2h_copies=int(solved),
        validation_d2h_bytes=4 * int(solved),
        validation_sync_count=int(solved),
        ad_tape_bytes=ad_tape,
    )
    return PropagationEvaluation(paths=paths, convention=_CONVENTION, capabilities=_CAPABILITIES,
                                 diagnostics=diagnostics)


# --- First-order AD of the scalar transport (both routes) ---------------------------


def _carries_ad(value: object) -> bool:
    if not isinstance(value, torch.Tensor):
        return False
    return value.requires_grad or torch.autograd.forward_ad.unpack_dual(value).tangent is not None


def _has_forward_tangent(value: object) -> bool:
    return isinstance(value, torch.Tensor) and torch.autograd.forward_ad.unpack_dual(value).tangent is not None


def _material_leaves(compiled: CompiledScene) -> list[tuple[str, object]]:
    """Every material value a caller can seed, named as in the capability
    record (a layered material's values also under ``materials.layer_*``)."""

    out: list[tuple[str, object]] = []
    for mat in compiled.materials:
        layers = mat.stack()
        for layer in layers:
            for name in ("eps_r", "sigma_e", "mu_r", "thickness_m"):
                value = getattr(layer, name, None)
                out.append(("materials." + name, value))
                if len(layers) > 1:
                    out.append(("materials.layer_" + name, value))
        out.append(("materials.gain", getattr(mat, "gain", None)))
    return out


def _require_ad_request(compiled: CompiledScene, request: Any, response: str, ad_mode: str) -> None:
    """Refusals of a differentiable request before any native work (reference
    ``consumer.py:268-371``): only the scalar coefficient is differentiated
    here; primal-only inputs must not carry AD; a reverse request must not
    carry a forward tangent (second order)."""

    if ad_mode == "none":
        return
    if response == "polarimetric_transport":
        raise NotImplementedError(f"ad_mode={ad_mode!r} is provided for scalar_transport and complex3_transport; "
                                  f"capabilities().ad_modes_for({response!r}) is {{'none'}}")
    values: list[tuple[str, object]] = [
        ("sources.powers_w", request.sources.powers_w), ("sources.polarizations", request.sources.polarizations),
        ("sinks.polarizations", request.sinks.polarizations),
        ("sources.polarization_basis", request.sources.polarization_basis),
        ("sinks.polarization_basis", request.sinks.polarization_basis),
    ]
    materials = _material_leaves(compiled)
    values += [(name, value) for name, value in materials if name not in _DIFFERENTIABLE_MATERIAL_LEAVES]
    for name, value in values:
        if _carries_ad(value):
            raise NotImplementedError(f"{name} is primal-only here: the native derivative kernels do not "
                                      "differentiate it (capabilities().primal_only_ad_inputs)")
    if ad_mode == "vjp":
        leaves = [("sources.positions_m", request.sources.positions_m), ("sinks.positions_m", request.sinks.positions_m),
                  ("reference_frequency_hz", request.reference_frequency_hz)] + materials
        leaves += [(f"structures[{i}].vertices", st.vertices) for i, st in enumerate(compiled.scene.structures)]
        for name, value in leaves:
            if _has_forward_tangent(value):
                raise NotImplementedError(f"ad_mode='vjp' with a forward dual on {name} is a second-order request; "
                                          "capabilities().supports_higher_order_ad is False")


def _differentiable_coefficient(compiled: CompiledScene, request: Any, coefficient: torch.Tensor,
                                rows: torch.Tensor, selected: torch.Tensor, live: torch.Tensor,
                                ep: engine.Endpoints, mats: Any, frequency: float, components: int,
                                max_depth: int) -> tuple[torch.Tensor, int]:
    """Attach the native fixed-topology derivatives to ``coefficient``.
    ``live`` (int64) are the published rows that carry derivatives and
    ``selected`` (int64) their native records in ``rows`` ((N,12) int32), one
    for one.  Returns the coefficient and the bytes kept for the backward
    pass."""

    device = coefficient.device
    freq = request.reference_frequency_hz
    freqs_t = freq.reshape(1).to(device=device, dtype=torch.float64) if isinstance(freq, torch.Tensor) else \
        torch.tensor([frequency], dtype=torch.float64, device=device)
    inputs = _ad._differentiable_inputs(compiled.scene, compiled, freqs_t, device)
    state = _ad._State(compiled=compiled, ep=ep, mats=mats, frequencies=[frequency], components=components,
                       max_depth=max_depth, coherent=True, rows=rows, selected=selected, flat={}, saved64=[None],
                       outputs32=[], layer_counts=inputs["layer_counts"], vertex_mask=inputs["vertex_mask"])
    out = _ad.RowFieldFunction.apply(state, coefficient, live, request.sources.positions_m,
                                     request.sinks.positions_m, inputs["vertices"], inputs["eps_r"],
                                     inputs["sigma_e"], inputs["layer_eps_r"], inputs["layer_sigma_e"],
                                     inputs["frequency"])
    tape = rows.numel() * 4 + (selected.numel() + live.numel()) * 8
    return out, tape


def _differentiable_field3(compiled: CompiledScene, request: Any, field: torch.Tensor, rows: torch.Tensor,
                           selected: torch.Tensor, live: torch.Tensor, ep: engine.Endpoints, mats: Any,
                           frequency: float, components: int, max_depth: int) -> tuple[torch.Tensor, int]:
    """Attach the native fixed-topology derivatives to the complex3 field
    ``field`` (K,3): component k is the row's field projected on the world
    axis e_k, the scalar field with e_k as the sink polarization.  The field
    is transverse to its arrival direction, so that projection is E_k and its
    derivative is dE_k exactly (the direction's own derivative cancels)."""

    columns, tape = [], 0
    for k in range(3):
        axis = torch.zeros((1, 3), dtype=torch.float32, device=field.device)
        axis[0, k] = 1.0
        ep_k = engine.Endpoints(tx_pos=ep.tx_pos, tx_power=ep.tx_power, tx_pol=ep.tx_pol,
                                rx={**ep.rx, "pol": axis, "pol_stride": 0})
        col, t = _differentiable_coefficient(compiled, request, field[:, k].contiguous(), rows, selected, live,
                                             ep_k, mats, frequency, components, max_depth)
        columns.append(col)
        tape += t
    return torch.stack(columns, dim=1), tape


def _differentiable_lengths(compiled: CompiledScene, topology: PropagationTopology, sources: EndpointBatch,
                            sinks: EndpointBatch, length: torch.Tensor, valid: torch.Tensor | None,
                            frequency: float) -> torch.Tensor:
    """The replayed path lengths with the derivatives of their FP64 unfolded
    length: |sink - image| with the source mirrored across the planes of the
    recorded faces (each from its own vertices, the plane its coplanar group
    shares while the group holds), differentiable in the source and sink
    positions and the vertices, as the native derivative kernels take the
    winner faces' planes.  The values stay the kernel's; rows that stopped
    existing stay constant zeros."""

    device = length.device
    cid = topology.component_id.to(torch.int64)
    depth = topology.depth.to(torch.int64)
    img = sources.positions_m.index_select(0, topology.source_index.to(torch.int64)).to(torch.float64)
    snk = sinks.positions_m.index_select(0, topology.sink_index.to(torch.int64)).to(torch.float64)
    width = int(topology.primitive_sequence.shape[1])
    if width and bool((cid == 1).any()):
        freqs_t = torch.tensor([float(frequency)], dtype=torch.float64, device=device)
        V = _ad._differentiable_inputs(compiled.scene, compiled, freqs_t, device)["vertices"]
        faces = compiled.native.faces.to(torch.int64)
        seq = topology.primitive_sequence.to(torch.int64)
        for k in range(width):
            active = (cid == 1) & (depth > k)
            f = torch.where(active, seq[:, k], torch.zeros_like(seq[:, k]))
            a, b, c = (V.index_select(0, faces[f, j]) for j in range(3))
            n = torch.linalg.cross(b - a, c - a)
            n = n / torch.clamp(torch.linalg.vector_norm(n, dim=-1, keepdim=True), min=1e-6)
            off = (n * a).sum(-1, keepdim=True)
            mirrored = img - 2.0 * n * ((n * img).sum(-1, keepdim=True) - off)
            img = torch.where(active.unsqueeze(-1), mirrored, img)
    unfolded = torch.linalg.vector_norm(snk - img, dim=-1)
    out = length + (unfolded - unfolded.detach()).to(length.dtype)
    if valid is not None:
        out = torch.where(valid, out, torch.zeros_like(out))
    return out


def _frozen_records(topology: PropagationTopology) -> torch.Tensor:
    """Native row records (K,12) int32 of frozen rows: source, sink,
    component | depth << 16, five faces (-1 padded), no edge."""

    K = topology.row_count
    device = topology.device
    rec = torch.zeros((K, _native.ROW_WORDS), dtype=torch.int32, device=device)
    if K == 0:
        return rec
    width = int(topology.primitive_sequence.shape[1])
    rec[:, 0] = topology.source_index
    rec[:, 1] = topology.sink_index
    rec[:, 2] = topology.component_id + topology.depth * 65536
    seq = torch.full((K, MAX_DEPTH), -1, dtype=torch.int32, device=device)
    if width:
        seq[:, :width] = topology.primitive_sequence
    rec[:, 3:8] = seq
    rec[:, 8] = -1
    return rec


# --- Fixed-topology replay ----------------------------------------------------------


@dataclass(frozen=True, slots=True, eq=False)
class FixedTopologyBucket:
    """One host-known ``(component, depth)`` partition of a frozen topology
    (reference ``consumer.py:1228-1249``): ``rows`` are ascending int64 indices
    into the frozen rows."""

    component: str
    depth: int
    rows: torch.Tensor

    def __post_init__(self) -> None:
        _require_vocabulary("component", self.component, COMPONENTS)
        if type(self.depth) is not int or not 0 <= self.depth <= MAX_DEPTH:
            raise ValueError(f"depth must be an int in [0, {MAX_DEPTH}]")
        _require_tensor("rows", self.rows, dtype=torch.int64, ndim=1)

    @property
    def row_count(self) -> int:
        return int(self.rows.shape[0])


@dataclass(frozen=True, slots=True, eq=False)
class PreparedFixedTopology:
    """A frozen topology partitioned once for repeated replay (reference
    ``consumer.py:1252-1287``).

    ``buckets`` are the ascending ``(component, depth)`` partitions; the
    ``prepare_*`` counters describe the one preparation (its host reads), not
    a later replay.  ``execution_order`` (int32, the buckets' rows one after
    the other) is the order the native replay runs the rows in, so a warp
    stays on one component and depth; it changes no published value."""

    topology: PropagationTopology
    buckets: tuple[FixedTopologyBucket, ...]
    prepare_d2h_copies: int
    prepare_d2h_bytes: int
    prepare_synchronizations: int
    execution_order: torch.Tensor | None = None

    @property
    def row_count(self) -> int:
        return self.topology.row_count

    @property
    def device(self) -> torch.device:
        return self.topology.device

    @property
    def provenance(self) -> WorldProvenance | None:
        return self.topology.provenance


def _require_slot_divisible(name: str, count: int, slot_count: int) -> None:
    if count % slot_count:
        raise ValueError(f"{name} carries {count} entries, which is not a multiple of slot_count={slot_count}; "
                         "every slot must hold the same number")


def _require_slot_count(slot_count: object) -> int:
    if type(slot_count) is not int or slot_count <= 0:
        raise ValueError("slot_count must be a positive int")
    return slot_count


@dataclass(frozen=True, slots=True)
class FixedTopologyRequest:
    """A replay request against an already-discovered topology (reference
    ``consumer.py:1307-1418``).

    ``topology`` is a raw :class:`PropagationTopology` for the zero-interaction
    LoS route or a :class:`PreparedFixedTopology` for any route with
    interactions.  ``world_motion="frozen_world"`` accepts only the world the
    rows were discovered against; ``"fixed_winner_replay"`` also accepts moved
    geometry (a refitted scene) with the winner set held fixed.
    ``slot_count > 1`` stacks block-diagonal slots slot-major (see
    :attr:`PropagationConvention.slot_pair_layout` and
    :func:`replicate_over_slots`).  ``frequency_offsets_hz`` asks for the same
    rows at ``reference_frequency_hz + df_j`` as well (wideband payload)."""

    sources: EndpointBatch
    sinks: EndpointBatch
    reference_frequency_hz: float | torch.Tensor
    topology: PropagationTopology | PreparedFixedTopology
    response: PropagationResponse
    ad_mode: PropagationAdMode
    world_motion: PropagationWorldMotion = "frozen_world"
    slot_count: int = 1
    frequency_offsets_hz: tuple[float, ...] | None = None

    def __post_init__(self) -> None:
        _require_endpoints(self.sources, self.sinks)
        self._require_slots()
        object.__setattr__(self, "frequency_offsets_hz", require_frequency_offsets(self.frequency_offsets_hz))
        if not isinstance(self.topology, PropagationTopology | PreparedFixedTopology):
            raise TypeError("topology must be a PropagationTopology or a PreparedFixedTopology")
        response = _require_vocabulary("response", self.response, RESPONSES)
        _require_vocabulary("ad_mode", self.ad_mode, AD_MODES)
        _require_vocabulary("world_motion", self.world_motion, WORLD_MOTIONS)
        if response not in _CAPABILITIES.fixed_topology_responses:
            raise NotImplementedError(f"fixed-topology reevaluation does not support {response!r}; supported "
                                      f"responses are {sorted(_CAPABILITIES.fixed_topology_responses)}")
        if self.frequency_offsets_hz is not None and response not in _CAPABILITIES.wideband_responses:
            raise NotImplementedError(f"frequency_offsets_hz is not supported for {response!r}; "
                                      f"capabilities().wideband_responses is "
                                      f"{sorted(_CAPABILITIES.wideband_responses)}")

    def _require_slots(self) -> None:
        slot_count = _require_slot_count(self.slot_count)
        if slot_count == 1:
            return
        if isinstance(self.topology, PropagationTopology):
            raise NotImplementedError("slot_count > 1 requires a PreparedFixedTopology; call prepare_fixed_topology "
                                      "and replicate_over_slots first")
        _require_slot_divisible("sources", self.sources.count, slot_count)
        _require_slot_divisible("sinks", self.sinks.count, slot_count)
        _require_slot_divisible("topology rows", self.frozen_topology.row_count, slot_count)

    @property
    def frozen_topology(self) -> PropagationTopology:
        if isinstance(self.topology, PreparedFixedTopology):
            return self.topology.topology
        return self.topology


@dataclass(frozen=True, slots=True, eq=False)
class FixedTopologyEvaluation:
    """A replayed batch of frozen rows (reference ``consumer.py:1421-1480``).

    ``row_valid`` (bool, frozen row order) is present on the prepared route and
    is the sole authority on whether a row's payload means anything: a LoS row
    whose segment is now blocked, or a reflection row whose bounce left its
    coplanar group or whose legs are now blocked, is published with
    ``row_valid=False`` and exact zeros.  A reflection row keeps its original
    face labels when its bounce slides onto a coplanar twin triangle.  Replay
    is subtractive: a path that comes into existence is not discovered here."""

    paths: PropagationPathBatch
    convention: PropagationConvention
    capabilities: PropagationCapabilities
    diagnostics: PropagationDiagnostics
    row_valid: torch.Tensor | None = None

    def __post_init__(self) -> None:
        if self.row_valid is None:
            return
        _require_tensor("row_valid", self.row_valid, dtype=torch.bool, shape=(self.paths.path_count,))


def _fixed_topology_component_name(component_id: int) -> str:
    for name, value in _FIXED_TOPOLOGY_COMPONENT_IDS:
        if value == component_id:
            return name
    raise NotImplementedError(f"fixed-topology reevaluation does not support component id {component_id}; "
                              f"supported components are {sorted(_CAPABILITIES.fixed_topology_components)}")


def _require_bucket_depth(component: str, depth: int) -> None:
    if component == "los" and depth != 0:
        raise ValueError("a los row must have depth 0")
    if component == "reflection" and depth < 1:
        raise ValueError("a reflection row must have depth >= 1")


def _malformed_rows(topology: PropagationTopology, width: int) -> torch.Tensor:
    """Rows whose depth or interaction padding contradicts the contract:
    depth outside ``[0, width]``, a negative id on an active slot, or an
    unused slot that does not hold -1."""

    depth = topology.depth.to(dtype=torch.int64)
    slots = torch.arange(width, device=topology.device, dtype=torch.int64).reshape(1, -1)
    active = slots < depth.reshape(-1, 1)
    sequence = topology.primitive_sequence.to(dtype=torch.int64)
    return (depth < 0) | (depth > width) | ((sequence < 0) & active).any(dim=1) | ((sequence != -1) & ~active).any(dim=1)


def prepare_fixed_topology(topology: PropagationTopology) -> PreparedFixedTopology:
    """Partition a frozen topology by component and interaction depth
    (reference ``consumer.py:1518-1570``).

    The one place the frozen rows are looked at on the host: it validates the
    depth / interaction padding of every row, refuses components outside
    ``capabilities().fixed_topology_components``, and returns the ascending
    ``(component, depth)`` buckets.  It synchronises: call it once per frozen
    topology and reuse the handle."""

    if not isinstance(topology, PropagationTopology):
        raise TypeError("topology must be a PropagationTopology")
    if topology.row_count == 0:
        return PreparedFixedTopology(topology=topology, buckets=(), prepare_d2h_copies=0, prepare_d2h_bytes=0,
                                     prepare_synchronizations=0,
                                     execution_order=torch.zeros(0, dtype=torch.int32, device=topology.device))
    width = int(topology.primitive_sequence.shape[1])
    if width > MAX_DEPTH:
        raise ValueError(f"primitive_sequence width {width} exceeds the maximum depth {MAX_DEPTH}")
    if bool(_malformed_rows(topology, width).any().item()):
        raise ValueError("frozen topology rows disagree with their interaction sequence padding; depth must be in "
                         "[0, sequence width] and unused slots must hold -1")
    key = topology.component_id.to(dtype=torch.int64) * (width + 1) + topology.depth.to(dtype=torch.int64)
    distinct = torch.unique(key).tolist()
    buckets = []
    for value in distinct:
        component_id, depth = divmod(int(value), width + 1)
        component = _fixed_topology_component_name(component_id)
        _require_bucket_depth(component, depth)
        buckets.append(FixedTopologyBucket(component=component, depth=depth,
                                           rows=torch.nonzero(key == value, as_tuple=False).reshape(-1)))
    order = torch.cat([bucket.rows for bucket in buckets]).to(torch.int32)
    return PreparedFixedTopology(topology=topology, buckets=tuple(buckets), prepare_d2h_copies=2 + len(buckets),
                                 prepare_d2h_bytes=1 + 8 * (len(distinct) + len(buckets)),
                                 prepare_synchronizations=2 + len(buckets), execution_order=order)


def replicate_over_slots(prepared: PreparedFixedTopology, slot_count: int, *, source_count: int,
                         sink_count: int) -> PreparedFixedTopology:
    """Tile a frozen topology over ``slot_count`` block-diagonal slots
    (reference ``consumer.py:1573-1650``).

    ``source_count`` / ``sink_count`` are the per-slot endpoint counts.  Row
    ``t*K + r`` is frozen row ``r`` shifted into slot ``t``; index arithmetic
    only, no host observation; ``slot_count == 1`` returns the handle."""

    if not isinstance(prepared, PreparedFixedTopology):
        raise TypeError("prepared must be a PreparedFixedTopology")
    slot_count = _require_slot_count(slot_count)
    for name, value in (("source_count", source_count), ("sink_count", sink_count)):
        if type(value) is not int or value <= 0:
            raise ValueError(f"{name} must be a positive int")
    if slot_count == 1:
        return prepared
    topology = prepared.topology
    rows = topology.row_count
    device = topology.device
    slot = torch.arange(slot_count, device=device, dtype=torch.int32)
    replicated = PropagationTopology(
        source_index=topology.source_index.repeat(slot_count) + slot.mul(source_count).repeat_interleave(rows),
        sink_index=topology.sink_index.repeat(slot_count) + slot.mul(sink_count).repeat_interleave(rows),
        source_id=topology.source_id.repeat(slot_count), sink_id=topology.sink_id.repeat(slot_count),
        depth=topology.depth.repeat(slot_count), component_id=topology.component_id.repeat(slot_count),
        primitive_id=topology.primitive_id.repeat(slot_count), edge_id=topology.edge_id.repeat(slot_count),
        material_id=topology.material_id.repeat(slot_count),
        primitive_sequence=topology.primitive_sequence.repeat(slot_count, 1),
        material_sequence=topology.material_sequence.repeat(slot_count, 1),
        interaction_type=topology.interaction_type.repeat(slot_count, 1),
        provenance=topology.provenance,
    )
    row_offset = torch.arange(slot_count, device=device, dtype=torch.int64).mul(rows).reshape(-1, 1)
    buckets = tuple(
        FixedTopologyBucket(component=bucket.component, depth=bucket.depth,
                            rows=(bucket.rows.reshape(1, -1) + row_offset).reshape(-1))
        for bucket in prepared.buckets
    )
    order = (torch.cat([bucket.rows for bucket in buckets]).to(torch.int32) if buckets
             else torch.zeros(0, dtype=torch.int32, device=device))
    return PreparedFixedTopology(topology=replicated, buckets=buckets,
                                 prepare_d2h_copies=prepared.prepare_d2h_copies,
                                 prepare_d2h_bytes=prepared.prepare_d2h_bytes,
                                 prepare_synchronizations=prepared.prepare_synchronizations, execution_order=order)


def _source_moved_domain(compiled: CompiledScene) -> str | None:
    """The version domain a scene mutated after its compile moved, read from
    the compile's record of the scene's structures (tensor identities and
    in-place versions, face tables, materials, metadata)."""

    from ..compiler import _geometry_token

    token, _refs = _geometry_token(compiled.scene)
    old = compiled.source_token
    if token == old:
        return None
    if len(token) != len(old) or token[-1] != old[-1]:
        return "topology_version"
    for o, n in zip(old[:-1], token[:-1]):
        if o[2] != n[2]:
            return "topology_version"
        if o[3] != n[3] or o[4] != n[4]:
            return "assignment_version"
    return "geometry_version"


def rediscovery_required(compiled_scene: CompiledScene, topology: PropagationTopology | PreparedFixedTopology, *,
                         revalidate_source: bool = False) -> str | None:
    """Name the version domain that moved under a frozen topology, or ``None``
    (reference ``consumer.py:3554-3594``).  The default check is four host
    integer comparisons; ``revalidate_source=True`` also compares the compile
    with the live scene, which catches a scene mutated in place after its
    compile (host work over the scene's structures)."""

    if not isinstance(compiled_scene, CompiledScene):
        raise TypeError("rediscovery_required requires a CompiledScene")
    if not isinstance(topology, PropagationTopology | PreparedFixedTopology):
        raise TypeError("topology must be a PropagationTopology or a PreparedFixedTopology")
    provenance = topology.provenance
    if provenance is not None:
        moved = provenance.moved_domain(WorldProvenance.of(compiled_scene))
        if moved is not None:
            return moved
    if not revalidate_source:
        return None
    return _source_moved_domain(compiled_scene)


def _require_current_world(compiled: CompiledScene, request: FixedTopologyRequest) -> None:
    """Refuse a frozen replay against a world that moved (reference ``consumer.py:3523-3551``)."""

    provenance = request.frozen_topology.provenance
    if provenance is None:
        return
    moved = provenance.moved_domain(WorldProvenance.of(compiled),
                                    allow_geometry=request.world_motion == "fixed_winner_replay")
    if moved is None:
        return
    remedy = ("declare world_motion='fixed_winner_replay' to hold the discrete winner set fixed while the geometry "
              "moves, or rediscover" if moved == "geometry_version"
              else "the frozen row labels no longer name the same world; rediscover")
    raise ValueError(f"frozen topology is stale: {moved} changed between discovery and this reevaluation; "
                     f"{remedy} with evaluate() and prepare_fixed_topology()")


def _require_resolvable_offsets(offsets: tuple[float, ...], reference_frequency_hz: float) -> None:
    """Refuse offsets the launch grid cannot tell apart (reference ``consumer.py:3630-3658``;
    here the grid is float64, see :func:`native_frequency_resolution_hz`)."""

    resolution = native_frequency_resolution_hz(reference_frequency_hz)
    for offset in offsets:
        if offset != 0.0 and abs(offset) < resolution:
            raise ValueError(f"frequency_offsets_hz entry {offset!r} Hz is below the native frequency resolution "
                             f"{resolution!r} Hz at {reference_frequency_hz!r} Hz")
    ordered = sorted(offsets)
    for lower, upper in zip(ordered, ordered[1:]):
        if upper - lower < resolution:
            raise ValueError(f"frequency_offsets_hz entries {lower!r} Hz and {upper!r} Hz are closer than the native "
                             f"frequency resolution {resolution!r} Hz at {reference_frequency_hz!r} Hz")
    for offset in offsets:
        if not reference_frequency_hz + offset > 0.0:
            raise ValueError(f"frequency_offsets_hz entry {offset!r} Hz gives a non-positive frequency")


def _preflight_reevaluate(compiled: object, request: object) -> float:
    """Everything refused before native work (reference ``consumer.py:3720-3764``)."""

    if not isinstance(compiled, CompiledScene):
        raise TypeError("reevaluate requires a CompiledScene")
    if not isinstance(request, FixedTopologyRequest):
        raise TypeError("request must be a FixedTopologyRequest")
    _require_current_world(compiled, request)
    if request.frozen_topology.device != request.sources.device:
        raise ValueError("fixed topology and endpoint batches must share a device")
    if compiled.face_material.device != request.sources.device:
        raise ValueError("the compiled scene and the endpoint batches must share one CUDA device")
    if request.ad_mode not in _CAPABILITIES.ad_modes_for(request.response):
        raise NotImplementedError(f"fixed-topology {request.response} does not support AD mode {request.ad_mode!r}")
    frequency = request.reference_frequency_hz
    if request.ad_mode == "none" and isinstance(frequency, torch.Tensor) and frequency.requires_grad:
        raise NotImplementedError("a differentiable reference frequency needs ad_mode 'vjp' or 'jvp'")
    _require_ad_request(compiled, request, request.response, request.ad_mode)
    if isinstance(request.topology, PropagationTopology) and request.topology.primitive_sequence.shape[1] != 0:
        raise NotImplementedError("fixed LoS reevaluation requires zero-width interaction sequences; call "
                                  "prepare_fixed_topology first to reevaluate a topology that carries interactions")
    if request.response == "polarimetric_transport":
        if request.sources.polarization_basis is None or request.sinks.polarization_basis is None:
            raise ValueError("polarimetric_transport requires source and sink polarization_basis tensors")
        if isinstance(request.topology, PropagationTopology):
            raise NotImplementedError("fixed-topology polarimetric_transport requires a PreparedFixedTopology; the "
                                      "raw-topology form is the zero-interaction scalar and complex3 fast path")
    value = _frequency_value(frequency)
    if request.frequency_offsets_hz is not None:
        _require_resolvable_offsets(request.frequency_offsets_hz, value)
        if request.ad_mode != "none":
            raise NotImplementedError("frequency_offsets_hz with ad_mode != 'none' is not provided: the wideband "
                                      "columns carry no derivative here")
    return value


def _endpoint_struct(batch: EndpointBatch, with_basis: bool) -> Any:
    e = _native.EndpointBatch()
    e.count = batch.count
    e.positions = _native.ptr(batch.positions_m)
    e.polarizations = _native.ptr(batch.polarizations)
    e.stable_ids = _native.ptr(batch.stable_ids)
    e.powers = _native.ptr(batch.powers_w)
    e.polarization_basis = _native.ptr(batch.polarization_basis) if with_basis else None
    return e


_REPLAY_CONTRACT_BITS = ((1, "a source or sink index outside its endpoint batch"),
                         (2, "in-bounds rows not in non-decreasing pair order"),
                         (16, "a stable id that differs from the endpoint batch's"),
                         (32, "a slot-batched row whose sink lies outside its source's slot"))


def reevaluate(compiled_scene: CompiledScene, request: FixedTopologyRequest) -> FixedTopologyEvaluation:
    """Re-evaluate frozen rows at the request's endpoints without discovery or
    compaction (reference ``consumer.py:3846-4110``).

    One native launch replays every row and every frequency column (the
    reference frequency, then ``reference_frequency_hz + df_j``): the
    endpoint gather, the contract validation (index bounds, pair order,
    stable ids, slot blocks), the visibility re-test of the prepared route
    and the image-method geometry are done once per row; a second launch
    segments the rows by pair.  One 8-byte status read per call."""

    frequency = _preflight_reevaluate(compiled_scene, request)
    compiled = compiled_scene
    prepared = request.topology if isinstance(request.topology, PreparedFixedTopology) else None
    topology = request.frozen_topology
    sources, sinks = request.sources, request.sinks
    device = sources.device
    K = topology.row_count
    width = int(topology.primitive_sequence.shape[1])
    S, R = sources.count, sinks.count
    slot_count = request.slot_count
    if K > 0 and (S == 0 or R == 0):
        raise ValueError("non-empty frozen topology requires endpoint rows")
    pair_count = slot_count * (S // slot_count) * (R // slot_count)
    offsets = request.frequency_offsets_hz
    columns = [frequency] + ([frequency + df for df in offsets] if offsets is not None else [])
    extra = len(columns) - 1
    response = request.response
    polarimetric = response == "polarimetric_transport"

    def empty(*shape: int, dtype: torch.dtype = torch.float32) -> torch.Tensor:
        return torch.empty(shape, dtype=dtype, device=device)

    coefficient = empty(K, dtype=torch.complex64) if response == "scalar_transport" else None
    coefficient_offsets = empty(K, extra, dtype=torch.complex64) if coefficient is not None and extra else None
    field = empty(K, 3, dtype=torch.complex64) if response == "complex3_transport" else None
    field_offsets = empty(K, extra, 3, dtype=torch.complex64) if field is not None and extra else None
    length = empty(K)
    delay = empty(K)
    direction = empty(K, 3)
    positions = empty(K, width, 3)
    normals = empty(K, width, 3)
    row_valid = empty(K, dtype=torch.bool) if prepared is not None else None
    jones = empty(K, 2, 2, dtype=torch.complex64) if polarimetric else None
    source_basis = empty(K, 2, 3) if polarimetric else None
    sink_basis = empty(K, 2, 3) if polarimetric else None
    pair_index = empty(K, dtype=torch.int64)
    pair_offsets = empty(pair_count + 1, dtype=torch.int64)
    status = torch.zeros(2, dtype=torch.int32, device=device)
    launches0 = _native.launch_count()
    with torch.cuda.device(device):
        mats, freqs = compiled.resident_tables(columns, device)
        rows = _native.FrozenRows()
        rows.num_rows = K
        rows.width = width
        keep = {name: getattr(topology, name).contiguous()
                for name in ("component_id", "depth", "primitive_sequence", "source_index", "sink_index",
                             "source_id", "sink_id")}
        for name, value in keep.items():
            setattr(rows, name, _native.ptr(value))
        rows.order = _native.ptr(prepared.execution_order) if prepared is not None else None
        out = _native.ReplayOutputs()
        for name, value in (("coefficient", coefficient), ("coefficient_offsets", coefficient_offsets),
                            ("field", field), ("field_offsets", field_offsets), ("path_length_m", length),
                            ("delay_s", delay), ("direction", direction), ("interaction_positions", positions),
                            ("interaction_normals", normals), ("row_valid", row_valid), ("jones", jones),
                            ("source_basis", source_basis), ("sink_basis", sink_basis), ("pair_index", pair_index),
                            ("pair_offsets", pair_offsets)):
            setattr(out, name, _native.ptr(value))
        src = _endpoint_struct(sources, polarimetric)
        snk = _endpoint_struct(sinks, polarimetric)
        m = mats.as_struct()
        lib = _native.load()
        _native.check(lib.wcb_rows_replay(compiled.native.handle, _native.ctypes.byref(rows),
                                          _native.ctypes.byref(src), _native.ctypes.byref(snk), slot_count,
                                          _native.ctypes.byref(m), _native.ptr(freqs), len(columns),
                                          int(prepared is not None), _native.ctypes.byref(out),
                                          _native.ptr(status), _native.stream_handle(device)), "wcb_rows_replay")
        contract, engine_bits = (int(v) for v in status.tolist()) if K > 0 else (0, 0)
    if contract:
        reasons = "; ".join(text for bit, text in _REPLAY_CONTRACT_BITS if contract & bit)
        raise ValueError(f"frozen topology validation failed against the current endpoint batches (error bitmask "
                         f"{contract}: {reasons})")
    if engine_bits & 6:
        raise ValueError("frozen topology carries a row this replay cannot evaluate (a component other than los / "
                         "reflection, a depth outside the row's sequence, or a face id outside the compiled scene)")
    if engine_bits & 1:
        raise _native.NativeError(_native.WCB_ERR_BVH_DEPTH, "wcb_rows_replay")
    ad_tape = 0
    if request.ad_mode != "none":
        live = torch.nonzero(row_valid).reshape(-1) if row_valid is not None else \
            torch.arange(K, device=device, dtype=torch.int64)
        ep = engine.Endpoints(
            tx_pos=sources.positions_m.detach(), tx_power=sources.powers_w.detach(),
            tx_pol=sources.polarizations.detach(),
            rx={"kind": "point", "grid": None, "count": R, "shape": None, "pol": sinks.polarizations.detach(),
                "pol_stride": 3 if R > 0 else 0, "positions": sinks.positions_m.detach()})
        mats1 = compiled.material_tables([frequency], device)
        bits = engine.component_bits(frozenset({"los", "reflection"}))
        if response == "scalar_transport":
            coefficient, ad_tape = _differentiable_coefficient(
                compiled, request, coefficient, _frozen_records(topology), live, live, ep, mats1, frequency, bits,
                max(width, 1))
        else:
            field, ad_tape = _differentiable_field3(
                compiled, request, field, _frozen_records(topology), live, live, ep, mats1, frequency, bits,
                max(width, 1))
        length = _differentiable_lengths(compiled, topology, sources, sinks, length, row_valid, frequency)
        delay = delay + ((length - length.detach()) / _C0_M_PER_S).to(delay.dtype)
    if polarimetric:
        transport: PropagationTransport = JonesTransport(matrix=jones, source_basis=source_basis,
                                                         sink_basis=sink_basis)
    elif response == "scalar_transport":
        transport = ScalarTransport(coefficient=coefficient, coefficient_offsets=coefficient_offsets,
                                    frequency_offsets_hz=offsets)
    else:
        transport = Complex3Transport(field=field, direction=direction, field_offsets=field_offsets,
                                      frequency_offsets_hz=offsets)
    paths = PropagationPathBatch(
        pair_count=pair_count, path_count=K, pair_index=pair_index, pair_offsets=pair_offsets, topology=topology,
        geometry=PropagationGeometry(path_length_m=length, delay_s=delay, field_direction=direction,
                                     interaction_positions_m=positions, interaction_normals=normals),
        transport=transport,
    )
    diagnostics = PropagationDiagnostics(
        discovery_launch_count=_native.launch_count() - launches0, candidate_count=0, visibility_rejection_count=0,
        compact_count_d2h_copies=0, compact_count_d2h_bytes=0, compact_sync_count=0,
        validation_d2h_copies=int(K > 0), validation_d2h_bytes=8 * int(K > 0), validation_sync_count=int(K > 0),
        frequency_column_count=1 if offsets is None else len(offsets), ad_tape_bytes=ad_tape,
    )
    return FixedTopologyEvaluation(paths=paths, convention=_CONVENTION, capabilities=_CAPABILITIES,
                                   diagnostics=diagnostics, row_valid=row_valid)


# --- Time-varying replay (reference consumer.py:4113-4318) ----------------------------


def _slot_view(values: torch.Tensor, slot_count: int) -> torch.Tensor:
    """A slot-major row axis as ``[slot_count, K, ...]`` (a view)."""

    return values.view(slot_count, -1, *values.shape[1:])


@dataclass(frozen=True, slots=True)
class TimeVaryingRequest:
    """One prepared topology replayed across slot-major endpoint batches, one
    slot per instant of ``times_s`` (float64, 1-D, non-empty).  The times label
    the slots; the endpoint positions carry the motion."""

    sources: EndpointBatch
    sinks: EndpointBatch
    reference_frequency_hz: float | torch.Tensor
    topology: PreparedFixedTopology
    times_s: torch.Tensor
    response: PropagationResponse
    ad_mode: PropagationAdMode
    world_motion: PropagationWorldMotion = "frozen_world"

    def __post_init__(self) -> None:
        if not isinstance(self.topology, PreparedFixedTopology):
            raise TypeError("topology must be a PreparedFixedTopology; call prepare_fixed_topology once per frozen "
                            "topology and reuse it")
        times = self.times_s
        if not isinstance(times, torch.Tensor):
            raise TypeError("times_s must be a torch.Tensor")
        if times.dtype != torch.float64:
            raise TypeError(f"times_s must use torch.float64, got {times.dtype}")
        if times.ndim != 1 or int(times.shape[0]) == 0:
            raise ValueError("times_s must be a non-empty 1-D tensor")

    @property
    def slot_count(self) -> int:
        return int(self.times_s.shape[0])


@dataclass(frozen=True, slots=True, eq=False)
class TimeVaryingTransport:
    """Slot-shaped views of the replayed transport; only the requested
    response's tensors are present."""

    response: PropagationResponse
    coefficient: torch.Tensor | None = None
    field: torch.Tensor | None = None
    direction: torch.Tensor | None = None
    matrix: torch.Tensor | None = None
    source_basis: torch.Tensor | None = None
    sink_basis: torch.Tensor | None = None

    @classmethod
    def from_transport(cls, transport: PropagationTransport, slot_count: int) -> TimeVaryingTransport:
        if isinstance(transport, ScalarTransport):
            return cls(response="scalar_transport", coefficient=_slot_view(transport.coefficient, slot_count))
        if isinstance(transport, Complex3Transport):
            return cls(response="complex3_transport", field=_slot_view(transport.field, slot_count),
                       direction=_slot_view(transport.direction, slot_count))
        return cls(response="polarimetric_transport", matrix=_slot_view(transport.matrix, slot_count),
                   source_basis=_slot_view(transport.source_basis, slot_count),
                   sink_basis=_slot_view(transport.sink_basis, slot_count))


@dataclass(frozen=True, slots=True, eq=False)
class TimeVaryingEvaluation:
    """One frozen topology at ``slot_count`` instants: every tensor is
    slot-major (``[t]`` is the whole frozen row set at ``times_s[t]``);
    ``pair_offsets`` and ``pair_count`` are per slot."""

    slot_count: int
    row_count: int
    times_s: torch.Tensor
    delay_s: torch.Tensor
    path_length_m: torch.Tensor
    transport: TimeVaryingTransport
    pair_count: int
    pair_offsets: torch.Tensor
    convention: PropagationConvention
    capabilities: PropagationCapabilities
    diagnostics: PropagationDiagnostics
    row_valid: torch.Tensor | None = None

    @classmethod
    def from_evaluation(cls, evaluation: FixedTopologyEvaluation, times_s: torch.Tensor,
                        slot_count: int) -> TimeVaryingEvaluation:
        paths = evaluation.paths
        pair_count = paths.pair_count // slot_count
        return cls(
            slot_count=slot_count, row_count=paths.path_count // slot_count, times_s=times_s,
            delay_s=_slot_view(paths.geometry.delay_s, slot_count),
            path_length_m=_slot_view(paths.geometry.path_length_m, slot_count),
            transport=TimeVaryingTransport.from_transport(paths.transport, slot_count), pair_count=pair_count,
            pair_offsets=paths.pair_offsets[: pair_count + 1], convention=evaluation.convention,
            capabilities=evaluation.capabilities, diagnostics=evaluation.diagnostics,
            row_valid=None if evaluation.row_valid is None else _slot_view(evaluation.row_valid, slot_count),
        )


def evaluate_time_varying(compiled_scene: CompiledScene, request: TimeVaryingRequest) -> TimeVaryingEvaluation:
    """Replay one frozen topology across a block of instants in one call
    (reference ``consumer.py:4259-4318``): the topology is replicated over
    ``len(times_s)`` slots and replayed once."""

    if not isinstance(request, TimeVaryingRequest):
        raise TypeError("request must be a TimeVaryingRequest")
    slot_count = request.slot_count
    _require_slot_divisible("sources", request.sources.count, slot_count)
    _require_slot_divisible("sinks", request.sinks.count, slot_count)
    replicated = replicate_over_slots(request.topology, slot_count,
                                      source_count=request.sources.count // slot_count,
                                      sink_count=request.sinks.count // slot_count)
    evaluation = reevaluate(compiled_scene, FixedTopologyRequest(
        sources=request.sources, sinks=request.sinks, reference_frequency_hz=request.reference_frequency_hz,
        topology=replicated, response=request.response, ad_mode=request.ad_mode, world_motion=request.world_motion,
        slot_count=slot_count))
    return TimeVaryingEvaluation.from_evaluation(evaluation, request.times_s, slot_count)


__all__ = [
    "AD_MODES",
    "COMPONENTS",
    "CONTRACT_VERSION",
    "MAX_DEPTH",
    "RESPONSES",
    "TOPOLOGY_MODES",
    "WORLD_MOTIONS",
    "WORLD_VERSION_DOMAINS",
    "Complex3Transport",
    "EndpointBatch",
    "FixedTopologyBucket",
    "FixedTopologyEvaluation",
    "FixedTopologyRequest",
    "JonesTransport",
    "LoSJonesRows",
    "PreparedFixedTopology",
    "PropagationAdMode",
    "PropagationCapabilities",
    "PropagationComponent",
    "PropagationConvention",
    "PropagationDiagnostics",
    "PropagationEvaluation",
    "PropagationGeometry",
    "PropagationPathBatch",
    "PropagationRequest",
    "PropagationResponse",
    "PropagationTopology",
    "PropagationTopologyMode",
    "PropagationWorldMotion",
    "ScalarTransport",
    "TimeVaryingEvaluation",
    "TimeVaryingRequest",
    "TimeVaryingTransport",
    "WorldProvenance",
    "capabilities",
    "consumer_los_jones",
    "evaluate",
    "evaluate_time_varying",
    "native_frequency_resolution_hz",
    "prepare_fixed_topology",
    "rediscovery_required",
    "reevaluate",
    "replicate_over_slots",
    "require_frequency_offsets",
    "require_wideband_payload",
]
