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
(``consumer_los_jones``, ``:2037-2093``); AD mode "none".  AD modes other than
"none", the fixed-topology replay (``prepare_fixed_topology`` /
``reevaluate``), wideband offsets and the time-varying route are not
advertised, and requests for them fail before any native work.
"""

from __future__ import annotations

import math
from dataclasses import dataclass
from typing import Any, Literal, TypeAlias, get_args

import torch

from .. import _native, engine
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

COMPONENTS: frozenset[str] = frozenset(get_args(PropagationComponent))
RESPONSES: frozenset[str] = frozenset(get_args(PropagationResponse))
TOPOLOGY_MODES: frozenset[str] = frozenset(get_args(PropagationTopologyMode))
AD_MODES: frozenset[str] = frozenset(get_args(PropagationAdMode))

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

_COMPONENT_MATERIAL_LEAVES: tuple[tuple[str, tuple[str, ...]], ...] = (
    ("diffraction", ("eps_r", "sigma_e", "thickness_m", "gain")),
    ("los", ()),
    ("reflection", ("eps_r", "sigma_e", "thickness_m", "gain")),
    ("transmission", ("layer_eps_r", "layer_sigma_e", "layer_thickness_m")),
)

_PRIMAL_ONLY_AD_INPUTS: tuple[str, ...] = (
    "materials.layer_mu_r",
    "materials.mu_r",
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


# --- Result records -------------------------------------------------------------


@dataclass(frozen=True, slots=True, eq=False)
class PropagationTopology:
    """Compact discrete rows in pair-major order (reference ``consumer.py:656-737``).

    ``provenance`` names the world the rows were discovered against; the
    scenes here carry no world version counters, so discovery leaves it
    ``None``."""

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
    ``consumer.py:796-833``).  This engine publishes no wideband payload."""

    coefficient: torch.Tensor
    coefficient_offsets: torch.Tensor | None = None
    frequency_offsets_hz: tuple[float, ...] | None = None

    def __post_init__(self) -> None:
        _require_tensor("coefficient", self.coefficient, dtype=torch.complex64, ndim=1)
        if self.coefficient_offsets is not None or self.frequency_offsets_hz is not None:
            raise NotImplementedError("wideband offset payloads are not produced by this engine")

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
    ``field`` on the sink polarization gives :attr:`ScalarTransport.coefficient`."""

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
        if self.field_offsets is not None or self.frequency_offsets_hz is not None:
            raise NotImplementedError("wideband offset payloads are not produced by this engine")

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
    ad_modes=_SUPPORTED_AD_MODES,
    world_motions=frozenset(),
    world_version_domains=WORLD_VERSION_DOMAINS,
    response_components=_RESPONSE_COMPONENTS,
    response_ad_modes=tuple((response, _SUPPORTED_AD_MODES) for response in sorted(_SUPPORTED_RESPONSES)),
    component_ad_modes=tuple((component, _SUPPORTED_AD_MODES) for component in sorted(COMPONENTS)),
    fixed_topology_components=frozenset(),
    fixed_topology_responses=frozenset(),
    supports_fixed_topology=False,
    supports_los_jones=True,
    fixed_topology_row_validity_components=frozenset(),
    polarimetric_frozen_ad_inputs=("tx_power", "mu_r", "source_basis", "sink_basis", "endpoint_polarizations"),
    supports_slot_batching=False,
    max_slot_count=None,
    supports_wideband_offsets=False,
    wideband_responses=frozenset(),
    wideband_components=frozenset(),
    wideband_dispersive_materials=False,
    wideband_rough_materials=False,
    max_frequency_offset_count=None,
    native_frequency_resolution_law=NATIVE_FREQUENCY_RESOLUTION_LAW,
    component_material_leaves=_COMPONENT_MATERIAL_LEAVES,
    differentiable_geometry_outputs=(("discovery", frozenset()),),
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
    if isinstance(frequency, torch.Tensor) and frequency.requires_grad:
        raise NotImplementedError("a differentiable reference frequency needs an AD mode this engine does not offer")
    if request.max_depth < 1 and request.components & {"reflection", "diffraction", "transmission"}:
        raise ValueError("reflection, diffraction and transmission rows require max_depth >= 1")
    if compiled.face_material.device != request.sources.device:
        raise ValueError("the compiled scene and the endpoint batches must share one CUDA device")
    return _frequency_value(frequency)


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
        )
        direction = take(table.field_direction, torch.float32)
        geometry = PropagationGeometry(
            path_length_m=take(table.path_length_m, torch.float32), delay_s=take(table.delay_s, torch.float32),
            field_direction=direction,
            interaction_positions_m=take(table.interaction_positions, torch.float32),
            interaction_normals=take(table.interaction_normals, torch.float32),
        )
        if request.response == "scalar_transport":
            transport: PropagationTransport = ScalarTransport(coefficient=take(ev["path_field"], torch.complex64))
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
            field = take(ev["field_xyz"], torch.complex64) * amplitude.view(-1, 1)
            transport = Complex3Transport(field=field.contiguous(), direction=direction)
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
    )
    return PropagationEvaluation(paths=paths, convention=_CONVENTION, capabilities=_CAPABILITIES,
                                 diagnostics=diagnostics)


__all__ = [
    "AD_MODES",
    "COMPONENTS",
    "CONTRACT_VERSION",
    "MAX_DEPTH",
    "RESPONSES",
    "TOPOLOGY_MODES",
    "WORLD_VERSION_DOMAINS",
    "Complex3Transport",
    "EndpointBatch",
    "JonesTransport",
    "LoSJonesRows",
    "PropagationCapabilities",
    "PropagationConvention",
    "PropagationDiagnostics",
    "PropagationEvaluation",
    "PropagationGeometry",
    "PropagationPathBatch",
    "PropagationRequest",
    "PropagationTopology",
    "ScalarTransport",
    "capabilities",
    "consumer_los_jones",
    "evaluate",
    "native_frequency_resolution_hz",
]
