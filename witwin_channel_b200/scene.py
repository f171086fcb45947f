"""Minimal logical scene model for the deterministic solver.

The reference takes its scene objects from ``witwin.core`` (``witwin==0.4.0``),
which is a separate package.  This module defines the subset of that model the
deterministic path reads, duck-type compatible with it, so that user code
written against ``witwin.core`` (``Scene``, ``Structure``, ``Mesh``,
``PhysicalMaterial``, ``MaterialLayer``, ``AntennaState``, ``ReceiverGrid``)
keeps working.  Field usage follows the reference's fixtures
(``tests/support/core_world.py:9-75``, ``tests/support/scenes.py``) and its
compiler (``witwin/channel/scene/compiler.py:967-1035``).

Material parameters may be Python floats, callables of the frequency in Hz
(dispersive ITU-style laws), or 0-d torch tensors; a tensor that requires
grad receives a gradient from a ``vjp`` solve.
"""

from __future__ import annotations

import itertools
from dataclasses import dataclass, field
from typing import Any, Callable, Sequence

import torch

_ids = itertools.count(1)


def new_antenna_id() -> int:
    return next(_ids)


MaterialValue = float | torch.Tensor | Callable[[float], float]


def evaluate_material_value(value: MaterialValue, frequency_hz: float) -> Any:
    """Return a float or a 0-d tensor for a material parameter at ``frequency_hz``."""

    if callable(value) and not isinstance(value, torch.Tensor):
        return value(frequency_hz)
    return value


@dataclass(frozen=True)
class MaterialLayer:
    """One physical layer of a thin-sheet stack (entry side first)."""

    thickness_m: MaterialValue
    eps_r: MaterialValue
    sigma_e: MaterialValue = 0.0
    mu_r: MaterialValue = 1.0


_GEOMETRY_MODES = ("thin_sheet", "volumetric")


@dataclass(frozen=True)
class PhysicalMaterial:
    """Per-structure electromagnetic material.

    Without explicit ``layers`` the material is one layer of
    ``(thickness_m, eps_r, sigma_e, mu_r)``; with layers, the first layer is the
    scalar Fresnel view used by reflection and the whole stack is used by
    transmission (``witwin/channel/scene/compiler.py:967-1035``).
    """

    eps_r: MaterialValue = 1.0
    sigma_e: MaterialValue = 0.0
    mu_r: MaterialValue = 1.0
    gain: MaterialValue = 1.0
    thickness_m: MaterialValue = 0.2
    layers: tuple[MaterialLayer, ...] = ()
    conductor_model: str | None = None
    geometry_mode: str = "thin_sheet"
    name: str = ""

    def __post_init__(self) -> None:
        if self.geometry_mode not in _GEOMETRY_MODES:
            raise ValueError(f"geometry_mode must be one of {_GEOMETRY_MODES}")

    @classmethod
    def perfect_conductor(cls, *, thickness_m: float = 0.2, name: str = "pec") -> "PhysicalMaterial":
        return cls(eps_r=1.0, sigma_e=0.0, conductor_model="perfect", thickness_m=thickness_m, name=name)

    def stack(self) -> tuple[MaterialLayer, ...]:
        if self.layers:
            return tuple(self.layers)
        return (
            MaterialLayer(
                thickness_m=self.thickness_m,
                eps_r=self.eps_r,
                sigma_e=self.sigma_e,
                mu_r=self.mu_r,
            ),
        )


@dataclass
class Mesh:
    vertices: torch.Tensor
    faces: torch.Tensor

    def __post_init__(self) -> None:
        if not isinstance(self.vertices, torch.Tensor):
            self.vertices = torch.as_tensor(self.vertices, dtype=torch.float32)
        if not isinstance(self.faces, torch.Tensor):
            self.faces = torch.as_tensor(self.faces, dtype=torch.int64)
        if self.vertices.ndim != 2 or self.vertices.shape[-1] != 3:
            raise ValueError("vertices must have shape (V, 3)")
        if self.faces.ndim != 2 or self.faces.shape[-1] != 3:
            raise ValueError("faces must have shape (F, 3)")


class Structure:
    """A triangle mesh with one material.  ``surface_id`` keys coplanar grouping."""

    def __init__(
        self,
        geometry: Mesh | None = None,
        material: PhysicalMaterial | None = None,
        *,
        vertices: torch.Tensor | None = None,
        faces: torch.Tensor | None = None,
        surface_id: int | None = None,
        name: str = "",
        **_: Any,
    ) -> None:
        if geometry is None:
            if vertices is None or faces is None:
                raise ValueError("Structure needs a Mesh or vertices and faces")
            geometry = Mesh(vertices, faces)
        if material is None:
            raise ValueError("Structure needs a material")
        self.geometry = geometry
        self.material = material
        self.surface_id = surface_id
        self.name = name

    @property
    def vertices(self) -> torch.Tensor:
        return self.geometry.vertices

    @property
    def faces(self) -> torch.Tensor:
        return self.geometry.faces


def _vec3(value: Any) -> torch.Tensor:
    if isinstance(value, torch.Tensor):
        return value.reshape(3)
    return torch.tensor(tuple(float(v) for v in value), dtype=torch.float32)


_PATTERN_KINDS = ("isotropic", "vertical", "horizontal", "custom")


class AntennaPattern:
    """Element field pattern in the endpoint-local frame (the reference's
    ``witwin.core.AntennaPattern``, evaluated by
    ``witwin/channel/scene/endpoints.py:66-95``): ``isotropic`` (1),
    ``vertical`` (sqrt(1 - z^2)), ``horizontal`` (sqrt(1 - x^2)) of the local
    unit direction, or ``custom`` (a callable of the (..., 3) local unit
    directions returning their complex responses)."""

    def __init__(self, kind: str = "isotropic", custom: Any = None) -> None:
        if kind not in _PATTERN_KINDS:
            raise ValueError(f"pattern kind must be one of {_PATTERN_KINDS}")
        if (kind == "custom") != (custom is not None):
            raise ValueError("a custom pattern needs its callable, and only a custom pattern takes one")
        self.kind = kind
        self.custom = custom


def _pattern(value: Any) -> AntennaPattern:
    if isinstance(value, AntennaPattern):
        return value
    if value is None:
        return AntennaPattern("isotropic")
    if isinstance(value, str):
        return AntennaPattern(value)
    raise TypeError("pattern must be an AntennaPattern or a pattern kind string")


def orientation_matrix(orientation: torch.Tensor) -> torch.Tensor:
    """Local-to-world rotation of a ``(yaw, pitch, roll)`` orientation in
    radians, intrinsic Z-Y-X (reference ``scene/endpoints.py:42-63``)."""

    o = torch.as_tensor(orientation, dtype=torch.float32).reshape(-1)
    if o.shape != (3,):
        raise ValueError("orientation must be (yaw, pitch, roll)")
    yaw, pitch, roll = o.unbind()
    cy, sy = torch.cos(yaw), torch.sin(yaw)
    cp, sp = torch.cos(pitch), torch.sin(pitch)
    cr, sr = torch.cos(roll), torch.sin(roll)
    return torch.stack((
        torch.stack((cy * cp, cy * sp * sr - sy * cr, cy * sp * cr + sy * sr)),
        torch.stack((sy * cp, sy * sp * sr + cy * cr, sy * sp * cr - cy * sr)),
        torch.stack((-sp, cp * sr, cp * cr)),
    )).to(torch.float32)


class _ArrayEndpoint:
    """Antenna-array attributes shared by point endpoints and receiver grids:
    element positions (A, 3) in the local frame (one element at the origin
    by default), orientation, element pattern, per-element weights
    (precoding on a transmitter, combining on a receiver) and whether the
    array is synthetic (one traced path set, far-field phase per element) or
    explicit (every element traced)."""

    def _init_array(self, *, orientation: Any, element_positions: Any, weights: Any, synthetic_array: bool,
                    pattern: Any) -> None:
        self.orientation = None if orientation is None else torch.as_tensor(orientation, dtype=torch.float32).reshape(3)
        if element_positions is None:
            positions = torch.zeros((1, 3), dtype=torch.float32)
        else:
            positions = torch.as_tensor(element_positions, dtype=torch.float32)
            if positions.ndim != 2 or positions.shape[1] != 3 or positions.shape[0] < 1:
                raise ValueError("element_positions must have shape (A, 3) with A >= 1")
        self.element_positions = positions
        if weights is not None:
            weights = torch.as_tensor(weights).to(torch.complex64).reshape(-1)
            if weights.shape[0] != positions.shape[0]:
                raise ValueError("weights must hold one entry per antenna element")
        self.weights = weights
        self.synthetic_array = bool(synthetic_array)
        self.pattern = _pattern(pattern)

    @property
    def num_antennas(self) -> int:
        return int(self.element_positions.shape[0])

    @property
    def precoding(self) -> torch.Tensor | None:
        return self.weights if getattr(self, "role", None) == "tx" else None

    @property
    def combining(self) -> torch.Tensor | None:
        return self.weights if getattr(self, "role", None) == "rx" else None

    def rotation(self) -> torch.Tensor:
        return torch.eye(3) if self.orientation is None else orientation_matrix(self.orientation)

    def element_world_positions(self, origin: torch.Tensor) -> torch.Tensor:
        """World positions of the elements about ``origin`` (reference
        ``scene/endpoints.py:201-205``)."""
        return origin.reshape(1, 3).to(torch.float32) + self.element_positions @ self.rotation().T


class AntennaState(_ArrayEndpoint):
    """A transmitter (``role="tx"``) or point receiver (``role="rx"``), with
    an optional antenna array (see :class:`_ArrayEndpoint`).

    ``polarization`` is the world polarization: the given vector, or (0, 0, 1)
    ((1, 0, 0) for a horizontal pattern), normalised and turned by the
    orientation when one is given."""

    def __init__(
        self,
        id: int,
        role: str,
        position: Any,
        *,
        polarization: Any = None,
        power_w: float | torch.Tensor = 1.0,
        orientation: Any = None,
        element_positions: Any = None,
        weights: Any = None,
        synthetic_array: bool = True,
        pattern: Any = "isotropic",
        **_: Any,
    ) -> None:
        if role not in ("tx", "rx"):
            raise ValueError("role must be 'tx' or 'rx'")
        self.id = id
        self.role = role
        self.position = _vec3(position)
        self._init_array(orientation=orientation, element_positions=element_positions, weights=weights,
                         synthetic_array=synthetic_array, pattern=pattern)
        default = (1.0, 0.0, 0.0) if self.pattern.kind == "horizontal" else (0.0, 0.0, 1.0)
        pol = torch.tensor(default) if polarization is None else _vec3(polarization)
        if self.orientation is not None:
            pol = self.rotation() @ (pol.float() / torch.linalg.vector_norm(pol.float()))
        self.polarization = pol
        self.power_w = 1.0 if power_w is None else power_w


ReceiverPoint = AntennaState


class ReceiverGrid(_ArrayEndpoint):
    """A planar receiver grid.

    Point ``(row, col)`` sits at ``origin + x_axis*row*spacing[0] +
    y_axis*col*spacing[1]``; results come back as ``(T, shape[1], shape[0])``
    (``witwin/channel/propagation/geometry.py:71-89``; ``los.cu:391-420``).
    Every grid point carries the grid's antenna array (synthetic only).
    """

    role = "rx"

    def __init__(
        self,
        id: int,
        origin: Any,
        x_axis: Any,
        y_axis: Any,
        shape: Sequence[int],
        spacing: Sequence[float],
        *,
        polarization: Any = None,
        orientation: Any = None,
        element_positions: Any = None,
        weights: Any = None,
        synthetic_array: bool = True,
        pattern: Any = "isotropic",
        **_: Any,
    ) -> None:
        self._init_array(orientation=orientation, element_positions=element_positions, weights=weights,
                         synthetic_array=synthetic_array, pattern=pattern)
        rows, cols = (int(shape[0]), int(shape[1]))
        if rows < 0 or cols < 0:
            raise ValueError("shape entries must be non-negative")
        if float(spacing[0]) <= 0.0 or float(spacing[1]) <= 0.0:
            raise ValueError("spacing entries must be positive")
        self.id = id
        self.origin = _vec3(origin)
        self.x_axis = _vec3(x_axis)
        self.y_axis = _vec3(y_axis)
        self.shape = (rows, cols)
        self.spacing = (float(spacing[0]), float(spacing[1]))
        default = (1.0, 0.0, 0.0) if self.pattern.kind == "horizontal" else (0.0, 0.0, 1.0)
        pol = torch.tensor(default) if polarization is None else _vec3(polarization)
        if self.orientation is not None:
            pol = self.rotation() @ (pol.float() / torch.linalg.vector_norm(pol.float()))
        self.polarization = pol
        self.position = self.origin

    @property
    def count(self) -> int:
        return self.shape[0] * self.shape[1]

    def points(self) -> torch.Tensor:
        """Grid points in float32, row-major over ``(row, col)``."""

        rows, cols = self.shape
        r = torch.arange(rows, dtype=torch.float32).repeat_interleave(cols) * self.spacing[0]
        c = torch.arange(cols, dtype=torch.float32).repeat(rows) * self.spacing[1]
        o = self.origin.detach().float()
        return o[None, :] + self.x_axis.float()[None, :] * r[:, None] + self.y_axis.float()[None, :] * c[:, None]


_EDGE_SELECTION_MODES = ("all_edges", "vertical_only")
_BOUNDARY_EDGE_POLICIES = ("exclude", "half_plane")


@dataclass
class EdgePolicy:
    """Diffraction edge selection read from ``scene.metadata["imported_edge_policy"]``
    (same fields and checks as the reference's ``scene/resources.py:248-273``):
    ``vertical_only`` keeps edges with |dz|/length above ``vertical_ratio``;
    boundary edges (one adjacent face) are kept as half-planes or excluded."""

    vertical_ratio: float = 0.7
    edge_selection_mode: str = "all_edges"
    edge_diffraction: bool | None = True
    boundary_edge_policy: str | None = None

    def __post_init__(self) -> None:
        mode = str(self.edge_selection_mode)
        if mode not in _EDGE_SELECTION_MODES:
            raise ValueError(f"edge_selection_mode must be one of {sorted(_EDGE_SELECTION_MODES)}")
        wanted = None if self.edge_diffraction is None else bool(self.edge_diffraction)
        if self.boundary_edge_policy is None:
            boundary = "exclude" if wanted is False else "half_plane"
        else:
            boundary = str(self.boundary_edge_policy)
        if boundary not in _BOUNDARY_EDGE_POLICIES:
            raise ValueError(f"boundary_edge_policy must be one of {sorted(_BOUNDARY_EDGE_POLICIES)}")
        if wanted is not None and wanted != (boundary == "half_plane"):
            raise ValueError(f"edge_diffraction={wanted!r} conflicts with boundary_edge_policy={boundary!r}")
        self.vertical_ratio = float(self.vertical_ratio)
        self.edge_selection_mode = mode
        self.edge_diffraction = boundary == "half_plane"
        self.boundary_edge_policy = boundary


@dataclass
class Scene:
    structures: list[Structure] = field(default_factory=list)
    endpoints: list[Any] = field(default_factory=list)
    metadata: dict[str, Any] = field(default_factory=dict)
    versions: Any = None

    @property
    def transmitters(self) -> list[AntennaState]:
        return [e for e in self.endpoints if getattr(e, "role", None) == "tx"]

    @property
    def receivers(self) -> list[Any]:
        return [e for e in self.endpoints if getattr(e, "role", None) == "rx"]


_ARRAY_KEYS = ("orientation", "element_positions", "weights", "synthetic_array", "pattern")


def make_transmitter(position: Any, *, polarization: Any = None, power_w: float = 1.0, **kw: Any) -> AntennaState:
    return AntennaState(new_antenna_id(), "tx", position, polarization=polarization, power_w=power_w,
                        **{k: kw[k] for k in _ARRAY_KEYS if k in kw})


def make_receiver(position: Any, *, polarization: Any = None, **kw: Any) -> AntennaState:
    return AntennaState(new_antenna_id(), "rx", position, polarization=polarization,
                        **{k: kw[k] for k in _ARRAY_KEYS if k in kw})


def make_receiver_grid(*, origin: Any, x_axis: Any, y_axis: Any, shape: Sequence[int], spacing: Sequence[float], polarization: Any = None, **kw: Any) -> ReceiverGrid:
    return ReceiverGrid(new_antenna_id(), origin, x_axis, y_axis, shape, spacing, polarization=polarization,
                        **{k: kw[k] for k in _ARRAY_KEYS if k in kw})


def make_mesh_structure(*, vertices: Any, faces: Any, material: PhysicalMaterial, surface_id: int | None = None, name: str = "", **kw: Any) -> Structure:
    return Structure(Mesh(vertices, faces), material, surface_id=surface_id, name=name)


__all__ = [
    "AntennaPattern",
    "AntennaState",
    "MaterialLayer",
    "Mesh",
    "PhysicalMaterial",
    "ReceiverGrid",
    "ReceiverPoint",
    "Scene",
    "Structure",
    "evaluate_material_value",
    "make_mesh_structure",
    "make_receiver",
    "make_receiver_grid",
    "make_transmitter",
    "orientation_matrix",
]
