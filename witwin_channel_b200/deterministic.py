"""Deterministic radiomap/path solver: the drop-in ``Config``/``Result``/``solve`` contract.

Restates the public contract of the reference's ``witwin/channel/deterministic.py``:
``Config`` (``:105-217``) with its validation, ``PathTable`` (``:222-248``),
``Result`` (``:250-258``), the accumulation semantics (``:281-458``), the path
table (``:461-514``), the pipeline (``:786-949``) and ``solve`` (``:960-971``).
Every stage runs in the native library (``_native``); there is no CPU path.
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import Any

import torch

from . import _native, engine
from .compiler import compile_scene, receiver_setup
from .constants import PHASE_CONVENTION
from .scene import ReceiverGrid

VALID_COMPONENTS = frozenset({"los", "reflection", "diffraction", "transmission", "scattering"})
DEFAULT_COMPONENTS = frozenset({"los", "reflection", "diffraction"})
DEPTH_CAPPED_COMPONENTS = frozenset({"reflection", "transmission"})
AD_MODES = frozenset({"none", "jvp", "vjp"})
_VALID_SORT_KEYS = frozenset({"receiver_transmitter_depth_component"})
_VALID_MAX_PATHS_SCOPES = frozenset({"global", "per_pair"})
_SLOTS = {"los": 0, "reflection": 1, "diffraction": 2, "transmission": 3, "scattering": 4, "coupled": 5}
_BASE_COMPONENTS = ("los", "reflection", "diffraction")
_OPTIONAL_COMPONENTS = ("transmission", "scattering")


@dataclass(frozen=True, slots=True)
class Config:
    max_depth: int = 1
    max_diffraction_order: int = 1
    components: frozenset[str] | set[str] | tuple[str, ...] | list[str] = DEFAULT_COMPONENTS
    coherent: bool = True
    return_field: bool = True
    export_paths: bool = False
    max_paths: int | None = None
    max_paths_scope: str = "global"
    sort_key: str = "receiver_transmitter_depth_component"
    diagnostics: bool = False
    ad_mode: str = "none"
    coupled_paths: bool = False
    coupled_candidate_limit: int = 1_000_000
    scattering_samples_per_m2: float = 8.0
    scattering_max_paths_per_pair: int = 4096
    scattering_power_threshold: float = 0.0
    scattering_coherent: bool = False
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
        if self.max_diffraction_order < 0:
            raise ValueError("max_diffraction_order must be 0 or 1")
        if self.max_diffraction_order > 1:
            raise RuntimeError("max_diffraction_order above 1 is not supported yet")
        components = frozenset(self.components)
        if not components or not components.issubset(VALID_COMPONENTS):
            raise ValueError(f"components must be a non-empty subset of {sorted(VALID_COMPONENTS)}")
        if self.scattering_coherent and "scattering" not in components:
            raise RuntimeError("scattering_coherent=True requires the 'scattering' component")
        if self.max_depth > 5 and components & DEPTH_CAPPED_COMPONENTS:
            raise RuntimeError("deterministic reflection/transmission currently support max_depth <= 5")
        if self.coupled_candidate_limit <= 0:
            raise ValueError("coupled_candidate_limit must be positive")
        if self.max_paths is not None and self.max_paths <= 0:
            raise ValueError("max_paths must be positive when set")
        if self.max_paths_scope not in _VALID_MAX_PATHS_SCOPES:
            raise ValueError("max_paths_scope must be 'global' or 'per_pair'")
        if self.sort_key not in _VALID_SORT_KEYS:
            raise ValueError(f"sort_key must be one of {sorted(_VALID_SORT_KEYS)}")
        if self.ad_mode not in AD_MODES:
            raise RuntimeError(f"deterministic ad_mode must be one of {sorted(AD_MODES)}")
        object.__setattr__(self, "components", components)


@dataclass(frozen=True, slots=True)
class PathTable:
    valid: torch.Tensor
    tx_id: torch.Tensor
    rx_id: torch.Tensor
    depth: torch.Tensor
    component_id: torch.Tensor
    primitive_id: torch.Tensor
    edge_id: torch.Tensor
    path_length_m: torch.Tensor
    delay_s: torch.Tensor
    path_gain: torch.Tensor
    interaction_position: torch.Tensor
    interaction_normal: torch.Tensor
    material_id: torch.Tensor
    primitive_sequence: torch.Tensor
    material_sequence: torch.Tensor
    interaction_positions: torch.Tensor
    interaction_normals: torch.Tensor
    field_real: torch.Tensor
    field_imag: torch.Tensor
    coefficient: torch.Tensor
    field_xyz: torch.Tensor
    field_direction: torch.Tensor
    phase_rad: torch.Tensor
    interaction_count: torch.Tensor


@dataclass(frozen=True, slots=True)
class Result:
    path_gain: torch.Tensor
    field: torch.Tensor
    component_power: dict[str, torch.Tensor]
    component_fields: dict[str, torch.Tensor]
    paths: PathTable | None
    metadata: dict[str, Any]
    diagnostics: dict[str, Any] | None = None


# --------------------------------------------------------------------------
def _frequency_value(reference_frequency_hz: Any) -> float:
    if isinstance(reference_frequency_hz, torch.Tensor):
        if reference_frequency_hz.numel() != 1:
            raise ValueError("reference_frequency_hz must be a scalar")
        value = float(reference_frequency_hz.detach())
    else:
        value = float(reference_frequency_hz)
    if not (value > 0.0):
        raise ValueError("reference_frequency_hz must be positive")
    return value


def _validate(scene: Any, config: Config) -> None:
    if config.coupled_paths:
        raise NotImplementedError("coupled reflection-diffraction paths are outside this engine")
    if "scattering" in config.components:
        raise NotImplementedError("rough-surface scattering is outside this engine")
    if config.isb_boundary_taper:
        raise NotImplementedError("the ISB boundary taper is outside this engine")
    if "reflection" in config.components and config.max_depth < 1:
        raise RuntimeError("deterministic reflection requires max_depth >= 1")
    if "diffraction" in config.components:
        if config.max_depth < 1:
            raise RuntimeError("deterministic diffraction requires max_depth >= 1")
        if config.max_diffraction_order < 1:
            raise RuntimeError("deterministic diffraction requires max_diffraction_order >= 1")
    receivers = scene.receivers
    # scalar endpoints only (reference scene/endpoints.py:173-190): arrays,
    # directional patterns and weights belong to the path solver
    for endpoint in (*scene.transmitters, *receivers):
        if int(getattr(endpoint, "num_antennas", 1)) != 1:
            raise ValueError("the deterministic solver does not support antenna arrays")
        pattern = getattr(endpoint, "pattern", None)
        if pattern is not None and pattern.kind != "isotropic":
            raise ValueError("the deterministic solver does not support directional antenna patterns")
        if getattr(endpoint, "weights", None) is not None:
            raise ValueError("the deterministic solver does not support precoding or combining")
    has_grid = any(isinstance(r, ReceiverGrid) for r in receivers)
    if has_grid and len(receivers) > 1 and not config.export_paths:
        raise RuntimeError("mixed point/grid receivers require export_paths=True")
    if not torch.cuda.is_available():
        raise RuntimeError("witwin_channel_b200.deterministic requires CUDA")


def _endpoints(scene: Any, device: torch.device) -> engine.Endpoints:
    txs = scene.transmitters
    if txs:
        # positions, powers and polarisations in one host buffer and one copy
        T = len(txs)
        host = torch.empty(7 * T, dtype=torch.float32)
        host[:3 * T] = torch.stack([t.position.detach().to(torch.float32).reshape(3) for t in txs]).reshape(-1)
        host[3 * T:4 * T] = torch.tensor([float(t.power_w.detach()) if isinstance(t.power_w, torch.Tensor)
                                          else float(t.power_w) for t in txs], dtype=torch.float32)
        host[4 * T:] = torch.stack([t.polarization.detach().to(torch.float32).reshape(3) for t in txs]).reshape(-1)
        buf = host.pin_memory().to(device, non_blocking=True)
        pos = buf[:3 * T].view(T, 3)
        pw = buf[3 * T:4 * T]
        pol = buf[4 * T:].view(T, 3)
    else:
        pos = torch.zeros((0, 3), dtype=torch.float32, device=device)
        pw = torch.zeros((0,), dtype=torch.float32, device=device)
        pol = torch.zeros((0, 3), dtype=torch.float32, device=device)
    return engine.Endpoints(tx_pos=pos, tx_power=pw, tx_pol=pol, rx=receiver_setup(scene, device))


def _layout(values: torch.Tensor, rx: dict) -> torch.Tensor:
    """Grid results are ``(T, shape[1], shape[0])`` (propagation/geometry.py:79-89)."""
    if rx["kind"] == "grid":
        rows, cols = rx["shape"]
        return values.reshape(values.shape[0], rows, cols).transpose(1, 2).contiguous()
    return values.contiguous()


def _metadata(config: Config, counts: dict, path_count: int, launches: int, extra: dict) -> dict:
    components = {c: ("enabled" if c in config.components else "not_requested") for c in sorted(VALID_COMPONENTS)}
    if "transmission" in config.components:
        components["transmission"] = "enabled" if counts.get("transmission", 0) > 0 else "enabled_no_paths"
    meta = {
        "max_depth": config.max_depth,
        "max_diffraction_order": config.max_diffraction_order,
        "coherent": config.coherent,
        "return_field": config.return_field,
        "export_paths": config.export_paths,
        "max_paths": config.max_paths,
        "max_paths_scope": config.max_paths_scope,
        "sort_key": config.sort_key,
        "accumulation_strategy": "coherent" if config.coherent else "incoherent",
        "components": components,
        "counts": {"path_count": path_count, "valid_path_count": path_count, "components": counts},
        "capability": {"native": True, "cuda_available": True, "arch": "sm_100a"},
        "kernel": {"primitive": "deterministic_solver", "forward_launch_count": launches,
                   "accumulation_strategy": "register_sum_one_write_per_cell", "ad_status": config.ad_mode},
        "field_abi": "complex3_v1",
        "phase_convention": dict(PHASE_CONVENTION),
        "coefficient_semantics": "unit_excitation_dimensionless_receiver_projection",
        "coupled_paths": {"requested": False, "geometry": "not_requested", "coefficient": "not_requested"},
    }
    if "transmission" in config.components:
        meta["transmission"] = {"thin_sheet_straight_path_approximation": True, "group_delay": "geometric"}
    meta.update(extra)
    return meta


def _component_counts(component_id: torch.Tensor) -> dict[str, int]:
    """Rows per component (one device-to-host copy)."""
    n = torch.bincount(component_id.to(torch.int64), minlength=8).cpu().tolist() if component_id.numel() else [0] * 8
    return {name: int(n[c]) for name, c in (("los", 0), ("reflection", 1), ("diffraction", 2), ("transmission", 5))}


def _needs_rows(config: Config) -> bool:
    return config.export_paths or config.max_paths is not None or config.ad_mode != "none"


def solve(scene: Any, config: Config, *, reference_frequency_hz, precision: str = "mixed") -> Result:
    """Run the deterministic propagation pipeline on the GPU.

    ``precision`` selects ``"mixed"`` (FP32 traversal and fields; FP64 image
    solve, path length and phase) or ``"fp64"`` (every stage in FP64; cell
    mode, or the differentiable forward of ``ad_mode="vjp"``/``"jvp"``).
    """

    if not isinstance(config, Config):
        raise TypeError("config must be a witwin_channel_b200.deterministic.Config")
    frequency = _frequency_value(reference_frequency_hz)
    _validate(scene, config)
    if config.ad_mode in ("vjp", "jvp"):
        # one differentiable fixed-topology forward serves both modes: reverse
        # mode through backward(), forward mode through the jvp of the same
        # autograd Function when the scene values are forward-mode dual tensors
        from .autograd import solve_vjp

        return solve_vjp(scene, config, reference_frequency_hz, precision=precision)
    device = torch.device("cuda", torch.cuda.current_device())
    compiled = compile_scene(scene, device)
    ep = _endpoints(scene, device)
    mats = compiled.material_tables([frequency], device)
    bits = engine.component_bits(config.components)
    T, R = ep.num_tx, ep.num_rx
    launches0 = _native.launch_count()
    prec = _native.PRECISION_FP64 if precision == "fp64" else _native.PRECISION_MIXED
    paths = None
    counts: dict[str, int] = {}
    extra: dict[str, Any] = {}
    if _needs_rows(config):
        if prec == _native.PRECISION_FP64:
            raise NotImplementedError("fp64 precision is provided for cell-mode solves")
        res = engine.run_solve(compiled, ep, mats, [frequency], components=bits, max_depth=config.max_depth,
                               coherent=config.coherent, want_rows=True)
        rows = res["rows"]
        width = max(int(config.max_depth), 0)
        selected = engine.select_rows(rows, width, config.max_paths, config.max_paths_scope)
        ev = engine.evaluate_rows(compiled, ep, mats, [frequency], 0, rows, selected, width, components=bits,
                                  max_depth=config.max_depth, coherent=config.coherent)
        cells = engine.accumulate_rows(rows, selected, ev["path_gain"], ev["path_field"], ev["field_xyz"], ep.tx_power,
                                       T, R, config.coherent)
        dec = engine.decode_rows(rows, selected)
        counts.update(_component_counts(dec["component_id"]))
        path_count = int(selected.shape[0])
        if config.export_paths:
            paths = _path_table(dec, ev, width, compiled, config.return_field)
    else:
        cells = engine.alloc_cells(1, T, R, device, fp64=(prec == _native.PRECISION_FP64))
        res = engine.run_solve(compiled, ep, mats, [frequency], components=bits, max_depth=config.max_depth,
                               coherent=config.coherent, precision=prec, cells=cells)
        path_count = -1
    if "transmission" in config.components:
        # tx-rx segments crossing more than max_depth walls (no transmission path)
        extra["transmission_overflow"] = int(res["transmission_overflow"].item())
    rx = ep.rx
    path_gain = cells.path_gain[0]
    field = cells.field[0]
    extra_components = tuple(n for n in _OPTIONAL_COMPONENTS if n in config.components)
    names = _BASE_COMPONENTS + extra_components
    comp_power = {n: _layout(cells.comp_power[_SLOTS[n], 0], rx) for n in names}
    comp_fields = {n: (_layout(cells.comp_field[_SLOTS[n], 0], rx) if config.return_field
                       else torch.empty((0,), dtype=torch.complex64, device=device)) for n in names}
    exact = None
    if "diffraction" in config.components and rx["kind"] == "grid" and len(scene.receivers) == 1:
        exact = _layout(cells.diff_vec_power[0], rx)
        previous = comp_power["diffraction"]
        comp_power["diffraction"] = exact
        if not config.coherent:
            path_gain = path_gain - _layout_inverse(previous, rx) + _layout_inverse(exact, rx)
    launches = _native.launch_count() - launches0
    meta = _metadata(config, counts, path_count, launches, extra)
    diagnostics = None
    if config.diagnostics:
        diagnostics = {
            "path_gain_shape": tuple(_layout(path_gain, rx).shape),
            "path_count": path_count,
            "component_counts": counts,
            "coherent": config.coherent,
            "accumulation_mode": "coherent" if config.coherent else "incoherent",
            "native_launch_count": launches,
            "diffraction_accumulation": "exact_vector_coherent_paths" if exact is not None else "scalar_path_accumulation",
            "scene": {"faces": compiled.native.num_faces, "groups": compiled.native.num_groups,
                      "edges": compiled.native.num_edges, "bvh_depth": compiled.native.bvh_depth},
        }
    return Result(
        path_gain=_layout(path_gain, rx),
        field=_layout(field, rx) if config.return_field else torch.empty((0,), dtype=torch.complex64, device=device),
        component_power=comp_power,
        component_fields=comp_fields,
        paths=paths,
        metadata=meta,
        diagnostics=diagnostics,
    )


def _layout_inverse(values: torch.Tensor, rx: dict) -> torch.Tensor:
    if rx["kind"] == "grid":
        rows, cols = rx["shape"]
        return values.transpose(1, 2).reshape(values.shape[0], rows * cols)
    return values


def _path_table(dec: dict, ev: dict, width: int, compiled, include_fields: bool) -> PathTable:
    device = dec["tx_id"].device
    K = int(dec["tx_id"].shape[0])
    seq = dec["seq"][:, :width].contiguous()
    cid = dec["component_id"]
    prim = torch.where((cid == 1) | (cid == 5), dec["seq"][:, 0], torch.full_like(cid, -1))
    fm = compiled.face_material.to(torch.int32)
    if fm.numel():
        mat_seq = torch.where(seq >= 0, fm[seq.clamp_min(0).long()], torch.full_like(seq, -1))
        mat_id = torch.where(prim >= 0, fm[prim.clamp_min(0).long()], torch.full_like(prim, -1))
    else:
        mat_seq = torch.full_like(seq, -1)
        mat_id = torch.full_like(prim, -1)
    pos = ev["interaction_positions"][:, :width].contiguous()
    nrm = ev["interaction_normals"][:, :width].contiguous()
    first_pos = ev["interaction_positions"][:, 0].contiguous() if K else torch.zeros((0, 3), device=device)
    first_nrm = ev["interaction_normals"][:, 0].contiguous() if K else torch.zeros((0, 3), device=device)
    has_event = (dec["depth"] > 0).unsqueeze(-1)
    first_pos = torch.where(has_event, first_pos, torch.zeros_like(first_pos))
    first_nrm = torch.where(has_event, first_nrm, torch.zeros_like(first_nrm))
    if include_fields:
        pf = ev["path_field"]
        phase = ev["phase_rad"]
    else:
        pf = torch.sqrt(ev["path_gain"]).to(torch.complex64)
        phase = torch.zeros_like(ev["path_gain"])
    edge = torch.where(cid == 2, dec["edge_id"], torch.full_like(cid, -1))
    return PathTable(
        valid=torch.ones(K, dtype=torch.bool, device=device),
        tx_id=dec["tx_id"], rx_id=dec["rx_id"], depth=dec["depth"], component_id=cid,
        primitive_id=prim.contiguous(), edge_id=edge.contiguous(),
        path_length_m=ev["path_length_m"], delay_s=ev["delay_s"], path_gain=ev["path_gain"],
        interaction_position=first_pos, interaction_normal=first_nrm, material_id=mat_id.contiguous(),
        primitive_sequence=seq, material_sequence=mat_seq.contiguous(), interaction_positions=pos,
        interaction_normals=nrm, field_real=pf.real.contiguous(), field_imag=pf.imag.contiguous(),
        coefficient=ev["coefficient"], field_xyz=ev["field_xyz"], field_direction=ev["field_direction"],
        phase_rad=phase, interaction_count=dec["depth"].contiguous(),
    )


__all__ = ["Config", "PathTable", "Result", "solve"]
