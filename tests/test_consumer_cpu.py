"""Propagation consumer contract on the CPU: the capability record, the
structural checks of the request and result records, and the interaction
flags (reference ``propagation/consumer.py``, ``propagation/topology.py``;
tests after ``tests/propagation/test_contracts.py``)."""

from __future__ import annotations

import math

import pytest
import torch

from witwin_channel_b200.propagation import consumer as c


def _interaction_flags_restated(component_id: list[int], depth: list[int], width: int) -> list[list[int]]:
    """The per-slot flag law of reference ``propagation/topology.py:89-107``
    written out row by row: reflection 1 and transmission 4 on every active
    slot, diffraction 2 on slot 0."""
    out = []
    for cid, d in zip(component_id, depth):
        row = [0] * width
        for k in range(width):
            if k < d and cid == 1:
                row[k] = 1
            if k < d and cid == 5:
                row[k] = 4
        if cid == 2 and d > 0 and width:
            row[0] = 2
        out.append(row)
    return out


def test_capability_record_is_frozen_and_truthful():
    caps = c.capabilities()
    assert caps is c.capabilities()
    assert caps.contract_version == c.CONTRACT_VERSION == 6
    assert caps.components == c.COMPONENTS == frozenset({"los", "reflection", "transmission", "diffraction"})
    assert caps.responses == c.RESPONSES
    assert caps.ad_modes == frozenset({"none"})
    for response in caps.responses:
        want = frozenset({"los"}) if response == "polarimetric_transport" else c.COMPONENTS
        assert caps.components_for(response) == want
        assert caps.ad_modes_for(response) == frozenset({"none"})
    assert caps.supports_los_jones
    for component in c.COMPONENTS:
        assert caps.ad_modes_for_component(component) == frozenset({"none"})
    assert caps.material_leaves_for("los") == ()
    assert "layer_eps_r" in caps.material_leaves_for("transmission")
    assert caps.differentiable_geometry_for("discovery") == frozenset()
    assert not caps.supports_fixed_topology and not caps.supports_wideband_offsets
    with pytest.raises(Exception):
        caps.contract_version = 7  # frozen


def test_convention_pair_layout_and_units():
    conv = c.PropagationConvention()
    assert conv.pair_layout == "sink_major_source_minor:pair_index=sink_index*source_count+source_index"
    assert conv.distance_unit == "m" and conv.delay_unit == "s"
    assert conv.phasor == "exp(-j*k*d)"
    assert conv.complex3_basis == "world_cartesian"


def test_native_frequency_resolution():
    assert c.native_frequency_resolution_hz(28.0e9) == math.ulp(28.0e9)
    with pytest.raises(ValueError):
        c.native_frequency_resolution_hz(0.0)
    with pytest.raises(ValueError):
        c.native_frequency_resolution_hz(float("inf"))


def test_endpoint_batch_checks():
    pos = torch.zeros((2, 3), dtype=torch.float32)
    ids = torch.arange(2, dtype=torch.int64)
    pol = torch.zeros((2, 3), dtype=torch.float32)
    with pytest.raises(ValueError, match="CUDA"):
        c.EndpointBatch(stable_ids=ids, positions_m=pos, polarizations=pol)
    with pytest.raises(TypeError):
        c.EndpointBatch(stable_ids=ids, positions_m=pos.double(), polarizations=pol)
    with pytest.raises(ValueError):
        c.EndpointBatch(stable_ids=ids, positions_m=torch.zeros((2, 2)), polarizations=pol)
    with pytest.raises(TypeError):
        c.EndpointBatch(stable_ids=ids, positions_m=[[0.0, 0.0, 0.0]], polarizations=pol)


def test_request_requires_endpoint_batches():
    with pytest.raises(TypeError):
        c.PropagationRequest(sources=None, sinks=None, reference_frequency_hz=1e9, components=frozenset({"los"}),
                             max_depth=0, response="scalar_transport", topology_mode="discover", ad_mode="none")


def _topology(K: int, W: int, **over) -> dict:
    i32 = lambda n: torch.zeros(n, dtype=torch.int32)
    fields = dict(
        source_index=i32(K), sink_index=i32(K), source_id=torch.zeros(K, dtype=torch.int64),
        sink_id=torch.zeros(K, dtype=torch.int64), depth=i32(K), component_id=i32(K), primitive_id=i32(K),
        edge_id=i32(K), material_id=i32(K), primitive_sequence=torch.zeros((K, W), dtype=torch.int32),
        material_sequence=torch.zeros((K, W), dtype=torch.int32), interaction_type=torch.zeros((K, W), dtype=torch.int32),
    )
    fields.update(over)
    return fields


def _geometry(K: int, W: int) -> c.PropagationGeometry:
    return c.PropagationGeometry(path_length_m=torch.zeros(K), delay_s=torch.zeros(K),
                                 field_direction=torch.zeros((K, 3)), interaction_positions_m=torch.zeros((K, W, 3)),
                                 interaction_normals=torch.zeros((K, W, 3)))


def test_row_records_validate_shapes_and_dtypes():
    K, W = 4, 2
    topo = c.PropagationTopology(**_topology(K, W))
    assert topo.row_count == K
    with pytest.raises(TypeError):
        c.PropagationTopology(**_topology(K, W, depth=torch.zeros(K, dtype=torch.int64)))
    with pytest.raises(ValueError):
        c.PropagationTopology(**_topology(K, W, material_sequence=torch.zeros((K, W + 1), dtype=torch.int32)))
    geo = _geometry(K, W)
    with pytest.raises(ValueError):
        c.PropagationGeometry(path_length_m=torch.zeros(K), delay_s=torch.zeros(K), field_direction=torch.zeros((K, 3)),
                              interaction_positions_m=torch.zeros((K, W, 2)), interaction_normals=torch.zeros((K, W, 2)))
    scalar = c.ScalarTransport(coefficient=torch.zeros(K, dtype=torch.complex64))
    with pytest.raises(NotImplementedError):
        c.ScalarTransport(coefficient=torch.zeros(K, dtype=torch.complex64),
                          coefficient_offsets=torch.zeros((K, 1), dtype=torch.complex64), frequency_offsets_hz=(0.0,))
    c3 = c.Complex3Transport(field=torch.zeros((K, 3), dtype=torch.complex64), direction=torch.zeros((K, 3)))
    assert c3.row_count == K
    with pytest.raises(ValueError):
        c.JonesTransport(matrix=torch.zeros((K, 2, 3), dtype=torch.complex64), source_basis=torch.zeros((K, 2, 3)),
                         sink_basis=torch.zeros((K, 2, 3)))
    batch = c.PropagationPathBatch(pair_count=2, path_count=K, pair_index=torch.tensor([0, 0, 1, 1]),
                                   pair_offsets=torch.tensor([0, 2, 4]), topology=topo, geometry=geo, transport=scalar)
    assert batch.path_count == K
    with pytest.raises(ValueError):
        c.PropagationPathBatch(pair_count=2, path_count=K, pair_index=torch.tensor([0, 0, 1, 1]),
                               pair_offsets=torch.tensor([0, 4]), topology=topo, geometry=geo, transport=scalar)
    with pytest.raises(ValueError):
        c.PropagationPathBatch(pair_count=2, path_count=K, pair_index=torch.tensor([0, 0, 1, 1]),
                               pair_offsets=torch.tensor([0, 2, 4]), topology=topo, geometry=_geometry(K - 1, W),
                               transport=scalar)


@pytest.mark.parametrize("width", [0, 1, 3, 5])
def test_interaction_flags_follow_the_reference_law(width):
    g = torch.Generator().manual_seed(width)
    comps = torch.tensor([0, 1, 2, 5], dtype=torch.int32)[torch.randint(0, 4, (64,), generator=g)]
    depth = torch.randint(0, width + 1, (64,), generator=g).to(torch.int32)
    depth = torch.where(comps == 0, torch.zeros_like(depth), depth)
    depth = torch.where(comps == 2, torch.clamp(depth, max=1), depth)
    got = c._interaction_types(comps, depth, width)
    assert got.dtype == torch.int32 and tuple(got.shape) == (64, width)
    assert got.tolist() == _interaction_flags_restated(comps.tolist(), depth.tolist(), width)


def test_los_jones_input_checks_before_any_launch():
    pair = torch.zeros(1, dtype=torch.int64)
    pos = torch.zeros((1, 3), dtype=torch.float32)
    basis = torch.zeros((1, 2, 3), dtype=torch.float32)
    kw = dict(pair_index=pair, source_positions=pos, sink_positions=pos, source_reference_basis=basis,
              sink_reference_basis=basis, frequency_hz=1.0e9)
    with pytest.raises(TypeError):
        c.consumer_los_jones(**{**kw, "pair_index": [0]})
    with pytest.raises(RuntimeError, match="does not support AD"):
        c.consumer_los_jones(**{**kw, "source_positions": pos.clone().requires_grad_()})
    with pytest.raises(TypeError):
        c.consumer_los_jones(**{**kw, "pair_index": pair.int()})
    with pytest.raises(ValueError, match="CUDA"):
        c.consumer_los_jones(**kw)
