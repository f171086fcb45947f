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
    assert caps.ad_modes == c.AD_MODES == frozenset({"none", "jvp", "vjp"})
    for response in caps.responses:
        want = frozenset({"los"}) if response == "polarimetric_transport" else c.COMPONENTS
        assert caps.components_for(response) == want
        want_ad = frozenset({"none"}) if response == "polarimetric_transport" else c.AD_MODES
        assert caps.ad_modes_for(response) == want_ad
    assert caps.supports_los_jones
    for component in c.COMPONENTS:
        assert caps.ad_modes_for_component(component) == c.AD_MODES
    for name in ("materials.gain", "materials.mu_r", "materials.thickness_m", "sources.powers_w"):
        assert name in caps.primal_only_ad_inputs
    assert not caps.supports_higher_order_ad
    assert caps.material_leaves_for("los") == ()
    assert "layer_eps_r" in caps.material_leaves_for("transmission")
    assert caps.differentiable_geometry_for("discovery") == frozenset()
    assert caps.differentiable_geometry_for("fixed_topology") == frozenset({"path_length_m", "delay_s"})
    assert caps.supports_fixed_topology and caps.supports_wideband_offsets and caps.supports_slot_batching
    assert caps.fixed_topology_components == frozenset({"los", "reflection"})
    assert caps.fixed_topology_row_validity_components == frozenset({"los", "reflection"})
    assert caps.fixed_topology_responses == c.RESPONSES
    assert caps.wideband_responses == frozenset({"scalar_transport", "complex3_transport"})
    assert caps.world_motions == frozenset({"frozen_world", "fixed_winner_replay"})
    assert caps.max_slot_count is None and caps.max_frequency_offset_count is None
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
    wide = c.ScalarTransport(coefficient=torch.zeros(K, dtype=torch.complex64),
                             coefficient_offsets=torch.zeros((K, 2), dtype=torch.complex64),
                             frequency_offsets_hz=(0.0, 1.0e6))
    assert wide.coefficient_offsets.shape == (K, 2)
    with pytest.raises(ValueError, match="paired"):
        c.ScalarTransport(coefficient=torch.zeros(K, dtype=torch.complex64),
                          coefficient_offsets=torch.zeros((K, 1), dtype=torch.complex64))
    with pytest.raises(ValueError, match="shape"):
        c.ScalarTransport(coefficient=torch.zeros(K, dtype=torch.complex64),
                          coefficient_offsets=torch.zeros((K, 1), dtype=torch.complex64), frequency_offsets_hz=(0.0, 1.0))
    with pytest.raises(ValueError, match="shape"):
        c.Complex3Transport(field=torch.zeros((K, 3), dtype=torch.complex64), direction=torch.zeros((K, 3)),
                            field_offsets=torch.zeros((K, 3), dtype=torch.complex64), frequency_offsets_hz=(5.0,))
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


# --- fixed-topology replay: host logic (reference consumer.py:94-135, 466-512,
# 1228-1650; tests after tests/propagation/test_fixed_topology*.py) ---------


def test_frequency_offset_grid_checks():
    assert c.require_frequency_offsets(None) is None
    assert c.require_frequency_offsets((0.0, 1e6, -2e6)) == (0.0, 1e6, -2e6)
    assert c.require_frequency_offsets((1, 2)) == (1.0, 2.0)
    with pytest.raises(TypeError):
        c.require_frequency_offsets(torch.tensor([0.0]))
    with pytest.raises(TypeError):
        c.require_frequency_offsets([0.0])
    with pytest.raises(ValueError):
        c.require_frequency_offsets(())
    with pytest.raises(TypeError):
        c.require_frequency_offsets((True,))
    with pytest.raises(ValueError):
        c.require_frequency_offsets((float("nan"),))
    with pytest.raises(ValueError, match="repeat"):
        c.require_frequency_offsets((1.0, 1.0))
    with pytest.raises(ValueError, match="resolution"):
        c._require_resolvable_offsets((math.ulp(28e9) / 4,), 28e9)
    with pytest.raises(ValueError, match="closer"):
        c._require_resolvable_offsets((1.0e6, 1.0e6 + math.ulp(28e9) / 2), 28e9)
    with pytest.raises(ValueError, match="non-positive"):
        c._require_resolvable_offsets((-30e9,), 28e9)
    c._require_resolvable_offsets((0.0, 1.0e6), 28e9)


def test_world_provenance_names_the_first_moved_domain():
    a = c.WorldProvenance(topology_version=1, geometry_version=2, material_version=3, assignment_version=4)
    assert a.moved_domain(c.WorldProvenance(1, 2, 3, 4)) is None
    assert a.moved_domain(c.WorldProvenance(1, 9, 3, 4)) == "geometry_version"
    assert a.moved_domain(c.WorldProvenance(1, 9, 3, 4), allow_geometry=True) is None
    assert a.moved_domain(c.WorldProvenance(1, 9, 8, 4), allow_geometry=True) == "material_version"
    assert a.moved_domain(c.WorldProvenance(7, 9, 8, 0)) == "topology_version"

    class Compiled:
        topology_version, geometry_version, material_version, assignment_version = 5, 6, 7, 8

    assert c.WorldProvenance.of(Compiled()).moved_domain(c.WorldProvenance(5, 6, 7, 8)) is None


def _frozen(component, depth, seq, source=None, sink=None) -> c.PropagationTopology:
    K = len(component)
    seq_t = torch.as_tensor(seq, dtype=torch.int32).reshape(K, -1 if K else 2)
    W = int(seq_t.shape[1])
    src = torch.tensor(source if source is not None else [0] * K, dtype=torch.int32)
    snk = torch.tensor(sink if sink is not None else list(range(K)), dtype=torch.int32)
    return c.PropagationTopology(**_topology(
        K, W, component_id=torch.tensor(component, dtype=torch.int32), depth=torch.tensor(depth, dtype=torch.int32),
        primitive_sequence=seq_t, source_index=src, sink_index=snk, source_id=src.long() + 100,
        sink_id=snk.long() + 200))


def test_prepare_partitions_by_component_and_depth():
    topo = _frozen([1, 0, 1, 1, 0], [2, 0, 1, 2, 0], [[3, 4], [-1, -1], [5, -1], [6, 7], [-1, -1]])
    prepared = c.prepare_fixed_topology(topo)
    got = [(b.component, b.depth, b.rows.tolist()) for b in prepared.buckets]
    assert got == [("los", 0, [1, 4]), ("reflection", 1, [2]), ("reflection", 2, [0, 3])]
    assert prepared.execution_order.tolist() == [1, 4, 2, 0, 3]
    assert prepared.execution_order.dtype == torch.int32
    assert (prepared.prepare_d2h_copies, prepared.prepare_synchronizations) == (5, 5)
    assert prepared.row_count == 5 and prepared.provenance is None
    empty = c.prepare_fixed_topology(_frozen([], [], torch.zeros((0, 2))))
    assert empty.buckets == () and empty.prepare_d2h_copies == 0


@pytest.mark.parametrize("component, depth, seq, error", [
    ([1], [2], [[3, -1]], ValueError),        # active slot holds -1
    ([1], [1], [[3, 4]], ValueError),         # unused slot not -1
    ([1], [3], [[3, 4]], ValueError),         # depth beyond the sequence width
    ([0], [1], [[3, -1]], ValueError),        # a los row with an interaction
    ([1], [0], [[-1, -1]], ValueError),       # a reflection row without one
    ([2], [1], [[3, -1]], NotImplementedError),  # diffraction is not freezable
    ([5], [1], [[3, -1]], NotImplementedError),  # nor transmission
])
def test_prepare_refuses_malformed_or_unfreezable_rows(component, depth, seq, error):
    with pytest.raises(error):
        c.prepare_fixed_topology(_frozen(component, depth, seq))
    with pytest.raises(TypeError):
        c.prepare_fixed_topology("rows")


def test_replicate_over_slots_is_index_arithmetic():
    topo = _frozen([1, 0, 1], [1, 0, 1], [[3], [-1], [5]], source=[0, 1, 0], sink=[0, 0, 1])
    prepared = c.prepare_fixed_topology(topo)
    assert c.replicate_over_slots(prepared, 1, source_count=2, sink_count=2) is prepared
    rep = c.replicate_over_slots(prepared, 3, source_count=2, sink_count=2)
    t = rep.topology
    assert t.row_count == 9
    assert t.source_index.tolist() == [0, 1, 0, 2, 3, 2, 4, 5, 4]
    assert t.sink_index.tolist() == [0, 0, 1, 2, 2, 3, 4, 4, 5]
    assert t.source_id.tolist() == [100, 101, 100] * 3
    assert t.primitive_sequence.reshape(-1).tolist() == [3, -1, 5] * 3
    assert [(b.component, b.rows.tolist()) for b in rep.buckets] == [("los", [1, 4, 7]),
                                                                     ("reflection", [0, 2, 3, 5, 6, 8])]
    assert rep.execution_order.tolist() == [1, 4, 7, 0, 2, 3, 5, 6, 8]
    assert rep.prepare_d2h_copies == prepared.prepare_d2h_copies
    with pytest.raises(ValueError):
        c.replicate_over_slots(prepared, 0, source_count=2, sink_count=2)
    with pytest.raises(ValueError):
        c.replicate_over_slots(prepared, 2, source_count=0, sink_count=2)
    with pytest.raises(TypeError):
        c.replicate_over_slots(topo, 2, source_count=2, sink_count=2)


def test_time_varying_request_checks():
    topo = c.prepare_fixed_topology(_frozen([0], [0], [[-1]]))
    kw = dict(sources=None, sinks=None, reference_frequency_hz=1e9, topology=topo, response="scalar_transport",
              ad_mode="none")
    with pytest.raises(TypeError, match="float64"):
        c.TimeVaryingRequest(**{**kw, "times_s": torch.zeros(2)})
    with pytest.raises(ValueError):
        c.TimeVaryingRequest(**{**kw, "times_s": torch.zeros(0, dtype=torch.float64)})
    with pytest.raises(TypeError, match="PreparedFixedTopology"):
        c.TimeVaryingRequest(**{**kw, "topology": topo.topology, "times_s": torch.zeros(2, dtype=torch.float64)})
    assert c.TimeVaryingRequest(**{**kw, "times_s": torch.zeros(4, dtype=torch.float64)}).slot_count == 4
