"""Fixed-topology replay on the GPU (reference ``propagation/consumer.py``
``prepare_fixed_topology`` / ``reevaluate`` / ``evaluate_time_varying``;
tests after the reference's ``tests/propagation/test_fixed_topology*.py``).

Checked:

* a replay at the discovery endpoints reproduces the discovered rows bit for
  bit (coefficient, complex3 field, length, delay, direction, interaction
  table, pair segmentation), every row valid;
* at moved sinks the replay is subtractive and exact against a fresh
  discovery (which the parity tests pin to the oracle): every row it
  publishes as valid is a row discovery finds at the new endpoints, with the
  same numbers, every invalid row is one discovery no longer finds, and a row
  whose segment is now blocked is published as exact zeros;
* at a moved grid, the replayed rows against the FP64 oracle's discovery
  there (0.01 dB, 1e-3 rad);
* wideband columns equal one replay per absolute frequency, bit for bit, and a
  zero offset reproduces the reference column;
* slot batching and the time-varying route equal one replay per slot;
* the polarimetric response equals the native LoS Jones owner on LoS rows
  and the scalar response with the frame vectors as polarizations on
  reflection rows (to a few float32 ulps: separate code paths);
* the contract bitmask (index bounds, stable ids, slot blocks), stale worlds
  (refitted geometry, changed materials) and the refusals before native work.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from tests import scenes
from witwin_channel_b200.compiler import compile_scene
from witwin_channel_b200.propagation import consumer as c
from witwin_channel_b200.scene import PhysicalMaterial, Scene

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda", 0)
COMPS = {"los", "reflection"}


def _batch(positions, polarizations, ids, powers=None, basis=None) -> c.EndpointBatch:
    f32 = lambda x: torch.as_tensor(x, dtype=torch.float32).reshape(-1, 3).to(DEV).contiguous()
    return c.EndpointBatch(
        stable_ids=torch.as_tensor(ids, dtype=torch.int64).to(DEV).contiguous(),
        positions_m=f32(positions), polarizations=f32(polarizations),
        polarization_basis=None if basis is None else torch.as_tensor(basis, dtype=torch.float32).to(DEV).contiguous(),
        powers_w=None if powers is None else torch.as_tensor(powers, dtype=torch.float32).to(DEV).contiguous(),
    )


def _city_batches(scene, shift=(0.0, 0.0, 0.0)):
    txs = scene.transmitters
    sources = _batch(torch.stack([t.position.detach().float().reshape(3) for t in txs]),
                     torch.stack([t.polarization.detach().float().reshape(3) for t in txs]),
                     [100 + i for i in range(len(txs))], [float(t.power_w) for t in txs])
    grid = scene.receivers[0]
    pts = grid.points().float() + torch.tensor(shift, dtype=torch.float32)
    sinks = _batch(pts, grid.polarization.detach().float().reshape(1, 3).expand(pts.shape[0], 3),
                   [1000 + i for i in range(pts.shape[0])])
    return sources, sinks


def _discover(compiled, sources, sinks, freq, comps=COMPS, depth=2, response="scalar_transport"):
    return c.evaluate(compiled, c.PropagationRequest(
        sources=sources, sinks=sinks, reference_frequency_hz=freq, components=frozenset(comps), max_depth=depth,
        response=response, topology_mode="discover", ad_mode="none"))


def _replay(compiled, sources, sinks, freq, topology, response="scalar_transport", **kw):
    return c.reevaluate(compiled, c.FixedTopologyRequest(
        sources=sources, sinks=sinks, reference_frequency_hz=freq, topology=topology, response=response,
        ad_mode=kw.pop("ad_mode", "none"), **kw))


def _city(depth=2):
    scene, freq = scenes.small_city()
    compiled = compile_scene(scene, DEV)
    sources, sinks = _city_batches(scene)
    found = _discover(compiled, sources, sinks, freq, depth=depth)
    return scene, freq, compiled, sources, sinks, found


def test_replay_at_discovery_endpoints_is_bit_identical():
    scene, freq, compiled, sources, sinks, found = _city(depth=2)
    prepared = c.prepare_fixed_topology(found.paths.topology)
    assert {b.component for b in prepared.buckets} == {"los", "reflection"}
    out = _replay(compiled, sources, sinks, freq, prepared)
    p, q = out.paths, found.paths
    assert out.row_valid is not None and bool(out.row_valid.all())
    assert p.path_count == q.path_count > 0 and p.pair_count == q.pair_count
    assert torch.equal(p.pair_index, q.pair_index) and torch.equal(p.pair_offsets, q.pair_offsets)
    assert torch.equal(p.transport.coefficient, q.transport.coefficient)
    for name in ("path_length_m", "delay_s", "field_direction", "interaction_positions_m", "interaction_normals"):
        assert torch.equal(getattr(p.geometry, name), getattr(q.geometry, name)), name
    assert p.topology is found.paths.topology
    d = out.diagnostics
    assert (d.validation_d2h_copies, d.validation_d2h_bytes, d.validation_sync_count) == (1, 8, 1)
    assert d.discovery_launch_count == 2 and d.candidate_count == 0 and d.frequency_column_count == 1
    # complex3 response against the discovered complex3 rows
    found3 = _discover(compiled, sources, sinks, freq, depth=2, response="complex3_transport")
    out3 = _replay(compiled, sources, sinks, freq, prepared, response="complex3_transport")
    assert torch.equal(out3.paths.transport.field, found3.paths.transport.field)
    assert torch.equal(out3.paths.transport.direction, found3.paths.transport.direction)


def _row_keys(paths, face_group: np.ndarray) -> list[tuple]:
    t = paths.topology
    seq = t.primitive_sequence.cpu().numpy()
    groups = np.where(seq >= 0, face_group[np.clip(seq, 0, None)], -1)
    return [(int(pi), int(ci), int(di), tuple(int(x) for x in g))
            for pi, ci, di, g in zip(paths.pair_index.tolist(), t.component_id.tolist(), t.depth.tolist(), groups)]


@pytest.mark.parametrize("shift", [(0.7, -0.3, 0.0), (3.1, 2.4, 0.5)])
def test_moved_sinks_replay_is_an_exact_subset_of_rediscovery(shift):
    scene, freq, compiled, sources, sinks, found = _city(depth=2)
    prepared = c.prepare_fixed_topology(found.paths.topology)
    moved_sources, moved_sinks = _city_batches(scene, shift)
    out = _replay(compiled, moved_sources, moved_sinks, freq, prepared)
    fresh = _discover(compiled, moved_sources, moved_sinks, freq, depth=2)
    face_group = compiled.native.groups()[0].cpu().numpy()
    fresh_rows = {k: i for i, k in enumerate(_row_keys(fresh.paths, face_group))}
    valid = out.row_valid.cpu().numpy()
    coef = out.paths.transport.coefficient.cpu()
    fresh_coef = fresh.paths.transport.coefficient.cpu()
    length = out.paths.geometry.path_length_m.cpu()
    fresh_length = fresh.paths.geometry.path_length_m.cpu()
    frozen_keys = _row_keys(out.paths, face_group)
    assert valid.sum() > 0
    for i, key in enumerate(frozen_keys):
        j = fresh_rows.get(key)
        if valid[i]:
            assert j is not None, key
            torch.testing.assert_close(coef[i], fresh_coef[j], rtol=1e-6, atol=1e-12)
            torch.testing.assert_close(length[i], fresh_length[j], rtol=1e-7, atol=0.0)
        else:
            assert j is None, key
            assert coef[i] == 0 and length[i] == 0
    # every rediscovered row of a frozen (pair, component, groups) is replayed as valid
    frozen = {k: i for i, k in enumerate(frozen_keys)}
    for key in fresh_rows:
        if key in frozen:
            assert valid[frozen[key]], key


def test_blocked_line_of_sight_publishes_exact_zeros():
    freq = 3.0e9
    scene = scenes.two_wall_scene()
    compiled = compile_scene(scene, DEV)
    pol = [[0.0, 0.0, 1.0]]
    sources = _batch([[0.0, 0.0, 1.0]], pol, [7], [2.0])
    sinks = _batch([[0.0, 1.0, 1.0]], pol, [9])
    found = _discover(compiled, sources, sinks, freq, depth=2)
    t = found.paths.topology
    assert t.component_id.tolist().count(0) == 1
    prepared = c.prepare_fixed_topology(t)
    behind = _batch([[4.0, 1.0, 1.0]], pol, [9])  # behind the wall at x = 2
    out = _replay(compiled, sources, behind, freq, prepared)
    los = t.component_id == 0
    assert not bool(out.row_valid[los].any())
    assert bool((out.paths.transport.coefficient[los] == 0).all())
    assert bool((out.paths.geometry.path_length_m[los] == 0).all())
    assert bool((out.paths.geometry.field_direction[los] == 0).all())
    # the same topology replayed back in front of the wall is whole again
    again = _replay(compiled, sources, sinks, freq, prepared)
    assert bool(again.row_valid.all())
    assert torch.equal(again.paths.transport.coefficient, found.paths.transport.coefficient)


def test_wideband_columns_equal_one_replay_per_frequency():
    scene, freq, compiled, sources, sinks, found = _city(depth=2)
    prepared = c.prepare_fixed_topology(found.paths.topology)
    offsets = (0.0, 2.5e8, -1.0e9)
    for response, attr, wide in (("scalar_transport", "coefficient", "coefficient_offsets"),
                                 ("complex3_transport", "field", "field_offsets")):
        out = _replay(compiled, sources, sinks, freq, prepared, response=response, frequency_offsets_hz=offsets)
        payload = getattr(out.paths.transport, wide)
        assert payload.shape[1] == 3 and out.paths.transport.frequency_offsets_hz == offsets
        assert out.diagnostics.frequency_column_count == 3
        reference = getattr(out.paths.transport, attr)
        assert torch.equal(payload[:, 0], reference)
        for j, df in enumerate(offsets):
            single = _replay(compiled, sources, sinks, freq + df, prepared, response=response)
            assert torch.equal(payload[:, j], getattr(single.paths.transport, attr)), (response, df)
        plain = _replay(compiled, sources, sinks, freq, prepared, response=response)
        assert torch.equal(reference, getattr(plain.paths.transport, attr))


def _stack(batches: list[c.EndpointBatch]) -> c.EndpointBatch:
    cat = lambda name: None if getattr(batches[0], name) is None else torch.cat([getattr(b, name) for b in batches])
    return c.EndpointBatch(stable_ids=cat("stable_ids"), positions_m=cat("positions_m"),
                           polarizations=cat("polarizations"), polarization_basis=cat("polarization_basis"),
                           powers_w=cat("powers_w"))


def test_slots_and_time_varying_equal_one_replay_per_slot():
    scene, freq, compiled, sources, sinks, found = _city(depth=2)
    prepared = c.prepare_fixed_topology(found.paths.topology)
    shifts = [(0.0, 0.0, 0.0), (0.5, 0.2, 0.0), (1.5, -0.8, 0.3)]
    per_slot = [_city_batches(scene, s) for s in shifts]
    T = len(shifts)
    S, R = sources.count, sinks.count
    rep = c.replicate_over_slots(prepared, T, source_count=S, sink_count=R)
    stacked_sources = _stack([b[0] for b in per_slot])
    stacked_sinks = _stack([b[1] for b in per_slot])
    out = _replay(compiled, stacked_sources, stacked_sinks, freq, rep, slot_count=T)
    K = prepared.row_count
    assert out.paths.path_count == T * K and out.paths.pair_count == T * S * R
    assert out.diagnostics.validation_d2h_copies == 1
    for t, (src, snk) in enumerate(per_slot):
        single = _replay(compiled, src, snk, freq, prepared)
        rows = slice(t * K, (t + 1) * K)
        assert torch.equal(out.paths.transport.coefficient[rows], single.paths.transport.coefficient)
        assert torch.equal(out.row_valid[rows], single.row_valid)
        assert torch.equal(out.paths.geometry.delay_s[rows], single.paths.geometry.delay_s)
        assert torch.equal(out.paths.pair_index[rows], single.paths.pair_index + t * S * R)
        seg = out.paths.pair_offsets[t * S * R:(t + 1) * S * R + 1] - t * K
        assert torch.equal(seg, single.paths.pair_offsets)
    times = torch.tensor([0.0, 1.0e-3, 2.0e-3], dtype=torch.float64)
    tv = c.evaluate_time_varying(compiled, c.TimeVaryingRequest(
        sources=stacked_sources, sinks=stacked_sinks, reference_frequency_hz=freq, topology=prepared, times_s=times,
        response="scalar_transport", ad_mode="none"))
    assert (tv.slot_count, tv.row_count, tv.pair_count) == (T, K, S * R)
    assert torch.equal(tv.transport.coefficient, out.paths.transport.coefficient.view(T, K))
    assert torch.equal(tv.delay_s, out.paths.geometry.delay_s.view(T, K))
    assert torch.equal(tv.row_valid, out.row_valid.view(T, K))
    assert torch.equal(tv.pair_offsets, out.paths.pair_offsets[:S * R + 1])
    assert tv.transport.field is None and tv.transport.matrix is None


def _basis(n, seed):
    g = torch.Generator().manual_seed(seed)
    return torch.randn((n, 2, 3), generator=g)


def test_polarimetric_replay_matches_los_jones_and_scalar_frames():
    freq = 3.5e9
    # LoS rows: the native LoS Jones owner
    scene = Scene(structures=[], endpoints=[])
    compiled = compile_scene(scene, DEV)
    pol = [[0.0, 0.0, 1.0]]
    src = _batch([[0.0, 0.0, 0.0], [1.0, 2.0, 0.5]], pol * 2, [1, 2], [1.0, 2.0], basis=_basis(2, 1))
    snk = _batch([[3.0, 4.0, 0.0], [-2.0, 6.0, 1.0], [5.0, -1.0, 2.0]], pol * 3, [5, 6, 7], basis=_basis(3, 2))
    found = _discover(compiled, src, snk, freq, comps={"los"}, depth=0)
    prepared = c.prepare_fixed_topology(found.paths.topology)
    out = _replay(compiled, src, snk, freq, prepared, response="polarimetric_transport")
    ref = c.consumer_los_jones(pair_index=found.paths.pair_index, source_positions=src.positions_m,
                               sink_positions=snk.positions_m, source_reference_basis=src.polarization_basis,
                               sink_reference_basis=snk.polarization_basis, frequency_hz=freq)
    # two kernels: the compiler may fuse multiply-adds differently, so the
    # comparison allows a few float32 ulps
    torch.testing.assert_close(out.paths.transport.matrix, ref.matrix, rtol=2e-6, atol=1e-12)
    torch.testing.assert_close(out.paths.transport.source_basis, ref.source_basis, rtol=2e-6, atol=1e-7)
    torch.testing.assert_close(out.paths.transport.sink_basis, ref.sink_basis, rtol=2e-6, atol=1e-7)
    # reflection rows: entry (a, b) is the scalar response with source frame
    # vector b as the source polarization and sink frame vector a as the sink's
    scene = scenes.two_wall_scene()
    compiled = compile_scene(scene, DEV)
    src = _batch([[0.0, 0.0, 1.0]], pol, [7], [1.0], basis=_basis(1, 3))
    snk = _batch([[0.0, 1.0, 1.0]], pol, [9], basis=_basis(1, 4))
    found = _discover(compiled, src, snk, freq, depth=2)
    prepared = c.prepare_fixed_topology(found.paths.topology)
    jones = _replay(compiled, src, snk, freq, prepared, response="polarimetric_transport")
    tr = jones.paths.transport
    assert bool(jones.row_valid.all()) and found.paths.path_count >= 3
    for i in range(found.paths.path_count):
        for a in range(2):
            for b in range(2):
                s1 = _batch(src.positions_m, tr.source_basis[i, b].reshape(1, 3), [7], [1.0])
                k1 = _batch(snk.positions_m, tr.sink_basis[i, a].reshape(1, 3), [9])
                scalar = _replay(compiled, s1, k1, freq, prepared)
                torch.testing.assert_close(scalar.paths.transport.coefficient[i], tr.matrix[i, a, b], rtol=2e-6,
                                           atol=1e-12, msg=f"row {i} entry {a}{b}")


def test_raw_line_of_sight_route_and_empty_topology():
    freq = 2.4e9
    scene = Scene(structures=[], endpoints=[])
    compiled = compile_scene(scene, DEV)
    pol = [[0.0, 0.0, 1.0]]
    src = _batch([[0.0, 0.0, 0.0], [1.0, 2.0, 0.5]], pol * 2, [1, 2], [1.0, 2.0])
    snk = _batch([[3.0, 4.0, 0.0], [-2.0, 6.0, 1.0]], pol * 2, [5, 6])
    found = _discover(compiled, src, snk, freq, comps={"los"}, depth=0)
    out = _replay(compiled, src, snk, freq, found.paths.topology)
    assert out.row_valid is None
    assert torch.equal(out.paths.transport.coefficient, found.paths.transport.coefficient)
    moved = _batch([[3.5, 4.0, 0.0], [-2.0, 6.5, 1.0]], pol * 2, [5, 6])
    again = _replay(compiled, src, moved, freq, found.paths.topology)
    fresh = _discover(compiled, src, moved, freq, comps={"los"}, depth=0)
    assert torch.equal(again.paths.transport.coefficient, fresh.paths.transport.coefficient)
    assert torch.equal(again.paths.geometry.delay_s, fresh.paths.geometry.delay_s)
    with pytest.raises(NotImplementedError, match="PreparedFixedTopology"):
        _replay(compiled, src, snk, freq, found.paths.topology, slot_count=2)
    # an empty frozen topology: no rows, an all-zero segmentation
    t = found.paths.topology
    empty = c.PropagationTopology(**{name: getattr(t, name)[:0] for name in (
        "source_index", "sink_index", "source_id", "sink_id", "depth", "component_id", "primitive_id", "edge_id",
        "material_id", "primitive_sequence", "material_sequence", "interaction_type")})
    none = _replay(compiled, src, snk, freq, c.prepare_fixed_topology(empty))
    assert none.paths.path_count == 0 and none.paths.pair_offsets.tolist() == [0] * 5
    assert none.diagnostics.validation_d2h_copies == 0


def test_contract_bitmask_and_refusals():
    scene, freq, compiled, sources, sinks, found = _city(depth=2)
    prepared = c.prepare_fixed_topology(found.paths.topology)
    renamed = c.EndpointBatch(stable_ids=sinks.stable_ids + 1, positions_m=sinks.positions_m,
                              polarizations=sinks.polarizations)
    with pytest.raises(ValueError, match="bitmask 16"):
        _replay(compiled, sources, renamed, freq, prepared)
    fewer = c.EndpointBatch(stable_ids=sinks.stable_ids[:5].contiguous(), positions_m=sinks.positions_m[:5].contiguous(),
                            polarizations=sinks.polarizations[:5].contiguous())
    with pytest.raises(ValueError, match="bitmask 1"):
        _replay(compiled, sources, fewer, freq, prepared)
    rep = c.replicate_over_slots(prepared, 2, source_count=sources.count, sink_count=sinks.count)
    t = rep.topology
    sink_index = t.sink_index.clone()
    sink_index[0] += sinks.count  # row 0 of slot 0 now pairs with a slot-1 sink
    broken = c.PreparedFixedTopology(
        topology=c.PropagationTopology(**{**{n: getattr(t, n) for n in (
            "source_index", "source_id", "sink_id", "depth", "component_id", "primitive_id", "edge_id",
            "material_id", "primitive_sequence", "material_sequence", "interaction_type")},
            "sink_index": sink_index}),
        buckets=rep.buckets, prepare_d2h_copies=0, prepare_d2h_bytes=0, prepare_synchronizations=0,
        execution_order=rep.execution_order)
    # the row's pair index also jumps past its successors': slot block (32) and pair order (2)
    with pytest.raises(ValueError, match="bitmask 34"):
        _replay(compiled, _stack([sources, sources]), _stack([sinks, sinks]), freq, broken, slot_count=2)
    with pytest.raises(NotImplementedError):
        _replay(compiled, sources, sinks, freq, prepared, response="polarimetric_transport", ad_mode="vjp")
    with pytest.raises(ValueError, match="polarization_basis"):
        _replay(compiled, sources, sinks, freq, prepared, response="polarimetric_transport")
    with pytest.raises(NotImplementedError):
        _replay(compiled, sources, sinks, freq, prepared, response="polarimetric_transport",
                frequency_offsets_hz=(1.0e6,))
    with pytest.raises(ValueError, match="multiple of slot_count"):
        _replay(compiled, sources, sinks, freq, rep, slot_count=2)


def test_stale_world_is_refused_and_fixed_winner_replay_follows_refit():
    scene, freq, compiled, sources, sinks, found = _city(depth=2)
    prepared = c.prepare_fixed_topology(found.paths.topology)
    assert c.rediscovery_required(compiled, prepared) is None
    assert c.rediscovery_required(compiled, prepared, revalidate_source=True) is None
    st = scene.structures[1]
    st.geometry.vertices = st.vertices.detach() + torch.tensor([0.05, -0.03, 0.0])
    assert c.rediscovery_required(compiled, prepared, revalidate_source=True) == "geometry_version"
    moved = compile_scene(scene, DEV)
    assert moved is compiled  # refitted in place
    assert c.rediscovery_required(compiled, prepared) == "geometry_version"
    with pytest.raises(ValueError, match="geometry_version"):
        _replay(compiled, sources, sinks, freq, prepared)
    out = _replay(compiled, sources, sinks, freq, prepared, world_motion="fixed_winner_replay")
    fresh = _discover(compiled, sources, sinks, freq, depth=2)
    face_group = compiled.native.groups()[0].cpu().numpy()
    fresh_rows = {k: i for i, k in enumerate(_row_keys(fresh.paths, face_group))}
    valid = out.row_valid.cpu().numpy()
    for i, key in enumerate(_row_keys(out.paths, face_group)):
        assert (fresh_rows.get(key) is not None) == bool(valid[i]), key
    fresh_prepared = c.prepare_fixed_topology(fresh.paths.topology)
    assert c.rediscovery_required(compiled, fresh_prepared, revalidate_source=True) is None
    scene.structures[0].material = PhysicalMaterial(eps_r=7.5, sigma_e=0.02)
    assert c.rediscovery_required(compiled, fresh_prepared) is None  # the compiled scene has not seen it
    assert c.rediscovery_required(compiled, fresh_prepared, revalidate_source=True) == "assignment_version"
    recompiled = compile_scene(scene, DEV)
    assert recompiled is not compiled
    assert c.rediscovery_required(recompiled, prepared) == "material_version"
    with pytest.raises(ValueError, match="material_version"):
        _replay(recompiled, sources, sinks, freq, prepared, world_motion="fixed_winner_replay")


def test_moved_sink_replay_matches_the_oracle():
    """Replay at moved sinks against the FP64 oracle's own discovery at the
    moved grid: every valid replayed row is an oracle row (same pair,
    component and coplanar groups) with its gain within 0.01 dB and phase
    within 1e-3 rad; every oracle row of a frozen key is replayed as valid."""
    from oracle import solve as osolve
    from witwin_channel_b200.scene import make_receiver_grid

    scene, freq = scenes.small_city()
    compiled = compile_scene(scene, DEV)
    sources, sinks = _city_batches(scene)
    found = _discover(compiled, sources, sinks, freq, depth=2)
    prepared = c.prepare_fixed_topology(found.paths.topology)
    shift = (1.3, -0.9, 0.4)
    g = scene.receivers[0]
    moved_grid = make_receiver_grid(origin=(g.origin + torch.tensor(shift)).tolist(), x_axis=g.x_axis.tolist(),
                                    y_axis=g.y_axis.tolist(), shape=g.shape, spacing=g.spacing)
    # the moved sinks are exactly the oracle's moved grid points
    pts = moved_grid.points().float()
    moved_sinks = _batch(pts, g.polarization.detach().float().reshape(1, 3).expand(pts.shape[0], 3),
                         [1000 + i for i in range(pts.shape[0])])
    out = _replay(compiled, sources, moved_sinks, freq, prepared)
    moved_scene = Scene(structures=scene.structures, endpoints=[scene.transmitters[0], moved_grid])
    arr = osolve.scene_arrays(moved_scene, freq)
    ref = osolve.solve(arr, frequency=freq, components={"los", "reflection"}, max_depth=2, coherent=True)["rows"]
    face_group = compiled.native.groups()[0].cpu().numpy()
    S = sources.count

    def key(tx, rx, cid, depth, seq):
        groups = tuple(int(face_group[f]) if f >= 0 else -1 for f in seq)
        return (int(rx) * S + int(tx), int(cid), int(depth), groups)

    W = int(prepared.topology.primitive_sequence.shape[1])
    oracle_rows = {key(ref["tx_id"][i], ref["rx_id"][i], ref["component_id"][i], ref["depth"][i],
                       [int(x) for x in ref["primitive_sequence"][i][:W]]): complex(ref["path_field"][i])
                   for i in range(len(ref["tx_id"]))}
    t = out.paths.topology
    valid = out.row_valid.cpu().numpy()
    coef = out.paths.transport.coefficient.cpu().numpy().astype(np.complex128)
    strongest = max(abs(v) for v in oracle_rows.values())
    keys = [key(*row) for row in zip(t.source_index.tolist(), t.sink_index.tolist(), t.component_id.tolist(),
                                     t.depth.tolist(), t.primitive_sequence.tolist())]
    frozen = {k: i for i, k in enumerate(keys)}
    checked = 0
    for i, k in enumerate(keys):
        if not valid[i]:
            assert k not in oracle_rows, k
            continue
        assert k in oracle_rows, k
        want = oracle_rows[k]
        if abs(want) > 1e-3 * strongest:
            assert abs(20.0 * np.log10(abs(coef[i]) / abs(want))) <= 0.01, k
            assert abs(np.angle(coef[i] / want)) <= 1e-3, k
            checked += 1
    assert checked > 20
    for k in oracle_rows:
        if k in frozen:
            assert valid[frozen[k]], k
