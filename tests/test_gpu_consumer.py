"""Propagation consumer on the GPU: LoS rows in closed form, the pair-major
rows of a city against the oracle and against the deterministic path table
(same engine, bit for bit), the global path limit, empty batches and the
refusals made before any native work."""

from __future__ import annotations

import math

import numpy as np
import pytest
import torch

from oracle import solve as osolve
from tests import scenes
from witwin_channel_b200 import Config as DetConfig
from witwin_channel_b200 import solve as det_solve
from witwin_channel_b200.compiler import compile_scene
from witwin_channel_b200.propagation import consumer as c
from witwin_channel_b200.scene import Scene, make_transmitter

pytestmark = pytest.mark.gpu
C0 = 299_792_458.0
DB_TOL = 0.01
PHASE_TOL = 1.0e-3


def _batch(positions, polarizations, ids, powers=None) -> c.EndpointBatch:
    dev = torch.device("cuda", 0)
    f32 = lambda x: torch.as_tensor(x, dtype=torch.float32).reshape(-1, 3).to(dev).contiguous()
    return c.EndpointBatch(
        stable_ids=torch.as_tensor(ids, dtype=torch.int64).to(dev),
        positions_m=f32(positions), polarizations=f32(polarizations),
        powers_w=None if powers is None else torch.as_tensor(powers, dtype=torch.float32).to(dev),
    )


def _request(sources, sinks, freq, comps, depth, response="scalar_transport", **kw) -> c.PropagationRequest:
    return c.PropagationRequest(sources=sources, sinks=sinks, reference_frequency_hz=freq,
                                components=frozenset(comps), max_depth=depth, response=response,
                                topology_mode="discover", ad_mode=kw.pop("ad_mode", "none"), **kw)


def _scene_batches(scene):
    txs = scene.transmitters
    sources = _batch(torch.stack([t.position.detach().float().reshape(3) for t in txs]),
                     torch.stack([t.polarization.detach().float().reshape(3) for t in txs]),
                     [100 + i for i in range(len(txs))], [float(t.power_w) for t in txs])
    grid = scene.receivers[0]
    pts = grid.points()
    sinks = _batch(pts, grid.polarization.detach().float().reshape(1, 3).expand(pts.shape[0], 3),
                   [1000 + i for i in range(pts.shape[0])])
    return sources, sinks


def test_los_rows_closed_form_pair_order_and_complex3():
    f = 3.0e9
    scene = Scene(structures=[], endpoints=[])
    sources = _batch([[0.0, 0.0, 0.0], [0.0, 2.0, 0.0]], [[0.0, 0.0, 1.0]] * 2, [11, 12], [2.0, 0.5])
    sinks = _batch([[3.0, 4.0, 0.0], [6.0, 8.0, 0.0], [-5.0, 1.0, 0.0]], [[0.0, 0.0, 1.0]] * 3, [21, 22, 23])
    compiled = compile_scene(scene, torch.device("cuda", 0))
    out = c.evaluate(compiled, _request(sources, sinks, f, {"los"}, 0))
    p = out.paths
    assert p.pair_count == 6 and p.path_count == 6
    assert p.pair_index.tolist() == list(range(6))
    assert p.pair_offsets.tolist() == list(range(7))
    t = p.topology
    assert t.source_index.tolist() == [0, 1, 0, 1, 0, 1]
    assert t.sink_index.tolist() == [0, 0, 1, 1, 2, 2]
    assert t.source_id.tolist() == [11, 12, 11, 12, 11, 12]
    assert t.sink_id.tolist() == [21, 21, 22, 22, 23, 23]
    assert t.component_id.tolist() == [0] * 6 and t.depth.tolist() == [0] * 6
    assert tuple(t.primitive_sequence.shape) == (6, 0)
    src = sources.positions_m.double().cpu()
    dst = sinks.positions_m.double().cpu()
    coef = p.transport.coefficient.cpu()
    for k in range(6):
        d = float(torch.linalg.vector_norm(dst[k // 2] - src[k % 2]))
        assert abs(float(p.geometry.path_length_m[k]) - d) <= 1e-5 * d
        assert abs(float(p.geometry.delay_s[k]) * C0 - d) <= 1e-5 * d
        # excited amplitude sqrt(P) * lambda / (4 pi d), vertical polarisations, horizontal links
        want = math.sqrt([2.0, 0.5][k % 2]) * C0 / f / (4 * math.pi * d)
        assert abs(abs(complex(coef[k])) - want) <= 1e-5 * want
    assert out.diagnostics.candidate_count == 6
    assert out.diagnostics.discovery_launch_count > 0
    # complex3: the excited world field projected on the sink polarisation is the scalar coefficient
    out3 = c.evaluate(compiled, _request(sources, sinks, f, {"los"}, 0, response="complex3_transport"))
    field = out3.paths.transport.field.cpu()
    proj = (field * sinks.polarizations.cpu()[out3.paths.topology.sink_index.cpu().long()].to(torch.complex64)).sum(-1)
    np.testing.assert_allclose(proj.numpy(), coef.numpy(), rtol=1e-5, atol=1e-9 * float(coef.abs().max()))
    assert torch.equal(out3.paths.transport.direction, out.paths.geometry.field_direction)


def _two_tx_city():
    scene, freq = scenes.small_city()
    layout = scenes.city_layout(4, 7, lot_size=30.0, footprint=(8.0, 20.0), height=(6.0, 25.0))
    second = make_transmitter(scenes.street_point(layout, np.random.default_rng(2024), 8.0), power_w=0.25)
    return Scene(structures=scene.structures, endpoints=[scene.transmitters[0], second, scene.receivers[0]]), freq


def test_city_rows_match_oracle_in_pair_order():
    scene, freq = _two_tx_city()
    comps = {"los", "reflection", "diffraction", "transmission"}
    sources, sinks = _scene_batches(scene)
    out = c.evaluate(compile_scene(scene, torch.device("cuda", 0)), _request(sources, sinks, freq, comps, 2))
    p = out.paths
    S = sources.count
    arr = osolve.scene_arrays(scene, freq)
    ref = osolve.solve(arr, frequency=freq, components=comps, max_depth=2, coherent=True)["rows"]
    pair = np.asarray(ref["rx_id"], dtype=np.int64) * S + np.asarray(ref["tx_id"], dtype=np.int64)
    order = np.argsort(pair, kind="stable")
    assert p.path_count == len(order) > 0
    assert p.pair_index.cpu().numpy().tolist() == pair[order].tolist()
    offsets = p.pair_offsets.cpu().numpy()
    assert offsets[0] == 0 and offsets[-1] == p.path_count and np.all(np.diff(offsets) >= 0)
    assert np.array_equal(np.diff(offsets), np.bincount(pair, minlength=p.pair_count))
    t = p.topology
    W = t.primitive_sequence.shape[1]
    got = list(zip(t.source_index.tolist(), t.sink_index.tolist(), t.component_id.tolist(), t.depth.tolist(),
                   map(tuple, t.primitive_sequence.tolist())))
    want = [(int(ref["tx_id"][i]), int(ref["rx_id"][i]), int(ref["component_id"][i]), int(ref["depth"][i]),
             tuple(int(x) for x in ref["primitive_sequence"][i][:W])) for i in order]
    assert got == want
    assert t.source_id.tolist() == [100 + s for s in t.source_index.tolist()]
    assert t.sink_id.tolist() == [1000 + r for r in t.sink_index.tolist()]
    np.testing.assert_allclose(p.geometry.path_length_m.cpu().numpy(), np.asarray(ref["path_length_m"])[order],
                               rtol=1e-5, atol=1e-5)
    got_f = p.transport.coefficient.cpu().numpy().astype(np.complex128)
    want_f = np.asarray(ref["path_field"])[order]
    strong = np.abs(want_f) > 1e-3 * np.abs(want_f).max()
    db = np.abs(20.0 * np.log10(np.abs(got_f[strong]) / np.abs(want_f[strong])))
    assert np.all(db <= DB_TOL), db.max()
    assert np.all(np.abs(np.angle(got_f[strong] / want_f[strong])) <= PHASE_TOL)
    assert set(t.component_id.unique().tolist()) == {0, 1, 2, 5}


def test_city_rows_equal_the_deterministic_table():
    """One transmitter: the pair-major order is the table's canonical order,
    so the consumer rows and the exported table agree bit for bit."""
    scene, freq = scenes.small_city()
    comps = {"los", "reflection", "diffraction", "transmission"}
    sources, sinks = _scene_batches(scene)
    p = c.evaluate(compile_scene(scene, torch.device("cuda", 0)), _request(sources, sinks, freq, comps, 2)).paths
    table = det_solve(scene, DetConfig(max_depth=2, components=comps, export_paths=True),
                      reference_frequency_hz=freq).paths
    t = p.topology
    assert torch.equal(t.sink_index.cpu(), table.rx_id.cpu().to(torch.int32))
    assert torch.equal(t.component_id.cpu(), table.component_id.cpu().to(torch.int32))
    assert torch.equal(t.primitive_sequence.cpu(), table.primitive_sequence.cpu().to(torch.int32))
    assert torch.equal(t.material_sequence.cpu(), table.material_sequence.cpu().to(torch.int32))
    assert torch.equal(t.primitive_id.cpu(), table.primitive_id.cpu().to(torch.int32))
    assert torch.equal(t.edge_id.cpu(), table.edge_id.cpu().to(torch.int32))
    assert torch.equal(p.geometry.path_length_m.cpu(), table.path_length_m.cpu())
    assert torch.equal(p.geometry.interaction_positions_m.cpu(), table.interaction_positions.cpu())
    pf = torch.complex(table.field_real, table.field_imag).cpu()
    assert torch.equal(p.transport.coefficient.cpu(), pf)


def test_global_path_limit_keeps_the_tables_selection():
    scene, freq = scenes.small_city()
    comps = {"los", "reflection", "diffraction"}
    sources, sinks = _scene_batches(scene)
    compiled = compile_scene(scene, torch.device("cuda", 0))
    full = c.evaluate(compiled, _request(sources, sinks, freq, comps, 2)).paths
    limit = max(1, full.path_count // 3)
    part = c.evaluate(compiled, _request(sources, sinks, freq, comps, 2, max_paths=limit)).paths
    assert part.path_count == limit
    table = det_solve(scene, DetConfig(max_depth=2, components=comps, export_paths=True, max_paths=limit,
                                       max_paths_scope="global"), reference_frequency_hz=freq).paths
    key = lambda r, comp, seq: sorted(zip(r.tolist(), comp.tolist(), map(tuple, seq.tolist())))
    assert key(part.topology.sink_index.cpu(), part.topology.component_id.cpu(),
               part.topology.primitive_sequence.cpu()) == key(table.rx_id.cpu(), table.component_id.cpu(),
                                                               table.primitive_sequence.cpu())


def test_empty_batches_and_refusals():
    scene, freq = scenes.small_city()
    compiled = compile_scene(scene, torch.device("cuda", 0))
    sources, sinks = _scene_batches(scene)
    none = _batch(torch.zeros((0, 3)), torch.zeros((0, 3)), [])
    out = c.evaluate(compiled, _request(sources, none, freq, {"los", "reflection"}, 1))
    assert out.paths.path_count == 0 and out.paths.pair_count == 0
    assert out.paths.pair_offsets.tolist() == [0]
    assert tuple(out.paths.topology.primitive_sequence.shape) == (0, 1)
    with pytest.raises(ValueError):  # the polarimetric response needs both reference bases
        c.evaluate(compiled, _request(sources, sinks, freq, {"los"}, 0, response="polarimetric_transport"))
    for ad_mode in ("vjp", "jvp"):  # the Jones operator carries no derivative
        with pytest.raises(NotImplementedError):
            c.evaluate(compiled, _request(sources, sinks, freq, {"los"}, 0, response="polarimetric_transport",
                                          ad_mode=ad_mode))
    with pytest.raises(ValueError):
        c.evaluate(compiled, _request(sources, sinks, freq, {"reflection"}, 0))
    with pytest.raises(TypeError):
        c.evaluate(scene, _request(sources, sinks, freq, {"los"}, 0))
    with pytest.raises(ValueError):
        _request(sinks, sinks, freq, {"los"}, 0)  # a source batch needs powers_w


def _free_space_scalar(frequency_hz: float, distance_m: float) -> complex:
    k = 2.0 * math.pi * frequency_hz / C0
    return complex(math.cos(-k * distance_m), math.sin(-k * distance_m)) / (2.0 * k * distance_m)


def test_los_jones_rotated_basis_closed_form():
    """Source frame (x, y), sink frame (y, -x) on a link along +z: the operator
    is [[0, s], [-s, 0]] with s the free-space scalar (the reference's analytic
    case, ``tests/propagation/consumer/test_los_jones.py``)."""
    dev = torch.device("cuda", 0)
    rows = c.consumer_los_jones(
        pair_index=torch.tensor([0], dtype=torch.int64, device=dev),
        source_positions=torch.tensor([[0.0, 0.0, 0.0]], device=dev),
        sink_positions=torch.tensor([[0.0, 0.0, 2.0]], device=dev),
        source_reference_basis=torch.tensor([[[1.0, 0.0, 0.0], [0.0, 1.0, 0.0]]], device=dev),
        sink_reference_basis=torch.tensor([[[0.0, 1.0, 0.0], [-1.0, 0.0, 0.0]]], device=dev),
        frequency_hz=1.0e9)
    s = _free_space_scalar(1.0e9, 2.0)
    want = torch.tensor([[[0.0j, s], [-s, 0.0j]]], dtype=torch.complex64, device=dev)
    torch.testing.assert_close(rows.matrix, want, rtol=2.0e-5, atol=2.0e-7)
    torch.testing.assert_close(rows.source_basis.cpu(), torch.tensor([[[1.0, 0.0, 0.0], [0.0, 1.0, 0.0]]]))
    torch.testing.assert_close(rows.sink_basis.cpu(), torch.tensor([[[0.0, 1.0, 0.0], [-1.0, 0.0, 0.0]]]))
    assert rows.native_launch_count == 1
    empty = c.consumer_los_jones(
        pair_index=torch.empty((0,), dtype=torch.int64, device=dev),
        source_positions=torch.zeros((1, 3), device=dev), sink_positions=torch.ones((1, 3), device=dev),
        source_reference_basis=torch.zeros((1, 2, 3), device=dev), sink_reference_basis=torch.zeros((1, 2, 3), device=dev),
        frequency_hz=1.0e9)
    assert tuple(empty.matrix.shape) == (0, 2, 2) and empty.native_launch_count == 0


def test_los_jones_flags_a_pair_outside_the_batches():
    dev = torch.device("cuda", 0)
    with pytest.raises(IndexError):
        c.consumer_los_jones(
            pair_index=torch.tensor([0, 4], dtype=torch.int64, device=dev),
            source_positions=torch.zeros((2, 3), device=dev), sink_positions=torch.ones((2, 3), device=dev),
            source_reference_basis=torch.tensor([[[1.0, 0, 0], [0, 1.0, 0]]] * 2, device=dev),
            sink_reference_basis=torch.tensor([[[1.0, 0, 0], [0, 1.0, 0]]] * 2, device=dev), frequency_hz=1.0e9)


def _frame_restated(ref: np.ndarray, d: np.ndarray) -> np.ndarray:
    first, second = ref[0], ref[1]
    u = first - d * (first @ d)
    u = u / np.linalg.norm(u)
    v = np.cross(d, u)
    v = v / np.linalg.norm(v)
    return np.stack([u, -v if v @ second < 0 else v])


def test_polarimetric_evaluate_matches_frames_and_scalar_response():
    f = 3.5e9
    dev = torch.device("cuda", 0)
    g = torch.Generator().manual_seed(5)
    src_pos = torch.tensor([[0.0, 0.0, 1.0], [1.0, -2.0, 3.0]])
    snk_pos = torch.tensor([[7.0, 3.0, 1.5], [-4.0, 6.0, 2.0], [2.0, 9.0, -1.0]])
    src_ref = torch.randn((2, 2, 3), generator=g)
    snk_ref = torch.randn((3, 2, 3), generator=g)
    src_pol = torch.randn((2, 3), generator=g)
    snk_pol = torch.randn((3, 3), generator=g)

    def batch(pos, pol, ref, ids, powers=None):
        return c.EndpointBatch(stable_ids=torch.tensor(ids, dtype=torch.int64, device=dev),
                               positions_m=pos.to(dev).contiguous(), polarizations=pol.to(dev).contiguous(),
                               polarization_basis=ref.to(dev).contiguous(),
                               powers_w=None if powers is None else torch.tensor(powers, device=dev))

    sources = batch(src_pos, src_pol, src_ref, [1, 2], [1.0, 4.0])
    sinks = batch(snk_pos, snk_pol, snk_ref, [7, 8, 9])
    compiled = compile_scene(Scene(structures=[], endpoints=[]), dev)
    out = c.evaluate(compiled, _request(sources, sinks, f, {"los"}, 0, response="polarimetric_transport"))
    p = out.paths
    assert p.path_count == 6 and isinstance(p.transport, c.JonesTransport)
    scalar = c.evaluate(compiled, _request(sources, sinks, f, {"los"}, 0)).paths.transport.coefficient.cpu().numpy()
    M = p.transport.matrix.cpu().numpy()
    sb = p.transport.source_basis.cpu().numpy()
    kb = p.transport.sink_basis.cpu().numpy()
    for k in range(6):
        t, r = int(p.topology.source_index[k]), int(p.topology.sink_index[k])
        off = (snk_pos[r] - src_pos[t]).double().numpy()
        dist = float(np.linalg.norm(off))
        d = off / dist
        fs = _frame_restated(src_ref[t].double().numpy(), d)
        fk = _frame_restated(snk_ref[r].double().numpy(), d)
        np.testing.assert_allclose(sb[k], fs, atol=2e-6)
        np.testing.assert_allclose(kb[k], fk, atol=2e-6)
        s = _free_space_scalar(f, dist)
        np.testing.assert_allclose(M[k], s * (fk @ fs.T), rtol=0, atol=2e-5 * abs(s))
        # the operator reproduces the scalar response of the endpoint polarisations
        # (transverse parts in the two frames), times the source amplitude
        a = fs @ src_pol[t].double().numpy()
        b = fk @ snk_pol[r].double().numpy()
        want = math.sqrt([1.0, 4.0][t]) * (b @ M[k].astype(np.complex128) @ a)
        assert abs(scalar[k] - want) <= 1e-4 * abs(s) * math.sqrt([1.0, 4.0][t]) * (
            np.linalg.norm(src_pol[t].numpy()) * np.linalg.norm(snk_pol[r].numpy()))
    with pytest.raises(NotImplementedError):
        c.evaluate(compiled, _request(sources, sinks, f, {"los", "reflection"}, 1, response="polarimetric_transport"))
    no_basis = c.EndpointBatch(stable_ids=sinks.stable_ids, positions_m=sinks.positions_m,
                               polarizations=sinks.polarizations)
    with pytest.raises(ValueError):
        c.evaluate(compiled, _request(sources, no_basis, f, {"los"}, 0, response="polarimetric_transport"))
