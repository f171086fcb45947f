"""GPU parity: the native solve against the FP64 oracle and the reference's
golden vectors.  Tolerances: path gain 0.01 dB, phase 1e-3 rad, lengths
1e-5 relative; integer topology (path sets, sequences, edge ids) exact."""

from __future__ import annotations

import numpy as np
import pytest
import torch

from oracle import solve as osolve
from tests import scenes
from witwin_channel_b200 import Config, solve

pytestmark = pytest.mark.gpu

DB_TOL = 0.01
PHASE_TOL = 1.0e-3


def _oracle(scene, freq, **kw):
    arr = osolve.scene_arrays(scene, freq)
    return osolve.solve(arr, frequency=freq, edge_policy=scene.metadata.get("imported_edge_policy"), **kw)


def _grid_flat(x: torch.Tensor, shape):
    rows, cols = shape
    return x.transpose(1, 2).reshape(x.shape[0], rows * cols)


def _db(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    mask = (a > 0) | (b > 0)
    return np.abs(10.0 * np.log10(np.maximum(a[mask], 1e-300) / np.maximum(b[mask], 1e-300)))


def _rows_key(t, r, c, d, seq, e):
    return [(int(t[i]), int(r[i]), int(c[i]), int(d[i]), tuple(int(x) for x in seq[i]), int(e[i])) for i in range(len(t))]


def _cell_scale(ref, T, R):
    """Per-cell sum of |path field| (the magnitude a coherent sum can reach)."""
    r = ref["rows"]
    scale = np.zeros((T, R))
    np.add.at(scale, (r["tx_id"], r["rx_id"]), np.abs(r["path_field"]))
    return scale


def _check_cells(got_field, want_field, scale):
    """Coherent cell sums: |F - F_ref| <= 1e-3 * sum|f_p| (0.01 dB / 1e-3 rad
    of the constituent paths; a deep interference null is not a dB test)."""
    err = np.abs(np.asarray(got_field) - np.asarray(want_field))
    assert np.all(err <= 1e-3 * scale + 1e-30), (err / np.maximum(scale, 1e-300)).max()


def _compare_paths(res, ref, phases=True):
    p = res.paths
    got = _rows_key(p.tx_id.cpu(), p.rx_id.cpu(), p.component_id.cpu(), p.depth.cpu(), p.primitive_sequence.cpu(),
                    p.edge_id.cpu())
    r = ref["rows"]
    want = _rows_key(r["tx_id"], r["rx_id"], r["component_id"], r["depth"], r["primitive_sequence"], r["edge_id"])
    assert got == want
    np.testing.assert_allclose(p.path_length_m.cpu().numpy(), r["path_length_m"], rtol=1e-5, atol=1e-5)
    g = p.path_gain.cpu().numpy().astype(np.float64)
    w = np.asarray(r["path_gain"], dtype=np.float64)
    # dB bound for every path within 60 dB of the strongest; below that the
    # FP32 field sums cancel and only an absolute bound is meaningful
    strong_gain = w >= 1e-6 * w.max() if w.size else w.astype(bool)
    assert np.all(_db(g[strong_gain], w[strong_gain]) <= DB_TOL)
    if w.size:
        assert np.all(np.abs(g[~strong_gain] - w[~strong_gain]) <= 1e-8 * w.max())
    if not phases:
        return
    pf = torch.complex(p.field_real, p.field_imag).cpu().numpy()
    strong = np.abs(r["path_field"]) > 1e-3 * np.abs(r["path_field"]).max()
    ph = np.abs(np.angle(pf[strong] / r["path_field"][strong]))
    assert np.all(ph <= PHASE_TOL), ph.max()


def test_two_wall_multibounce_golden_and_oracle():
    scene = scenes.two_wall_scene()
    res = solve(scene, Config(components={"reflection"}, max_depth=2, coherent=True, export_paths=True),
                reference_frequency_hz=3.0e9)
    p = res.paths
    # golden: tests/deterministic/test_reflection_multibounce.py:185-205
    assert p.depth.tolist() == [1, 1, 2]
    assert p.primitive_sequence.tolist() == [[0, -1], [2, -1], [1, 2]]
    torch.testing.assert_close(p.path_length_m.cpu(), torch.tensor([4.123105526, 3.0, 5.0]), rtol=1e-5, atol=1e-6)
    ref = _oracle(scene, 3.0e9, components={"reflection"}, max_depth=2)
    _compare_paths(res, ref)
    torch.testing.assert_close(res.path_gain.cpu(), res.field.abs().square().cpu(), rtol=2e-4, atol=1e-10)


def test_single_wedge_edges_and_lengths_golden():
    scene = scenes.wedge_scene()
    res = solve(scene, Config(components={"diffraction"}, coherent=False, export_paths=True, return_field=False),
                reference_frequency_hz=3.0e9)
    p = res.paths
    # golden: tests/deterministic/test_diffraction_single_wedge.py:36-80
    assert p.edge_id.tolist() == [0, 1, 2, 5]
    torch.testing.assert_close(p.path_length_m.cpu(),
                               torch.tensor([3.650281668, 4.744879723, 3.768759727, 4.046976566]),
                               rtol=1e-5, atol=1e-6)
    ref = _oracle(scene, 3.0e9, components={"diffraction"}, max_depth=1, coherent=False)
    # return_field=False exports zero-phase fields (deterministic.py:473-478)
    _compare_paths(res, ref, phases=False)
    assert torch.all(res.paths.phase_rad == 0)
    # golden gains (test_diffraction_single_wedge.py:64-79) of edges 1, 2, 5;
    # edge 0 is a ~3e-18 null at the reference's float32 floor
    golden = np.array([2.980571e-18, 2.680186e-11, 1.471983e-08, 6.686395e-09])
    db = 10.0 * np.log10(p.path_gain.double().cpu().numpy() / golden)[1:]
    assert abs(db[0]) <= 0.1 and np.all(np.abs(db[1:]) <= 2.0), db


def test_los_grid_layout_matches_closed_form():
    scene = scenes.los_grid_scene()
    res = solve(scene, Config(max_depth=0, components={"los"}), reference_frequency_hz=3.0e9)
    assert tuple(res.path_gain.shape) == (1, 3, 2)
    # reference_channel.py:35-81 closed form
    grid = scene.receivers[0]
    pts = grid.points().double()
    tx = torch.tensor([0.0, 0.0, 0.0], dtype=torch.float64)
    d = pts - tx
    dist = d.norm(dim=-1)
    khat = d / dist[:, None]
    lam = 299792458.0 / 3.0e9
    pz = torch.tensor([0.0, 0.0, 1.0], dtype=torch.float64)
    dip = (1.0 - (khat @ pz) ** 2) ** 2
    want = 1.5 * (lam / (4 * np.pi * dist)) ** 2 * dip
    want = want.reshape(1, 2, 3).transpose(1, 2)
    torch.testing.assert_close(res.path_gain.double().cpu(), want, rtol=1e-5, atol=1e-12)


@pytest.mark.parametrize("export", [False, True])
def test_two_ray_radiomap_matches_oracle(export):
    from witwin_channel_b200.workloads import two_ray_scene

    scene, freq = two_ray_scene(shape=(16, 16), spacing=8.0)
    res = solve(scene, Config(components={"los", "reflection"}, max_depth=1, export_paths=export),
                reference_frequency_hz=freq)
    ref = _oracle(scene, freq, components={"los", "reflection"}, max_depth=1)
    got = _grid_flat(res.path_gain, (16, 16)).cpu().numpy()
    assert np.all(_db(got, ref["path_gain"]) <= DB_TOL)
    gf = _grid_flat(res.field, (16, 16)).cpu().numpy()
    assert np.all(np.abs(np.angle(gf / ref["field"])) <= PHASE_TOL)
    if export:
        _compare_paths(res, ref)


def test_thin_wall_transmission_matches_oracle():
    scene = scenes.thin_wall_scene()
    cfg = Config(components={"los", "reflection", "transmission"}, max_depth=2, export_paths=True)
    res = solve(scene, cfg, reference_frequency_hz=28.0e9)
    ref = _oracle(scene, 28.0e9, components={"los", "reflection", "transmission"}, max_depth=2)
    _compare_paths(res, ref)
    assert int((res.paths.component_id == 5).sum()) > 0


@pytest.mark.parametrize("coherent", [True, False])
def test_small_city_all_components_matches_oracle(coherent):
    scene, freq = scenes.small_city()
    comps = {"los", "reflection", "diffraction", "transmission"}
    cfg = Config(components=comps, max_depth=2, export_paths=True, coherent=coherent)
    res = solve(scene, cfg, reference_frequency_hz=freq)
    ref = _oracle(scene, freq, components=comps, max_depth=2, coherent=coherent)
    _compare_paths(res, ref)
    got = _grid_flat(res.path_gain, (8, 8)).cpu().numpy()
    want = ref["path_gain"]
    if not coherent:
        # grid: the diffraction component power is the exact vector sum
        want = want - ref["component_power"][2] + ref["diffraction_vector_power"]
        assert np.all(_db(got, want) <= DB_TOL)
    else:
        _check_cells(_grid_flat(res.field, (8, 8)).cpu().numpy(), ref["field"], _cell_scale(ref, 1, 64))
        for slot, name in ((0, "los"), (1, "reflection"), (3, "transmission")):
            if name in res.component_fields:
                _check_cells(_grid_flat(res.component_fields[name], (8, 8)).cpu().numpy(), ref["component_field"][slot],
                             _cell_scale(ref, 1, 64))


def test_cell_mode_equals_row_mode():
    scene, freq = scenes.small_city()
    comps = {"los", "reflection", "diffraction", "transmission"}
    a = solve(scene, Config(components=comps, max_depth=2), reference_frequency_hz=freq)
    b = solve(scene, Config(components=comps, max_depth=2, export_paths=True), reference_frequency_hz=freq)
    assert np.all(_db(a.path_gain.cpu().numpy(), b.path_gain.cpu().numpy()) <= 1e-3)
    for name in a.component_power:
        assert np.all(_db(a.component_power[name].cpu().numpy(), b.component_power[name].cpu().numpy()) <= 1e-3)


def test_fp64_mode_matches_mixed():
    scene, freq = scenes.small_city()
    comps = {"los", "reflection", "diffraction", "transmission"}
    a = solve(scene, Config(components=comps, max_depth=2), reference_frequency_hz=freq)
    b = solve(scene, Config(components=comps, max_depth=2), reference_frequency_hz=freq, precision="fp64")
    assert b.path_gain.dtype == torch.float64
    ref = _oracle(scene, freq, components=comps, max_depth=2)
    scale = _cell_scale(ref, 1, 64)
    _check_cells(_grid_flat(a.field, (8, 8)).cpu().numpy(), ref["field"], scale)
    _check_cells(_grid_flat(b.field, (8, 8)).cpu().numpy(), ref["field"], scale)


def test_solve_is_deterministic():
    scene, freq = scenes.small_city()
    cfg = Config(components={"los", "reflection", "diffraction"}, max_depth=2)
    a = solve(scene, cfg, reference_frequency_hz=freq).path_gain
    b = solve(scene, cfg, reference_frequency_hz=freq).path_gain
    assert torch.equal(a, b)


def test_compiled_scene_is_cached_and_invalidated():
    import torch as _t

    from witwin_channel_b200.compiler import compile_scene

    scene = scenes.two_wall_scene()
    dev = _t.device("cuda")
    a = compile_scene(scene, dev)
    assert compile_scene(scene, dev) is a
    with _t.no_grad():
        scene.structures[0].vertices.add_(0.0)  # bumps the tensor version: the vertices are re-read
    assert compile_scene(scene, dev) is a  # ... and refitted in place (no compile decision changed)
    st = scene.structures[0]
    st.geometry.faces = st.faces.flip(1).clone()  # a new face tensor: compiled again
    assert compile_scene(scene, dev) is not a


def _cell_maps(scene, freqs, comps):
    from witwin_channel_b200 import engine
    from witwin_channel_b200.compiler import compile_scene
    from witwin_channel_b200.deterministic import _endpoints

    device = torch.device("cuda", torch.cuda.current_device())
    compiled = compile_scene(scene, device)
    ep = _endpoints(scene, device)
    mats = compiled.material_tables(list(freqs), device)
    cells = engine.alloc_cells(len(freqs), ep.num_tx, ep.num_rx, device)
    engine.run_solve(compiled, ep, mats, list(freqs), components=engine.component_bits(comps), max_depth=1,
                     coherent=True, cells=cells)
    return cells


def test_diffraction_edge_chunks_match_one_chunk(monkeypatch):
    """The diffraction kernels split a long edge list into chunks whose
    visibility words fit a fixed budget; a tiny budget (32-edge chunks, with
    running sums carried between chunks) gives the same rows and, up to FP32
    summation order, the same maps as one chunk, also over two frequency
    blocks (5 frequencies)."""
    scene, freq = scenes.small_city(n_boxes=8, seed=11, grid=(12, 10))
    comps = {"los", "diffraction"}
    cfg = Config(components=comps, max_depth=1, export_paths=True, coherent=True)
    freqs = (3.5e9, 6.0e9, 12.0e9, 20.0e9, 28.0e9)
    one = solve(scene, cfg, reference_frequency_hz=freq)
    one_c = _cell_maps(scene, freqs, comps)
    monkeypatch.setenv("WCB_DIFFRACTION_CHUNK_WORDS", "1")
    many = solve(scene, cfg, reference_frequency_hz=freq)
    many_c = _cell_maps(scene, freqs, comps)
    assert int((one.paths.component_id == 2).sum()) > 32
    ka = _rows_key(one.paths.tx_id.cpu(), one.paths.rx_id.cpu(), one.paths.component_id.cpu(), one.paths.depth.cpu(),
                   one.paths.primitive_sequence.cpu(), one.paths.edge_id.cpu())
    kb = _rows_key(many.paths.tx_id.cpu(), many.paths.rx_id.cpu(), many.paths.component_id.cpu(),
                   many.paths.depth.cpu(), many.paths.primitive_sequence.cpu(), many.paths.edge_id.cpu())
    assert ka == kb
    pairs = ((one.component_power["diffraction"], many.component_power["diffraction"]),
             (one.path_gain, many.path_gain), (one_c.comp_power[2], many_c.comp_power[2]),
             (one_c.diff_vec_power, many_c.diff_vec_power), (one_c.path_gain, many_c.path_gain))
    for a, b in pairs:
        a = a.double().cpu()
        b = b.double().cpu()
        assert float(a.abs().max()) > 0
        assert torch.all((a - b).abs() <= 1e-5 * a.abs() + 1e-6 * float(a.abs().max()))


def test_chain_dedup_bitmap_equals_sort(monkeypatch):
    """Discovery-mode chains (16 boxes, depth 3: too many group sequences for
    the exhaustive tables) deduplicated through the bitmap and through the
    radix sort give the same chain tables, hence bit-identical maps."""
    scene, freq = scenes.small_city(n_boxes=16, seed=5, grid=(12, 10))
    cfg = Config(components={"los", "reflection"}, max_depth=3, coherent=True)
    a = solve(scene, cfg, reference_frequency_hz=freq)
    monkeypatch.setenv("WCB_CHAIN_BITMAP_BITS", "0")
    b = solve(scene, cfg, reference_frequency_hz=freq)
    assert float(a.path_gain.max()) > 0
    assert torch.equal(a.path_gain, b.path_gain)
    assert torch.equal(a.component_power["reflection"], b.component_power["reflection"])


def test_discovery_mode_paths_match_oracle():
    """Multi-bounce chains found by tracing Fibonacci rays (16 boxes, depth 3:
    too many group sequences for the exhaustive tables), deduplicated and
    validated on the GPU, against the oracle's FP64 discovery of the same
    8192 directions: identical path records."""
    from witwin_channel_b200 import engine
    from witwin_channel_b200.compiler import compile_scene
    from witwin_channel_b200.deterministic import _endpoints

    scene, freq = scenes.small_city(n_boxes=16, seed=5, grid=(6, 5), spacing=9.0)
    rays = 8192
    device = torch.device("cuda", torch.cuda.current_device())
    compiled = compile_scene(scene, device)
    ep = _endpoints(scene, device)
    mats = compiled.material_tables([freq], device)
    res = engine.run_solve(compiled, ep, mats, [freq], components=engine.component_bits({"reflection"}), max_depth=3,
                           coherent=True, want_rows=True, discovery_rays=rays)
    sel = engine.select_rows(res["rows"], 3, None, "global")
    dec = engine.decode_rows(res["rows"], sel)
    got = _rows_key(dec["tx_id"].cpu(), dec["rx_id"].cpu(), dec["component_id"].cpu(), dec["depth"].cpu(),
                    dec["seq"][:, :3].cpu(), dec["edge_id"].cpu())
    ref = _oracle(scene, freq, components={"reflection"}, max_depth=3, discovery_rays=rays)
    r = ref["rows"]
    want = _rows_key(r["tx_id"], r["rx_id"], r["component_id"], r["depth"], r["primitive_sequence"], r["edge_id"])
    assert max(len(got), len(want)) > 0
    assert sum(1 for k in got if k[3] >= 2) > 0  # multi-bounce records from discovered chains
    assert got == want
