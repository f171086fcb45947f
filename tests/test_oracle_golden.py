"""CPU: the oracle against the reference's golden vectors and known answers.

* field algebra against ``tests/golden/field_vectors.npz``, generated from the
  reference's complex128 mirror (``tests/ad/_reference_fields.py``) by
  ``tests/golden/make_field_vectors.py``;
* the flat accumulator against the reference's frozen SHA-256 outputs
  (``tests/ad/test_deterministic_accum_ad.py:37-80``);
* small-scene path sets, sequences, edge ids and lengths against the
  reference's deterministic tests (``tests/golden/reference_goldens.json``);
* the LoS grid layout against the closed form of
  ``tests/support/reference_channel.py:35-81``.
"""

from __future__ import annotations

import hashlib
import json
from pathlib import Path

import numpy as np
import pytest
import torch

from oracle import accumulate as oacc
from oracle import em
from oracle import solve as osolve
from tests import scenes
from witwin_channel_b200.scene import EdgePolicy, Scene

GOLDEN = Path(__file__).resolve().parent / "golden"
FIELDS = np.load(GOLDEN / "field_vectors.npz")
REF = json.loads((GOLDEN / "reference_goldens.json").read_text())

OUT_KEYS = ("field_vector", "coefficient", "path_field", "path_gain")


def _close(got, want, rtol=1e-9):
    """FP64 agreement: carrier phases reach k*d ~ 2.4e5 rad, where two libraries'
    complex exponentials differ by about k*d*2^-53 ~ 3e-11 relative."""
    got = np.asarray(got)
    want = np.asarray(want)
    scale = np.max(np.abs(want)) if want.size else 1.0
    np.testing.assert_allclose(got, want, rtol=rtol, atol=rtol * scale)


def test_free_space_matches_reference_mirror():
    f = FIELDS
    for i in range(f["fs_source"].shape[0]):
        out = em.free_space(f["fs_source"][i:i + 1], f["fs_target"][i:i + 1], f["fs_power"][i:i + 1],
                            f["fs_tx_pol"][i:i + 1], f["fs_rx_pol"][i:i + 1], float(f["fs_freq"][i]))
        for k in OUT_KEYS:
            _close(out[k][0], f["fs_" + k][i])


@pytest.mark.parametrize("depth", [1, 2, 3])
def test_reflection_chain_matches_reference_mirror(depth):
    p = f"rf{depth}_"
    f = {k[len(p):]: FIELDS[k] for k in FIELDS.files if k.startswith(p)}
    out = em.reflection_sequence(f["source"], f["target"], f["positions"], f["normals"], f["power"], f["tx_pol"],
                                 f["rx_pol"], f["eps_r"], f["sigma_e"], f["mu_r"], f["gain"], f["thickness"],
                                 float(f["freq"]))
    for k in OUT_KEYS:
        _close(out[k], f[k])


def test_transmission_stack_matches_reference_mirror():
    f = {k[3:]: FIELDS[k] for k in FIELDS.files if k.startswith("tr_")}
    layers = []
    for m in range(len(f["layer_offset"])):
        sl = slice(int(f["layer_offset"][m]), int(f["layer_offset"][m] + f["layer_count"][m]))
        layers.append((f["layer_thickness"][sl], f["layer_eps_r"][sl], f["layer_sigma_e"][sl], f["layer_mu_r"][sl]))
    out = em.transmission_sequence(f["source"], f["target"], f["normals"], f["material"], f["count"], f["power"],
                                   f["tx_pol"], f["rx_pol"], layers, float(f["freq"]))
    for k in OUT_KEYS:
        _close(out[k], f[k])


def _accum_fixture(dtype):
    fx = REF["accumulate_flat"]
    g = torch.Generator(device="cpu").manual_seed(fx["seed"])
    n = len(fx["tx_id"])
    gain = (torch.rand((n,), generator=g, dtype=torch.float64) + 0.25).numpy().astype(dtype)
    real = torch.randn((n,), generator=g, dtype=torch.float64).numpy().astype(dtype)
    imag = torch.randn((n,), generator=g, dtype=torch.float64).numpy().astype(dtype)
    return fx, gain, real, imag


@pytest.mark.parametrize("dtype", ["float32", "float64"])
@pytest.mark.parametrize("coherent", [True, False])
def test_accumulate_flat_reproduces_reference_sha256(dtype, coherent):
    fx, gain, real, imag = _accum_fixture(np.dtype(dtype).type)
    out = oacc.accumulate_flat(np.ones(len(gain), bool), fx["tx_id"], fx["rx_id"], fx["component_id"], gain, real,
                               imag, num_tx=fx["num_tx"], num_rx=fx["num_rx"], coherent=coherent,
                               dtype=np.dtype(dtype).type)
    payload = b"".join(np.ascontiguousarray(out[k]).tobytes() for k in oacc_fields())
    assert hashlib.sha256(payload).hexdigest() == fx["sha256"][f"{dtype}_{'coherent' if coherent else 'incoherent'}"]


def oacc_fields():
    return ("power_total", "field_total_real", "field_total_imag", "component_power", "component_field_real",
            "component_field_imag")


def test_accumulate_flat_drops_out_of_range_rows():
    fx, gain, real, imag = _accum_fixture(np.float64)
    keep = np.ones(len(gain), bool)
    keep[fx["dropped_rows"]] = False
    a = oacc.accumulate_flat(np.ones(len(gain), bool), fx["tx_id"], fx["rx_id"], fx["component_id"], gain, real,
                             imag, num_tx=2, num_rx=2, coherent=True, dtype=np.float64)
    b = oacc.accumulate_flat(keep, fx["tx_id"], fx["rx_id"], fx["component_id"], gain, real, imag, num_tx=2,
                             num_rx=2, coherent=True, dtype=np.float64)
    for k in oacc_fields():
        assert np.array_equal(a[k], b[k])


def _oracle(scene, freq, **kw):
    arr = osolve.scene_arrays(scene, freq)
    return osolve.solve(arr, frequency=freq, edge_policy=scene.metadata.get("imported_edge_policy"), **kw)


def test_two_wall_multibounce_golden():
    g = REF["two_wall_multibounce"]
    ref = _oracle(scenes.two_wall_scene(), 3.0e9, components={"reflection"}, max_depth=2)
    rows = ref["rows"]
    assert rows["depth"].tolist() == g["depth"]
    assert rows["primitive_sequence"].tolist() == g["primitive_sequence"]
    np.testing.assert_allclose(rows["path_length_m"], g["path_length_m"], rtol=1e-5, atol=1e-6)


def test_single_wedge_edge_ids_and_lengths_golden():
    g = REF["single_wedge"]
    ref = _oracle(scenes.wedge_scene(), 3.0e9, components={"diffraction"}, max_depth=1, coherent=False)
    rows = ref["rows"]
    assert rows["edge_id"].tolist() == g["edge_id"]
    np.testing.assert_allclose(rows["path_length_m"], g["path_length_m"], rtol=1e-5, atol=1e-6)


def test_single_wedge_gains_within_reference_test_tolerance():
    """The reference's own assertion (rtol 5e-3, atol 1e-8).  Its absolute
    term exceeds every golden gain, so this is a weak bound; the dB-level
    comparison below is the real one."""
    g = REF["single_wedge"]
    ref = _oracle(scenes.wedge_scene(), 3.0e9, components={"diffraction"}, max_depth=1, coherent=False)
    np.testing.assert_allclose(ref["rows"]["path_gain"], g["path_gain"], rtol=5e-3, atol=1e-8)


# Edge 0 (the merged vertical wedge) is a soft-polarisation null at ~3e-18,
# 1e-12 below the other rows: the golden there is the reference's float32
# rounding floor, so the dB comparisons use edges 1, 2 and 5.
_WEDGE_DB_ROWS = [1, 2, 3]


def _wedge_gain_db():
    g = np.asarray(REF["single_wedge"]["path_gain"])
    ref = _oracle(scenes.wedge_scene(), 3.0e9, components={"diffraction"}, max_depth=1, coherent=False)
    return 10 * np.log10(ref["rows"]["path_gain"] / g)[_WEDGE_DB_ROWS]


def test_single_wedge_gains_db_level():
    """Per-edge gains against the golden: edge 1 (a soft/hard cancellation
    that is sensitive to the wedge frame and to the half-plane's absent face)
    within 0.1 dB; the two slanted edges within 2 dB."""
    db = _wedge_gain_db()
    assert abs(db[0]) <= 0.1
    assert np.all(np.abs(db[1:]) <= 2.0)


@pytest.mark.xfail(strict=True, reason="the slanted half-plane edges 2 and 5 sit 1.7 and 1.4 dB above the golden; "
                                       "the residue lies in the reference's unshipped pair evaluation")
def test_single_wedge_gains_half_db():
    assert np.all(np.abs(_wedge_gain_db()) <= 0.5)


def test_vertical_only_edge_policy_keeps_three_edges():
    g = REF["single_wedge"]
    base = scenes.wedge_scene()
    filtered = Scene(structures=base.structures, endpoints=base.endpoints,
                     metadata={"imported_edge_policy": EdgePolicy(edge_selection_mode="vertical_only")})
    a = _oracle(base, 3.0e9, components={"diffraction"}, max_depth=1, coherent=False)
    b = _oracle(filtered, 3.0e9, components={"diffraction"}, max_depth=1, coherent=False)
    assert len(a["rows"]["edge_id"]) == g["rows_all_edges"]
    assert len(b["rows"]["edge_id"]) == g["rows_vertical_only"]


def test_los_grid_closed_form():
    scene = scenes.los_grid_scene()
    ref = _oracle(scene, 3.0e9, components={"los"}, max_depth=0)
    pts = scene.receivers[0].points().double().numpy()
    d = np.linalg.norm(pts, axis=1)
    khat = pts / d[:, None]
    lam = 299792458.0 / 3.0e9
    want = 1.5 * (lam / (4 * np.pi * d)) ** 2 * (1.0 - khat[:, 2] ** 2) ** 2
    np.testing.assert_allclose(np.asarray(ref["path_gain"]).reshape(-1), want, rtol=1e-5)


def test_edge_policy_validation_matches_reference():
    with pytest.raises(ValueError):
        EdgePolicy(edge_selection_mode="bogus")
    with pytest.raises(ValueError):
        EdgePolicy(boundary_edge_policy="bogus")
    with pytest.raises(ValueError):
        EdgePolicy(edge_diffraction=False, boundary_edge_policy="half_plane")
    assert EdgePolicy(edge_diffraction=False).boundary_edge_policy == "exclude"
    assert EdgePolicy().boundary_edge_policy == "half_plane"


def test_trace_reflections_between_parallel_mirrors():
    """Known-answer bounce chains between the mirrors x = 0 and x = 4 (each
    two triangles over y, z in [-100, 100]): a ray along +x alternates
    between them, a ray along +z escapes at once, and a ray that leaves the
    mirrors' extent after one bounce records one face then misses."""
    from oracle import geom

    sq = np.array([[-100, -100], [100, -100], [100, 100], [-100, 100]], dtype=np.float64)
    verts = np.concatenate([np.c_[np.zeros(4), sq], np.c_[np.full(4, 4.0), sq]])
    faces = np.array([[0, 1, 2], [0, 2, 3], [4, 5, 6], [4, 6, 7]])
    normals = np.array([[1.0, 0, 0], [1.0, 0, 0], [-1.0, 0, 0], [-1.0, 0, 0]])
    tris = geom.Triangles(verts, faces)
    dirs = np.array([[1.0, 0, 0], [0, 0, 1.0], [1.0 / np.sqrt(2), 0, 1.0 / np.sqrt(2)]])
    with np.errstate(invalid="raise"):
        chains = [geom.trace_reflections(tris, normals, np.array(o), dirs[i:i + 1], max_depth=4)[0].tolist()
                  for i, o in enumerate([(1.0, 0.3, 0.2), (1.0, 0.3, 0.2), (1.0, 0.3, 95.0)])]
    assert chains == [[2, 0, 2, 0], [-1, -1, -1, -1], [3, -1, -1, -1]]
