"""In-place scene refit after a vertex move (``wcb_scene_refit``).

A solve on a scene whose vertex tensors were replaced (same counts, same
faces, materials and surface ids) refits the compiled device scene instead of
compiling it again, when the move keeps every discrete compile decision
(coplanar groups as a partition, edge selection and wedge order,
shared-boundary merges).  Checked:

* the compiled scene object is reused exactly when the decisions hold (rigid
  moves of boxes and of a merged wedge pair), and recompiled when they break
  (a box top made non-planar, one half of a merged wedge moved alone);
* a refitted solve equals a fresh compile of the moved mesh: the same path
  rows and fields within 1e-6 relative (FP32 edge frames may differ in the
  last bit of an acos or atan2);
* an identity refit (a new tensor holding the same values) changes nothing;
* fixed-topology VJP gradients through a refitted scene equal those of a
  fresh compile.
"""

from __future__ import annotations

import math

import numpy as np
import pytest
import torch

from tests.test_gpu_vjp import wedge
from witwin_channel_b200 import Config, solve
from witwin_channel_b200.compiler import compile_scene
from witwin_channel_b200.workloads import urban_canyon_scene

pytestmark = pytest.mark.gpu

COMPS = {"los", "reflection", "diffraction"}


def _rows(res):
    p = res.paths
    cols = [p.tx_id, p.rx_id, p.component_id, p.depth, p.edge_id]
    key = np.stack([c.cpu().numpy().astype(np.int64) for c in cols], 1)
    seq = p.primitive_sequence.cpu().numpy().astype(np.int64).reshape(key.shape[0], -1)
    return np.concatenate([key, seq], 1)


def _same_result(a, b, rtol=1e-6):
    ra, rb = _rows(a), _rows(b)
    assert ra.shape == rb.shape and np.array_equal(ra, rb)
    torch.testing.assert_close(a.paths.field_real, b.paths.field_real, rtol=rtol, atol=1e-12)
    torch.testing.assert_close(a.paths.field_imag, b.paths.field_imag, rtol=rtol, atol=1e-12)
    torch.testing.assert_close(a.path_gain, b.path_gain, rtol=rtol, atol=1e-30)


def _rigid(v, shift, angle=0.0):
    """Rotate about the vertical axis through the centroid, then shift."""
    v = v.detach().clone()
    c = v.mean(0)
    ca, sa = math.cos(angle), math.sin(angle)
    x, y = v[:, 0] - c[0], v[:, 1] - c[1]
    v[:, 0] = c[0] + ca * x - sa * y + shift[0]
    v[:, 1] = c[1] + sa * x + ca * y + shift[1]
    v[:, 2] = v[:, 2] + shift[2]
    return v


def _canyon_moves(scene):
    """A translated box and a rotated box (rigid), as new tensors."""
    s1, s2 = scene.structures[1], scene.structures[5]
    s1.geometry.vertices = _rigid(s1.vertices, (0.37, -0.21, 0.0))
    s2.geometry.vertices = _rigid(s2.vertices, (0.0, 0.0, 0.0), angle=0.05)


def _solve(scene, f, **kw):
    return solve(scene, Config(components=COMPS, max_depth=2, export_paths=True, **kw), reference_frequency_hz=f)


def test_rigid_moves_refit_and_match_fresh_compile():
    scene, f = urban_canyon_scene(grid_side=64)
    _solve(scene, f)
    before = compile_scene(scene)
    _canyon_moves(scene)
    got = _solve(scene, f)
    assert compile_scene(scene) is before  # refitted in place
    fresh_scene, _ = urban_canyon_scene(grid_side=64)
    _canyon_moves(fresh_scene)
    want = _solve(fresh_scene, f)
    assert compile_scene(fresh_scene) is not before
    _same_result(got, want)


def test_identity_refit_changes_nothing():
    scene, f = urban_canyon_scene(grid_side=64)
    a = _solve(scene, f)
    before = compile_scene(scene)
    for st in scene.structures:
        st.geometry.vertices = st.vertices.detach().clone()
    b = _solve(scene, f)
    assert compile_scene(scene) is before
    _same_result(a, b, rtol=0.0)


def test_non_planar_move_recompiles():
    scene, f = urban_canyon_scene(grid_side=64)
    _solve(scene, f)
    before = compile_scene(scene)
    st = scene.structures[3]
    v = st.vertices.detach().clone()
    top = int(torch.argmax(v[:, 2]))
    v[top, 2] += 0.3  # the box top's two triangles are no longer coplanar
    st.geometry.vertices = v
    got = _solve(scene, f)
    assert compile_scene(scene) is not before
    fresh_scene, _ = urban_canyon_scene(grid_side=64)
    fresh_scene.structures[3].geometry.vertices = v.clone()
    _same_result(got, _solve(fresh_scene, f), rtol=0.0)


def _move_wedge(scene, which, shift):
    for i in which:
        st = scene.structures[i]
        st.geometry.vertices = (st.vertices.detach() + torch.tensor(shift)).requires_grad_(True)


@pytest.mark.parametrize("which, reused", [((0, 1), True), ((0,), False)])
def test_shared_boundary_merge_decides_refit(which, reused):
    freq = 3.0e9
    scene = wedge()
    cfg = Config(components={"diffraction"}, max_depth=1, export_paths=True)
    solve(scene, cfg, reference_frequency_hz=freq)
    before = compile_scene(scene)
    _move_wedge(scene, which, (0.011, -0.007, 0.003))
    got = solve(scene, cfg, reference_frequency_hz=freq)
    assert (compile_scene(scene) is before) == reused
    fresh = wedge()
    _move_wedge(fresh, which, (0.011, -0.007, 0.003))
    _same_result(got, solve(fresh, cfg, reference_frequency_hz=freq))


def test_vjp_through_refitted_scene_matches_fresh_compile():
    freq = 3.0e9

    def grads(scene):
        res = solve(scene, Config(components={"diffraction"}, max_depth=1, ad_mode="vjp"),
                    reference_frequency_hz=freq)
        loss = (res.path_gain.double() * 1e12).sum()
        loss.backward()
        return torch.cat([st.vertices.grad.reshape(-1) for st in scene.structures]), res

    scene = wedge()
    solve(scene, Config(components={"diffraction"}, max_depth=1), reference_frequency_hz=freq)
    before = compile_scene(scene)
    _move_wedge(scene, (0, 1), (0.02, 0.01, -0.01))
    g_refit, _ = grads(scene)
    assert compile_scene(scene) is before
    fresh = wedge()
    _move_wedge(fresh, (0, 1), (0.02, 0.01, -0.01))
    g_fresh, _ = grads(fresh)
    torch.testing.assert_close(g_refit, g_fresh, rtol=1e-6, atol=1e-12)


def test_device_lbvh_rebuild_keeps_every_result():
    """The device LBVH rebuild (``wcb_scene_rebuild_bvh``: Morton codes,
    radix sort, Karras radix tree, boxes bottom-up) changes only the tree:
    exhaustive-chain solves give identical rows and fields, and a refitted
    scene rebuilt on the device equals a fresh compile of the moved mesh."""
    from tests import scenes as sc

    scene, f = sc.small_city(grid=(10, 9))
    a = _solve(scene, f)
    compiled = compile_scene(scene)
    depth = compiled.native.rebuild_bvh()
    assert 1 <= depth <= 62
    b = _solve(scene, f)
    assert compile_scene(scene) is compiled
    _same_result(a, b, rtol=0.0)
    # the canyon: 262,144-ray discovery (closest hits), so compare the maps
    canyon, fc = urban_canyon_scene(grid_side=64)
    base = _solve(canyon, fc)
    cc = compile_scene(canyon)
    assert cc.native.rebuild_bvh() <= 62
    rebuilt = _solve(canyon, fc)
    g0, g1 = base.path_gain.double(), rebuilt.path_gain.double()
    off = ((g0 - g1).abs() > 1e-6 * g0.abs().max()).double().mean()
    assert float(off) < 1e-3
    # refit, then rebuild on the device: equal to a fresh compile of the moved mesh
    _canyon_moves(canyon)
    _solve(canyon, fc)
    assert compile_scene(canyon) is cc
    cc.native.rebuild_bvh()
    got = _solve(canyon, fc)
    fresh, _ = urban_canyon_scene(grid_side=64)
    _canyon_moves(fresh)
    want = _solve(fresh, fc)
    g0, g1 = want.path_gain.double(), got.path_gain.double()
    assert float(((g0 - g1).abs() > 1e-6 * g0.abs().max()).double().mean()) < 1e-3
