"""Failure paths of the native solve, provoked from the host.

The reference records capacity failures in a device bitmask and ends the
solve through a terminal check (``witwin/channel/runtime.py:1280-1437``).
Here no kernel traps: each failure ends in a documented status that the host
reads, and the context stays usable.  Every case is made on the host side (a
short buffer, a scene with more walls than max_depth, a traversal stack
smaller than the BVH depth); no GPU is faulted.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from oracle import solve as osolve
from tests import scenes
from witwin_channel_b200 import Config, _native, engine, solve
from witwin_channel_b200.compiler import compile_scene
from witwin_channel_b200.deterministic import _endpoints
from witwin_channel_b200.scene import PhysicalMaterial, Scene, make_mesh_structure, make_receiver, make_transmitter

pytestmark = pytest.mark.gpu


def _prepared(scene, f):
    device = torch.device("cuda", torch.cuda.current_device())
    compiled = compile_scene(scene, device)
    ep = _endpoints(scene, device)
    mats = compiled.material_tables([f], device)
    return compiled, ep, mats


def test_row_capacity_error_without_retry():
    scene, f = scenes.small_city(n_boxes=4, seed=7, grid=(6, 6), spacing=6.0)
    compiled, ep, mats = _prepared(scene, f)
    bits = engine.component_bits({"los", "reflection", "diffraction"})
    with pytest.raises(_native.NativeError) as err:
        engine.run_solve(compiled, ep, mats, [f], components=bits, max_depth=2, coherent=True, want_rows=True,
                         row_capacity=4, retry=False)
    assert err.value.status == _native.WCB_ERR_CAPACITY
    # the same solve with the retry: the reported count sizes the next buffer
    res = engine.run_solve(compiled, ep, mats, [f], components=bits, max_depth=2, coherent=True, want_rows=True,
                           row_capacity=4)
    assert int(res["rows"].shape[0]) > 4
    assert int(res["status"].item()) == 0


def _three_walls(max_depth):
    glass = PhysicalMaterial(eps_r=6.27, sigma_e=0.2287, thickness_m=0.012)
    walls = []
    for i, x in enumerate((2.0, 4.0, 6.0)):
        v = torch.tensor([[x, -3.0, -3.0], [x, 3.0, -3.0], [x, -3.0, 3.0], [x, 3.0, 3.0]])
        walls.append(make_mesh_structure(vertices=v, faces=torch.tensor([[0, 1, 2], [1, 3, 2]]), material=glass,
                                         surface_id=i + 1))
    return Scene(structures=walls, endpoints=[make_transmitter([0.0, 0.2, 0.1]), make_receiver([8.0, -0.3, 0.2]),
                                               make_receiver([5.0, 0.4, -0.1])])


def test_transmission_over_depth_is_counted():
    f = 28.0e9
    cfg2 = Config(components={"transmission"}, max_depth=2, export_paths=True)
    res2 = solve(_three_walls(2), cfg2, reference_frequency_hz=f)
    # receiver 0 is behind three walls (over depth 2: counted, no path); receiver 1 behind two
    assert res2.metadata["transmission_overflow"] == 1
    assert res2.paths.rx_id.tolist() == [1]
    ref = osolve.solve(osolve.scene_arrays(_three_walls(2), f), components={"transmission"}, max_depth=2, frequency=f)
    assert ref["transmission_overflow"] == 1
    res3 = solve(_three_walls(3), Config(components={"transmission"}, max_depth=3, export_paths=True),
                 reference_frequency_hz=f)
    assert res3.metadata["transmission_overflow"] == 0
    assert sorted(res3.paths.rx_id.tolist()) == [0, 1]
    assert res3.paths.depth.tolist() == [3, 2]


def test_traversal_stack_overflow_sets_status():
    scene, f = scenes.small_city(n_boxes=16, seed=5, grid=(6, 5), spacing=9.0)
    compiled, ep, mats = _prepared(scene, f)
    bits = engine.component_bits({"los", "reflection", "diffraction"})
    cells = engine.alloc_cells(1, ep.num_tx, ep.num_rx, torch.device("cuda", torch.cuda.current_device()))
    ok = engine.run_solve(compiled, ep, mats, [f], components=bits, max_depth=2, coherent=True, cells=cells)
    assert int(ok["status"].item()) == 0
    reference_gain = cells.path_gain.clone()
    # one stack entry per thread: descents that need a second entry drop the
    # far subtree and set bit 0; the solve completes and the host sees it
    short = engine.run_solve(compiled, ep, mats, [f], components=bits, max_depth=2, coherent=True, cells=cells,
                             check_status=False, stack_entries=1)
    assert int(short["status"].item()) & 1
    with pytest.raises(RuntimeError, match="traversal stack overflow"):
        engine.check_device_status(short["status"])
    # the context is still usable: the full stack gives the same map again
    again = engine.run_solve(compiled, ep, mats, [f], components=bits, max_depth=2, coherent=True, cells=cells)
    assert int(again["status"].item()) == 0
    assert torch.equal(cells.path_gain, reference_gain)
    assert np.isfinite(cells.path_gain.cpu().numpy()).all()
