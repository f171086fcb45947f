"""CPU: ``Config`` validation raises what the reference raises
(``witwin/channel/deterministic.py:105-217``), and the host-side layout and
frequency handling of ``solve``."""

from __future__ import annotations

import pytest
import torch

from witwin_channel_b200 import Config
from witwin_channel_b200.deterministic import _frequency_value, _layout, _layout_inverse


@pytest.mark.parametrize("kwargs,exc", [
    ({"max_depth": -1}, ValueError),
    ({"components": set()}, ValueError),
    ({"components": {"los", "bogus"}}, ValueError),
    ({"max_paths": 0}, ValueError),
    ({"max_paths_scope": "everywhere"}, ValueError),
    ({"sort_key": "by_gain"}, ValueError),
    ({"ad_mode": "forward"}, RuntimeError),
    ({"max_diffraction_order": 2}, RuntimeError),
    ({"max_diffraction_order": -1}, ValueError),
    ({"scattering_coherent": True}, RuntimeError),
    ({"max_depth": 6, "components": {"reflection"}}, RuntimeError),
    ({"isb_boundary_taper_width": 0.0}, ValueError),
    ({"coupled_candidate_limit": 0}, ValueError),
])
def test_config_rejects_like_the_reference(kwargs, exc):
    with pytest.raises(exc):
        Config(**kwargs)


def test_config_defaults_and_normalisation():
    c = Config()
    assert c.components == frozenset({"los", "reflection", "diffraction"})
    assert c.max_depth == 1 and c.coherent and c.return_field and not c.export_paths
    c = Config(components=["los", "los", "diffraction"], max_depth=6)  # depth cap applies to reflection only
    assert c.components == frozenset({"los", "diffraction"})


def test_reference_frequency_validation():
    assert _frequency_value(28e9) == 28e9
    assert _frequency_value(torch.tensor(3.5e9, dtype=torch.float64)) == 3.5e9
    with pytest.raises(ValueError):
        _frequency_value(-1.0)
    with pytest.raises(ValueError):
        _frequency_value(torch.tensor([1e9, 2e9]))


def test_grid_layout_round_trip():
    """Grid outputs are (T, shape[1], shape[0]) (``propagation/geometry.py:79-89``):
    flat receiver r = row * cols + col lands at [t, col, row]."""
    rows, cols = 3, 4
    rx = {"kind": "grid", "shape": (rows, cols), "count": rows * cols}
    flat = torch.arange(2 * rows * cols, dtype=torch.float32).reshape(2, rows * cols)
    grid = _layout(flat, rx)
    assert tuple(grid.shape) == (2, cols, rows)
    assert grid[1, 2, 1] == flat[1, 1 * cols + 2]
    assert torch.equal(_layout_inverse(grid, rx), flat)
