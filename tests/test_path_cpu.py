"""Path-solver packing on CPU tensors: ragged per-pair storage, the padded
result, its CIR and tap views and the type filter (the contract of the
reference's tests/path/test_path_result.py and test_path_signal_views.py)."""

from __future__ import annotations

from dataclasses import replace

import pytest
import torch

import witwin_channel_b200.path as path_api
from witwin_channel_b200.path import Config, InteractionType, PathResult, RaggedPathSoA


def test_public_names():
    assert set(path_api.__all__) == {"Config", "InteractionType", "PathResult", "RaggedPathSoA", "solve"}


def test_config_validation():
    with pytest.raises(ValueError, match="per_pair"):
        Config(max_paths_scope="global")
    with pytest.raises(ValueError, match="max_paths"):
        Config(max_paths=0)
    with pytest.raises(RuntimeError, match="max_depth <= 5"):
        Config(max_depth=6, components={"reflection"})
    with pytest.raises(ValueError, match="ad_mode"):
        Config(ad_mode="forward")
    assert Config(components=["los"]).components == frozenset({"los"})


def _ragged(*, count, rx_id=None, tx_id=None, field=None, depth=2, max_paths=None):
    rx_id = torch.tensor(rx_id if rx_id is not None else [0] * count, dtype=torch.int32)
    tx_id = torch.tensor(tx_id if tx_id is not None else [0] * count, dtype=torch.int32)
    field = field if field is not None else torch.ones((count, 1), dtype=torch.complex64)
    types = torch.zeros((count, depth), dtype=torch.int32)
    if count and depth:
        types[:, 0] = int(InteractionType.REFLECTION)
    return RaggedPathSoA.from_flat(
        num_rx=2, num_rx_ant=1, num_tx=2, num_tx_ant=1, rx_id=rx_id, tx_id=tx_id, field=field,
        delay_s=torch.arange(count, dtype=torch.float32) * 1.0e-9, theta_t=torch.zeros(count),
        phi_t=torch.zeros(count), theta_r=torch.zeros(count), phi_r=torch.zeros(count), interaction_type=types,
        primitive_id=torch.full((count, depth), -1, dtype=torch.int32),
        material_id=torch.full((count, depth), -1, dtype=torch.int32), position=torch.zeros((count, depth, 3)),
        normal=torch.zeros((count, depth, 3)), max_paths_per_pair=max_paths)


def test_zero_paths_keep_a_zero_width_path_dimension():
    result = PathResult.from_ragged(_ragged(count=0))
    assert result.a.shape == (2, 1, 2, 1, 0, 1)
    assert result.valid.shape == (2, 1, 2, 1, 0)
    assert result.num_paths.shape == (2, 1, 2, 1)
    assert int(result.num_paths.sum()) == 0


def test_ragged_packing_is_stable_per_pair_with_the_per_pair_limit():
    field = torch.tensor([[10], [20], [30], [40], [50]], dtype=torch.complex64)
    ragged = _ragged(count=5, rx_id=[1, 0, 1, 0, 1], tx_id=[0, 1, 0, 1, 0], field=field, max_paths=2)
    result = PathResult.from_ragged(ragged, max_paths_per_pair=2)
    assert result.metadata["max_paths_scope"] == "per_pair"
    assert int(result.num_paths[0, 0, 1, 0]) == 2
    assert int(result.num_paths[1, 0, 0, 0]) == 2
    assert result.a[0, 0, 1, 0, :, 0].real.tolist() == [20.0, 40.0]
    assert result.a[1, 0, 0, 0, :, 0].real.tolist() == [10.0, 30.0]
    with pytest.raises(ValueError, match="exceeds"):
        PathResult.from_ragged(_ragged(count=3), max_paths_per_pair=2)


@pytest.mark.parametrize(("field", "values"), [("rx_id", [-1]), ("rx_ant_id", [1]), ("tx_id", [2]), ("tx_ant_id", [1])])
def test_ragged_rejects_ids_outside_their_dimension(field, values):
    ids = {k: torch.tensor([0], dtype=torch.int32) for k in ("rx_id", "rx_ant_id", "tx_id", "tx_ant_id")}
    ids[field] = torch.tensor(values, dtype=torch.int32)
    with pytest.raises(ValueError, match=field):
        RaggedPathSoA.from_flat(num_rx=2, num_rx_ant=1, num_tx=2, num_tx_ant=1,
                                field=torch.ones((1, 1), dtype=torch.complex64), delay_s=torch.zeros(1),
                                theta_t=torch.zeros(1), phi_t=torch.zeros(1), theta_r=torch.zeros(1),
                                phi_r=torch.zeros(1), interaction_type=torch.empty((1, 0), dtype=torch.int32),
                                primitive_id=torch.empty((1, 0), dtype=torch.int32),
                                material_id=torch.empty((1, 0), dtype=torch.int32), position=torch.empty((1, 0, 3)),
                                normal=torch.empty((1, 0, 3)), **ids)


def test_result_validates_its_shapes():
    result = PathResult.from_ragged(_ragged(count=1))
    with pytest.raises(ValueError, match="tau"):
        replace(result, tau=torch.zeros(2))
    with pytest.raises(ValueError, match="complex64"):
        replace(result, a=result.a.to(torch.complex128))


def _signal_result() -> PathResult:
    field = torch.tensor([[1.0 + 0.0j], [0.0 + 2.0j]], dtype=torch.complex64)
    types = torch.tensor([[int(InteractionType.REFLECTION)], [int(InteractionType.DIFFRACTION)]], dtype=torch.int32)
    ragged = RaggedPathSoA.from_flat(
        num_rx=1, num_rx_ant=1, num_tx=1, num_tx_ant=1, rx_id=torch.zeros(2, dtype=torch.int32),
        tx_id=torch.zeros(2, dtype=torch.int32), field=field, delay_s=torch.tensor([1.0e-9, 3.0e-9]),
        theta_t=torch.zeros(2), phi_t=torch.zeros(2), theta_r=torch.zeros(2), phi_r=torch.zeros(2),
        interaction_type=types, primitive_id=torch.tensor([[3], [7]], dtype=torch.int32),
        material_id=torch.tensor([[1], [2]], dtype=torch.int32), position=torch.zeros((2, 1, 3)),
        normal=torch.zeros((2, 1, 3)))
    return PathResult.from_ragged(ragged)


def test_cir_masks_padding_and_normalises_delay_per_pair():
    result = _signal_result()
    coeff, tau = result.cir()
    assert torch.equal(coeff, result.a)
    assert torch.allclose(tau.flatten(), torch.tensor([0.0, 2.0e-9]))
    assert torch.allclose(result.path_length_m.flatten(), torch.tensor([1.0e-9, 3.0e-9]) * 299_792_458.0)


def test_taps_accumulate_into_rounded_bins():
    taps = _signal_result().taps(bandwidth=1.0e9, num_taps=4)
    assert taps.shape == (1, 1, 1, 1, 1, 4)
    assert taps[..., 0].item() == 1.0 + 0.0j
    assert taps[..., 2].item() == 0.0 + 2.0j
    with pytest.raises(ValueError, match="bandwidth"):
        _signal_result().taps(bandwidth=0.0, num_taps=4)


def test_filter_by_type_compacts_and_keeps_geometry():
    filtered = _signal_result().filter_by_type(InteractionType.DIFFRACTION)
    assert filtered.a.shape == (1, 1, 1, 1, 1, 1)
    assert int(filtered.num_paths.item()) == 1
    assert filtered.a.item() == 0.0 + 2.0j
    assert int(filtered.primitive_id.item()) == 7
    assert filtered.metadata["filtered_interaction_types"] == [2]
    empty = _signal_result().filter_by_type(InteractionType.TRANSMISSION)
    assert empty.a.shape == (1, 1, 1, 1, 1, 1)  # minimum width 1
    assert int(empty.num_paths.item()) == 0
    assert not bool(empty.valid.any())


def test_beamformed_views_weight_and_merge_antenna_pairs():
    result = _signal_result()
    bf = result.beamform(tx_weights=torch.tensor([2.0 + 0j]), rx_weights=torch.tensor([0.0 + 1.0j]))
    coeff, tau = bf.cir()
    # conj(rx) * tx = -2j
    assert torch.allclose(coeff.flatten(), torch.tensor([-2.0j, 4.0 + 0j], dtype=torch.complex64))
    assert torch.allclose(tau.flatten(), torch.tensor([0.0, 2.0e-9]))
    taps = bf.taps(bandwidth=1.0e9, num_taps=4)
    assert taps.shape == (1, 1, 1, 4)
    assert taps[0, 0, 0, 2].item() == 4.0 + 0j


def test_cfr_needs_the_gpu():
    with pytest.raises(RuntimeError, match="GPU"):
        _signal_result().cfr(torch.tensor([0.0, 1.0e6]))
