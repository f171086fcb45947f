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
    assert set(path_api.__all__) == {"Config", "InteractionType", "PathResult", "RaggedPathSoA", "solve",
                                     "apply_endpoint_weights", "pack_explicit_arrays", "pack_synthetic_arrays",
                                     "pattern_field_response", "steering_vector", "validate_synthetic_array_scene"}


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


# --- antenna arrays (reference path.py:1079-1486; the contract of the
# reference's tests/path/test_path_synthetic_arrays.py) ---------------------

import math

from witwin_channel_b200.scene import AntennaPattern, Scene, make_receiver, make_receiver_grid, make_transmitter


def _ula(n, spacing, axis=0):
    positions = torch.zeros((n, 3))
    positions[:, axis] = (torch.arange(n, dtype=torch.float32) - 0.5 * (n - 1)) * spacing
    return positions


def _ura(rows, cols, spacing):
    r, c = torch.meshgrid(torch.arange(rows) - 0.5 * (rows - 1), torch.arange(cols) - 0.5 * (cols - 1), indexing="ij")
    positions = torch.zeros((rows * cols, 3))
    positions[:, 0] = r.reshape(-1).float() * spacing
    positions[:, 1] = c.reshape(-1).float() * spacing
    return positions


def _centre(theta_t=math.pi / 2, phi_t=0.0, theta_r=math.pi / 2, phi_r=0.0):
    ragged = RaggedPathSoA.from_flat(
        num_rx=1, num_rx_ant=1, num_tx=1, num_tx_ant=1, rx_id=torch.zeros(1, dtype=torch.int32),
        tx_id=torch.zeros(1, dtype=torch.int32), field=torch.ones((1, 1), dtype=torch.complex64),
        delay_s=torch.tensor([1.0e-9]), theta_t=torch.tensor([theta_t]), phi_t=torch.tensor([phi_t]),
        theta_r=torch.tensor([theta_r]), phi_r=torch.tensor([phi_r]),
        interaction_type=torch.empty((1, 0), dtype=torch.int32), primitive_id=torch.empty((1, 0), dtype=torch.int32),
        material_id=torch.empty((1, 0), dtype=torch.int32), position=torch.empty((1, 0, 3)),
        normal=torch.empty((1, 0, 3)))
    return PathResult.from_ragged(ragged)


def test_synthetic_ula_adds_the_steering_phase_and_keeps_the_paths():
    # k = 2 pi at 1 lambda = 1 m: elements at x = -0.25, +0.25 along the
    # departure direction +x give phases -pi/2, +pi/2
    tx = make_transmitter(torch.zeros(3), element_positions=_ula(2, 0.5))
    out = path_api.pack_synthetic_arrays(_centre(), frequency_hz=299_792_458.0, transmitters=[tx],
                                         receivers=[make_receiver(torch.ones(3))])
    assert out.a.shape == (1, 1, 1, 2, 1, 1)
    torch.testing.assert_close(out.a[0, 0, 0, :, 0, 0], torch.tensor([-1.0j, 1.0j], dtype=torch.complex64),
                               atol=1e-6, rtol=1e-6)
    assert out.num_paths.tolist() == [[[[1, 1]]]]
    assert out.metadata["array_semantics"] == "synthetic_far_field_phase_weighting"
    assert out.metadata["num_tx_ant"] == 2 and out.metadata["num_rx_ant"] == 1
    torch.testing.assert_close(out.tau[0, 0, 0, :, 0], torch.tensor([1.0e-9, 1.0e-9]))


def test_synthetic_ura_is_row_major():
    tx = make_transmitter(torch.zeros(3), element_positions=_ura(2, 2, 0.5))
    out = path_api.pack_synthetic_arrays(_centre(), frequency_hz=299_792_458.0, transmitters=[tx],
                                         receivers=[make_receiver(torch.ones(3))])
    torch.testing.assert_close(out.a[0, 0, 0, :, 0, 0],
                               torch.tensor([-1.0j, -1.0j, 1.0j, 1.0j], dtype=torch.complex64), atol=1e-6, rtol=1e-6)


def test_rotated_directional_pattern_is_evaluated_in_the_local_frame():
    # a horizontal pattern is sqrt(1 - x^2) of the local direction: zero along
    # the world +x departure, one once the endpoint is turned 90 degrees in yaw
    rx = [make_receiver(torch.ones(3))]
    plain = path_api.pack_synthetic_arrays(
        _centre(), frequency_hz=1e9, transmitters=[make_transmitter(torch.zeros(3), pattern="horizontal")],
        receivers=rx)
    turned = path_api.pack_synthetic_arrays(
        _centre(), frequency_hz=1e9,
        transmitters=[make_transmitter(torch.zeros(3), orientation=[math.pi / 2, 0.0, 0.0], pattern="horizontal")],
        receivers=rx)
    torch.testing.assert_close(plain.a, torch.zeros_like(plain.a))
    torch.testing.assert_close(turned.a, torch.ones_like(turned.a), atol=1e-6, rtol=1e-6)


def test_receiver_steering_uses_the_arrival_source_direction_and_conjugate_pattern():
    custom = AntennaPattern("custom", custom=lambda d: torch.complex(d[..., 0], d[..., 1]))
    rx = make_receiver(torch.ones(3), element_positions=_ula(2, 0.5, axis=1), pattern=custom)
    out = path_api.pack_synthetic_arrays(_centre(theta_r=math.pi / 2, phi_r=math.pi / 2), frequency_hz=299_792_458.0,
                                         transmitters=[make_transmitter(torch.zeros(3))], receivers=[rx])
    # arrival source direction +y: steering -j, +j; the pattern (x + j y) = j,
    # conjugated -j
    want = torch.tensor([-1.0j, 1.0j], dtype=torch.complex64) * (-1.0j)
    torch.testing.assert_close(out.a[0, :, 0, 0, 0, 0], want, atol=1e-6, rtol=1e-6)


def test_grid_receivers_share_their_array():
    grid = make_receiver_grid(origin=[0, 0, 0], x_axis=[1, 0, 0], y_axis=[0, 1, 0], shape=(1, 2), spacing=(1, 1),
                              element_positions=_ula(3, 0.5))
    centre = _centre()
    two = replace(centre, **{name: torch.cat([getattr(centre, name)] * 2) for name in (
        "a", "tau", "theta_t", "phi_t", "theta_r", "phi_r", "valid", "interaction_type", "primitive_id",
        "material_id", "position", "normal", "num_paths", "field_xyz", "field_direction")})
    out = path_api.pack_synthetic_arrays(two, frequency_hz=1e9, transmitters=[make_transmitter(torch.zeros(3))],
                                         receivers=[grid])
    assert out.a.shape == (2, 3, 1, 1, 1, 1)
    torch.testing.assert_close(out.a[0], out.a[1])


def test_endpoint_weights_combine_like_the_reference_law():
    g = torch.Generator().manual_seed(3)
    h = torch.complex(torch.randn((2, 3, 2, 4, 5), generator=g), torch.randn((2, 3, 2, 4, 5), generator=g))
    tx = torch.complex(torch.randn((2, 4), generator=g), torch.randn((2, 4), generator=g))
    rx = torch.complex(torch.randn((2, 3), generator=g), torch.randn((2, 3), generator=g))
    got = path_api.apply_endpoint_weights(h, tx_weights=tx, rx_weights=rx)
    want = torch.einsum("ratbk,tb,ra->rtk", h, tx, rx.conj())
    torch.testing.assert_close(got, want, rtol=1e-5, atol=1e-5)
    with pytest.raises(ValueError):
        path_api.apply_endpoint_weights(h, tx_weights=tx[:, :3], rx_weights=rx)


def test_array_preflight_fails_before_any_device_work():
    mixed = Scene(structures=[], endpoints=[
        make_transmitter(torch.zeros(3), element_positions=torch.zeros((1, 3))),
        make_transmitter(torch.ones(3), element_positions=_ula(2, 0.5)),
        make_receiver(torch.tensor([0.0, 2.0, 0.0]))])
    with pytest.raises(ValueError, match="same antenna count"):
        path_api.solve(mixed, Config(components={"los"}), reference_frequency_hz=1e9)
    for synthetic in (True, False):
        partial = Scene(structures=[], endpoints=[
            make_transmitter(torch.zeros(3), element_positions=_ula(2, 0.5), synthetic_array=synthetic,
                             weights=torch.ones(2, dtype=torch.complex64)),
            make_transmitter(torch.ones(3), element_positions=_ula(2, 0.5), synthetic_array=synthetic),
            make_receiver(torch.tensor([0.0, 2.0, 0.0]))])
        with pytest.raises(ValueError, match="precoding must be configured on every"):
            path_api.solve(partial, Config(components={"los"}), reference_frequency_hz=1e9)
    explicit_grid = Scene(structures=[], endpoints=[
        make_transmitter(torch.zeros(3), element_positions=_ula(2, 0.5), synthetic_array=False),
        make_receiver_grid(origin=[0, 0, 0], x_axis=[1, 0, 0], y_axis=[0, 1, 0], shape=(1, 2), spacing=(1, 1))])
    with pytest.raises(ValueError, match="point receivers"):
        path_api.solve(explicit_grid, Config(components={"los"}), reference_frequency_hz=1e9)


def test_deterministic_solver_refuses_array_endpoints():
    from witwin_channel_b200 import deterministic

    for kw, match in ((dict(element_positions=_ula(2, 0.1)), "antenna arrays"),
                      (dict(pattern="vertical"), "directional antenna patterns"),
                      (dict(weights=torch.ones(1, dtype=torch.complex64)), "precoding or combining")):
        scene = Scene(structures=[], endpoints=[make_transmitter(torch.zeros(3), **kw),
                                                make_receiver(torch.tensor([1.0, 0.0, 0.0]))])
        with pytest.raises(ValueError, match=match):
            deterministic.solve(scene, deterministic.Config(components={"los"}), reference_frequency_hz=1e9)


def test_orientation_turns_the_polarization_and_the_elements():
    tx = make_transmitter(torch.zeros(3), polarization=[0.0, 0.0, 2.0], orientation=[0.0, math.pi / 2, 0.0],
                          element_positions=_ula(2, 1.0))
    torch.testing.assert_close(tx.polarization, torch.tensor([1.0, 0.0, 0.0]), atol=1e-6, rtol=0)
    world = tx.element_world_positions(torch.tensor([1.0, 2.0, 3.0]))
    torch.testing.assert_close(world, torch.tensor([[1.0, 2.0, 3.5], [1.0, 2.0, 2.5]]), atol=1e-6, rtol=0)
    default = make_transmitter(torch.zeros(3), pattern="horizontal")
    assert default.polarization.tolist() == [1.0, 0.0, 0.0]
