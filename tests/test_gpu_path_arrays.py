"""Antenna arrays on the path solver, on the GPU (reference ``path.py:1079-1486``;
the contract of the reference's ``tests/path/test_path_synthetic_arrays.py``).

Checked:

* explicit arrays trace every element: free-space delays are the exact
  element distances, and each element's rows on a two-wall scene equal a
  single-antenna solve with the endpoint moved to that element;
* synthetic arrays weight the centre paths by exp(+j k r . u) at each path's
  departure direction (restated here in numpy from the published angles);
* synthetic and explicit arrays agree in the far field;
* endpoint weights: the beamformed CFR equals the weighted raw CFR, the CIR
  sums to it and the taps sum to the zero-frequency CFR, and the raw result is
  left unchanged.
"""

from __future__ import annotations

import math

import numpy as np
import pytest
import torch

from tests import scenes
from witwin_channel_b200.path import Config, apply_endpoint_weights, solve
from witwin_channel_b200.scene import Scene, make_receiver, make_transmitter

pytestmark = pytest.mark.gpu
C0 = 299_792_458.0


def _ula(n, spacing, axis=0):
    positions = torch.zeros((n, 3))
    positions[:, axis] = (torch.arange(n, dtype=torch.float32) - 0.5 * (n - 1)) * spacing
    return positions


def test_explicit_array_traces_every_element_in_free_space():
    scene = Scene(structures=[], endpoints=[
        make_transmitter(torch.zeros(3), element_positions=_ula(2, 0.5), synthetic_array=False),
        make_receiver(torch.tensor([0.0, 2.0, 0.0]), element_positions=_ula(2, 0.5), synthetic_array=False)])
    result = solve(scene, Config(components={"los"}), reference_frequency_hz=1.0e9)
    assert result.a.shape == (1, 2, 1, 2, 1, 1)
    want = torch.tensor([[2.0, math.sqrt(4.25)], [math.sqrt(4.25), 2.0]], device=result.tau.device)
    torch.testing.assert_close(result.tau[0, :, 0, :, 0] * C0, want, rtol=1e-6, atol=1e-6)
    assert result.metadata["array_semantics"] == "explicit_per_element_topology"


def test_explicit_elements_equal_single_antenna_solves_on_two_walls():
    f = 3.5e9
    base = scenes.two_wall_scene()
    tx0, rx0 = base.transmitters[0], base.receivers[0]
    elements = _ula(3, 0.04, axis=2)
    scene = Scene(structures=base.structures, endpoints=[
        make_transmitter(tx0.position, element_positions=elements, synthetic_array=False),
        make_receiver(rx0.position)])
    cfg = Config(components={"los", "reflection"}, max_depth=2)
    result = solve(scene, cfg, reference_frequency_hz=f)
    assert result.a.shape[:4] == (1, 1, 1, 3)
    for k in range(3):
        single = Scene(structures=base.structures, endpoints=[
            make_transmitter(tx0.position + elements[k]), make_receiver(rx0.position)])
        one = solve(single, cfg, reference_frequency_hz=f)
        n = int(one.num_paths[0, 0, 0, 0])
        assert int(result.num_paths[0, 0, 0, k]) == n > 1
        torch.testing.assert_close(result.a[0, 0, 0, k, :n], one.a[0, 0, 0, 0, :n], rtol=0, atol=0)
        torch.testing.assert_close(result.tau[0, 0, 0, k, :n], one.tau[0, 0, 0, 0, :n], rtol=0, atol=0)


def test_synthetic_array_weights_each_path_by_its_departure_phase():
    f = 3.5e9
    base = scenes.two_wall_scene()
    tx0, rx0 = base.transmitters[0], base.receivers[0]
    elements = _ula(4, 0.03, axis=1)
    centre = solve(Scene(structures=base.structures, endpoints=[make_transmitter(tx0.position),
                                                                make_receiver(rx0.position)]),
                   Config(components={"los", "reflection"}, max_depth=2), reference_frequency_hz=f)
    scene = Scene(structures=base.structures, endpoints=[
        make_transmitter(tx0.position, element_positions=elements), make_receiver(rx0.position)])
    result = solve(scene, Config(components={"los", "reflection"}, max_depth=2), reference_frequency_hz=f)
    n = int(centre.num_paths[0, 0, 0, 0])
    assert n >= 3 and result.a.shape[3] == 4
    theta = centre.theta_t[0, 0, 0, 0, :n].double().cpu().numpy()
    phi = centre.phi_t[0, 0, 0, 0, :n].double().cpu().numpy()
    u = np.stack([np.sin(theta) * np.cos(phi), np.sin(theta) * np.sin(phi), np.cos(theta)], -1)
    k = 2.0 * math.pi * f / C0
    steer = np.exp(1j * k * (u @ elements.double().numpy().T))  # (path, element)
    a0 = centre.a[0, 0, 0, 0, :n, 0].cpu().numpy()
    got = result.a[0, 0, 0, :, :n, 0].cpu().numpy().T
    np.testing.assert_allclose(got, a0[:, None] * steer, rtol=2e-5, atol=1e-12)
    assert torch.equal(result.tau[0, 0, 0, 2, :n], centre.tau[0, 0, 0, 0, :n])


def test_synthetic_and_explicit_arrays_converge_in_the_far_field():
    elements = _ula(2, 0.01, axis=1)

    def run(synthetic):
        return solve(Scene(structures=[], endpoints=[
            make_transmitter(torch.zeros(3), element_positions=elements, synthetic_array=synthetic),
            make_receiver(torch.tensor([1000.0, 100.0, 0.0]))]), Config(components={"los"}),
            reference_frequency_hz=1.0e9)

    synthetic, explicit = run(True), run(False)
    torch.testing.assert_close(synthetic.a, explicit.a, rtol=2e-3, atol=1e-8)
    assert torch.unique(synthetic.tau).numel() == 1
    assert torch.unique(explicit.tau).numel() == 2


def test_endpoint_weights_beamform_cir_cfr_and_taps():
    tx_w = (torch.tensor([1.0, 0.5j], dtype=torch.complex64), torch.tensor([-0.25j, 1.0], dtype=torch.complex64))
    rx_w = (torch.tensor([1.0, -0.5j], dtype=torch.complex64), torch.tensor([0.25j, 0.75], dtype=torch.complex64))
    rx_elements = torch.zeros((2, 3))
    rx_elements[:, 1] = torch.tensor([-0.025, 0.025])
    scene = Scene(structures=[], endpoints=[
        make_transmitter(torch.tensor([0.0, float(i), 0.0]), element_positions=_ula(2, 0.05, axis=1), weights=tx_w[i])
        for i in range(2)] + [
        make_receiver(torch.tensor([20.0, float(i), 0.0]), element_positions=rx_elements, weights=rx_w[i])
        for i in range(2)])
    result = solve(scene, Config(components={"los"}), reference_frequency_hz=1.0e9)
    raw = result.a.clone()
    beamformed = result.beamform()
    freqs = torch.tensor([0.0, 1.0e6], device=result.a.device)
    raw_cfr = result.cfr(freqs, normalize_delays=False)
    want = apply_endpoint_weights(raw_cfr, tx_weights=torch.stack(tx_w).to(result.a.device),
                                  rx_weights=torch.stack(rx_w).to(result.a.device))
    torch.testing.assert_close(beamformed.cfr(freqs, normalize_delays=False), want)
    coefficient, tau = beamformed.cir(normalize_delays=False)
    assert coefficient.shape == (2, 2, 4, 1) and tau.shape == (2, 2, 4)
    torch.testing.assert_close(coefficient.sum(dim=2), want[..., 0])
    taps = beamformed.taps(1.0e9, 8, normalize_delays=True)
    torch.testing.assert_close(taps.sum(dim=-1), beamformed.cfr(torch.zeros(1, device=result.a.device))[..., 0])
    torch.testing.assert_close(result.a, raw)
