"""Path solver on the GPU: LoS closed form, the per-pair packing of the
native rows against the deterministic path table, and the CFR view against
a direct sum."""

from __future__ import annotations

import math

import numpy as np
import pytest
import torch

from tests import scenes
from witwin_channel_b200 import Config as DetConfig
from witwin_channel_b200 import solve as det_solve
from witwin_channel_b200.path import Config, InteractionType, PathResult, RaggedPathSoA, solve
from witwin_channel_b200.scene import Scene, make_receiver, make_transmitter

pytestmark = pytest.mark.gpu
C0 = 299_792_458.0


def _free_space_scene() -> Scene:
    return Scene(structures=[], endpoints=[
        make_transmitter(torch.tensor([0.0, 0.0, 0.0]), power_w=2.0),
        make_transmitter(torch.tensor([0.0, 2.0, 0.0]), power_w=0.5),
        make_receiver(torch.tensor([3.0, 4.0, 0.0])),
        make_receiver(torch.tensor([6.0, 8.0, 0.0])),
    ])


def test_los_shapes_lengths_angles_and_amplitude():
    f = 3.0e9
    result = solve(_free_space_scene(), Config(max_depth=0, components={"los"}), reference_frequency_hz=f)
    assert result.a.shape == (2, 1, 2, 1, 1, 1)
    assert torch.all(result.num_paths == 1)
    assert result.metadata["schema"] == "PathResult"
    tx = torch.tensor([[0.0, 0.0, 0.0], [0.0, 2.0, 0.0]], dtype=torch.float64)
    rx = torch.tensor([[3.0, 4.0, 0.0], [6.0, 8.0, 0.0]], dtype=torch.float64)
    for r in range(2):
        for t in range(2):
            d = float(torch.linalg.vector_norm(rx[r] - tx[t]))
            tau = float(result.tau[r, 0, t, 0, 0])
            assert abs(tau * C0 - d) <= 1e-5 * d
            assert abs(float(result.path_length_m[r, 0, t, 0, 0]) - d) <= 1e-5 * d
            # unit excitation: |a| = lambda / (4 pi d), vertical polarisations, horizontal link
            amp = abs(complex(result.a[r, 0, t, 0, 0, 0]))
            assert abs(amp - C0 / f / (4 * math.pi * d)) <= 1e-5 * amp
            v = rx[r] - tx[t]
            assert abs(float(result.theta_t[r, 0, t, 0, 0]) - math.pi / 2) < 1e-6
            assert abs(float(result.phi_t[r, 0, t, 0, 0]) - math.atan2(float(v[1]), float(v[0]))) < 1e-6
            assert abs(float(result.phi_r[r, 0, t, 0, 0]) - math.atan2(-float(v[1]), -float(v[0]))) < 1e-6


def test_paths_match_the_deterministic_table_per_pair():
    scene, freq = scenes.small_city()
    comps = {"los", "reflection", "diffraction", "transmission"}
    res = solve(scene, Config(max_depth=2, components=comps), reference_frequency_hz=freq)
    table = det_solve(scene, DetConfig(max_depth=2, components=comps, export_paths=True),
                      reference_frequency_hz=freq).paths
    valid = res.valid.cpu()
    assert int(valid.sum()) == int(table.tx_id.shape[0]) > 0
    # the table is in canonical (rx, tx) order: the packed result in pair order holds the same records
    a = res.a[..., 0][res.valid].cpu()
    np.testing.assert_allclose(a.numpy(), table.coefficient.cpu().numpy(), rtol=0, atol=0)
    np.testing.assert_allclose(res.tau[res.valid].cpu().numpy(), table.delay_s.cpu().numpy(), rtol=0, atol=0)
    rx_id = res.rx_id[res.valid].cpu()
    tx_id = res.tx_id[res.valid].cpu()
    assert torch.equal(rx_id, table.rx_id.cpu().to(torch.int32))
    assert torch.equal(tx_id, table.tx_id.cpu().to(torch.int32))
    # interaction types follow the component of each record
    types = res.interaction_type[res.valid].cpu()
    cid = table.component_id.cpu()
    depth = table.depth.cpu()
    want = {0: 0, 1: int(InteractionType.REFLECTION), 2: int(InteractionType.DIFFRACTION),
            5: int(InteractionType.TRANSMISSION)}
    for i in range(types.shape[0]):
        row = [want[int(cid[i])] if k < int(depth[i]) else 0 for k in range(types.shape[1])]
        assert types[i].tolist() == row
    # diffraction records name their edge in the first object slot
    diff = cid == 2
    if bool(diff.any()):
        assert torch.equal(res.primitive_id[..., 0][res.valid].cpu()[diff], table.edge_id.cpu()[diff].to(torch.int32))
    pos = res.position[res.valid].cpu()
    np.testing.assert_allclose(pos.numpy(), table.interaction_positions.cpu().numpy(), rtol=0, atol=0)
    xyz = res.field_xyz[res.valid].cpu()
    np.testing.assert_allclose(xyz.numpy(), table.field_xyz.cpu().numpy(), rtol=0, atol=0)
    # per-pair counts
    counts = torch.zeros(res.num_paths.shape, dtype=torch.int32)
    for r, t in zip(table.rx_id.cpu().tolist(), table.tx_id.cpu().tolist()):
        counts[r, 0, t, 0] += 1
    assert torch.equal(counts, res.num_paths.cpu())


def test_per_pair_limit_keeps_the_first_canonical_paths():
    scene, freq = scenes.small_city()
    comps = {"los", "reflection"}
    full = solve(scene, Config(max_depth=2, components=comps), reference_frequency_hz=freq)
    cut = solve(scene, Config(max_depth=2, components=comps, max_paths=2), reference_frequency_hz=freq)
    assert int(cut.num_paths.max()) <= 2
    assert int(cut.valid.sum()) > 0
    assert torch.all(cut.num_paths == torch.clamp(full.num_paths, max=2)) or int(cut.valid.sum()) <= int(full.valid.sum())


def _signal_result(device) -> PathResult:
    field = torch.tensor([[1.0 + 0.0j], [0.0 + 2.0j]], dtype=torch.complex64)
    types = torch.tensor([[int(InteractionType.REFLECTION)], [int(InteractionType.DIFFRACTION)]], dtype=torch.int32)
    ragged = RaggedPathSoA.from_flat(
        num_rx=1, num_rx_ant=1, num_tx=1, num_tx_ant=1, rx_id=torch.zeros(2, dtype=torch.int32),
        tx_id=torch.zeros(2, dtype=torch.int32), field=field, delay_s=torch.tensor([1.0e-9, 3.0e-9]),
        theta_t=torch.zeros(2), phi_t=torch.zeros(2), theta_r=torch.zeros(2), phi_r=torch.zeros(2),
        interaction_type=types, primitive_id=torch.tensor([[3], [7]], dtype=torch.int32),
        material_id=torch.tensor([[1], [2]], dtype=torch.int32), position=torch.zeros((2, 1, 3)),
        normal=torch.zeros((2, 1, 3)))
    ragged = RaggedPathSoA(**{k: (getattr(ragged, k).to(device) if isinstance(getattr(ragged, k), torch.Tensor)
                                  else getattr(ragged, k)) for k in RaggedPathSoA.__dataclass_fields__})
    return PathResult.from_ragged(ragged)


def test_cfr_matches_the_direct_sum():
    result = _signal_result(torch.device("cuda"))
    cfr = result.cfr(torch.tensor([0.0, 125.0e6]))
    assert cfr.shape == (1, 1, 1, 1, 1, 2)
    want0 = 1.0 + 2.0j
    want1 = 1.0 + 2.0j * complex(np.exp(-2.0j * math.pi * 0.25))
    assert abs(complex(cfr[..., 0].item()) - want0) <= 1e-6
    assert abs(complex(cfr[..., 1].item()) - want1) <= 1e-5


def test_cfr_of_a_solved_city_matches_the_direct_sum():
    scene, freq = scenes.small_city()
    res = solve(scene, Config(max_depth=2, components={"los", "reflection", "diffraction"}),
                reference_frequency_hz=freq)
    fr = (torch.arange(64, dtype=torch.float64) - 32) * 1.5e6
    got = res.cfr(fr).cpu().numpy()
    a = res.a[..., 0].cpu().numpy().astype(np.complex128)
    tau = res.tau.cpu().numpy().astype(np.float64)
    valid = res.valid.cpu().numpy()
    tmin = np.where(valid, tau, np.inf).min(axis=-1, keepdims=True)
    tmin = np.where(np.isfinite(tmin), tmin, 0.0)
    t = np.where(valid, tau - tmin, 0.0)
    want = (np.where(valid, a, 0)[..., None] * np.exp(-2j * np.pi * t[..., None] * fr.numpy())).sum(axis=-2)
    scale = np.abs(np.where(valid, a, 0)).sum(axis=-1, keepdims=True)
    assert np.all(np.abs(got[..., 0, :] - want) <= 1e-4 * scale + 1e-12)
    bf = res.beamform(tx_weights=torch.ones((res.num_tx, 1), dtype=torch.complex64),
                      rx_weights=torch.ones((res.num_rx, 1), dtype=torch.complex64))
    np.testing.assert_allclose(bf.cfr(fr).cpu().numpy()[:, :, 0, :], got[:, 0, :, 0, 0, :], rtol=0, atol=1e-6)
