"""The standalone CUDA field operators against the reference's own complex128
field mirror (golden vectors in ``tests/golden/field_vectors.npz``, made by
``tests/golden/make_field_vectors.py`` from ``tests/ad/_reference_fields.py``).

Tolerance: FP32 fields with the k*d phase reduced in FP64; the field vector
within 1e-4 of its norm (1e-3 dB, 1e-4 rad) and the projected coefficient to
the same absolute bound (a near-orthogonal receiver polarization cancels the
projection itself)."""

from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest
import torch

from witwin_channel_b200.fields import (
    field_free_space,
    field_project_complex3,
    field_reflection_sequence,
    field_transmission_sequence,
)

pytestmark = pytest.mark.gpu
G = np.load(Path(__file__).resolve().parent / "golden" / "field_vectors.npz")
TOL = 1e-4
# electrically thick lossy layers (0.2 m concrete at 28 GHz: k_z*d ~ 270 rad)
# carry their phase through FP32 exponentials: ~k_z*d*2^-23 per layer
TOL_STACK = 1e-3


def f32(x):
    return torch.tensor(np.asarray(x), dtype=torch.float32, device="cuda").contiguous()


def test_free_space_golden():
    n = G["fs_source"].shape[0]
    for freq in (3.5e9, 28.0e9):
        idx = np.nonzero(G["fs_freq"] == freq)[0]
        out = field_free_space(f32(G["fs_source"][idx]), f32(G["fs_target"][idx]), f32(G["fs_power"][idx]),
                               f32(G["fs_tx_pol"][idx]), f32(G["fs_rx_pol"][idx]), frequency_hz=freq)
        fv = out["field_vector"].cpu().numpy().astype(np.complex128)
        rv = G["fs_field_vector"][idx]
        scale = np.linalg.norm(rv, axis=-1)
        assert np.all(np.linalg.norm(fv - rv, axis=-1) <= TOL * scale)
        pf = out["path_field"].cpu().numpy().astype(np.complex128)
        assert np.all(np.abs(pf - G["fs_path_field"][idx]) <= TOL * scale * np.sqrt(G["fs_power"][idx]))
        proj = field_project_complex3(out["field_vector"], out["direction"], f32(G["fs_rx_pol"][idx]))
        torch.testing.assert_close(proj["coefficient"], out["coefficient"], rtol=1e-5, atol=1e-12)
    assert n == 64


@pytest.mark.parametrize("depth", [1, 2, 3])
def test_reflection_sequence_golden(depth):
    p = f"rf{depth}_"
    out = field_reflection_sequence(*(f32(G[p + k]) for k in ("source", "target", "positions", "normals", "power",
                                                               "tx_pol", "rx_pol", "eps_r", "sigma_e", "mu_r", "gain",
                                                               "thickness")),
                                    frequency_hz=float(G[p + "freq"]))
    fv = out["field_vector"].cpu().numpy().astype(np.complex128)
    rv = G[p + "field_vector"]
    scale = np.linalg.norm(rv, axis=-1)
    assert np.all(np.linalg.norm(fv - rv, axis=-1) <= TOL * scale)
    pf = out["path_field"].cpu().numpy().astype(np.complex128)
    assert np.all(np.abs(pf - G[p + "path_field"]) <= TOL * scale * np.sqrt(G[p + "power"]))


def test_transmission_sequence_golden():
    n, depth = G["tr_normals"].shape[:2]
    valid = np.arange(depth)[None, :] < G["tr_count"][:, None]
    out = field_transmission_sequence(
        torch.ones(n, dtype=torch.bool, device="cuda"), f32(G["tr_source"]), f32(G["tr_target"]),
        torch.zeros((n, depth, 3), dtype=torch.float32, device="cuda"), f32(G["tr_normals"]),
        torch.tensor(G["tr_material"], dtype=torch.int32, device="cuda"),
        torch.tensor(valid, device="cuda"), f32(G["tr_power"]), f32(G["tr_tx_pol"]), f32(G["tr_rx_pol"]),
        torch.tensor(G["tr_layer_offset"], dtype=torch.int32, device="cuda"),
        torch.tensor(G["tr_layer_count"], dtype=torch.int32, device="cuda"), f32(G["tr_layer_thickness"]),
        f32(G["tr_layer_eps_r"]), f32(G["tr_layer_sigma_e"]), f32(G["tr_layer_mu_r"]),
        frequency_hz=float(G["tr_freq"]))
    fv = out["field_vector"].cpu().numpy().astype(np.complex128)
    rv = G["tr_field_vector"]
    scale = np.linalg.norm(rv, axis=-1)
    assert np.all(np.linalg.norm(fv - rv, axis=-1) <= TOL_STACK * scale)
    pf = out["path_field"].cpu().numpy().astype(np.complex128)
    assert np.all(np.abs(pf - G["tr_path_field"]) <= TOL_STACK * scale * np.sqrt(G["tr_power"]))


def test_transmission_masked_walls_and_invalid_paths():
    """A wall whose valid flag is False is skipped wherever it sits; an invalid path returns zeros."""
    n, depth = G["tr_normals"].shape[:2]
    valid = np.arange(depth)[None, :] < G["tr_count"][:, None]
    # move every row's walls to the back: same valid set, different slots
    shift = depth - G["tr_count"]
    normals = np.zeros_like(G["tr_normals"])
    mids = np.zeros_like(G["tr_material"])
    moved = np.zeros_like(valid)
    for i in range(n):
        c, s = int(G["tr_count"][i]), int(shift[i])
        normals[i, s:s + c] = G["tr_normals"][i, :c]
        mids[i, s:s + c] = G["tr_material"][i, :c]
        moved[i, s:s + c] = True
    path_valid = torch.ones(n, dtype=torch.bool, device="cuda")
    path_valid[3] = False
    args = lambda nrm, mid, vl: (  # noqa: E731
        path_valid, f32(G["tr_source"]), f32(G["tr_target"]), torch.zeros((n, depth, 3), device="cuda"), f32(nrm),
        torch.tensor(mid, dtype=torch.int32, device="cuda"), torch.tensor(vl, device="cuda"), f32(G["tr_power"]),
        f32(G["tr_tx_pol"]), f32(G["tr_rx_pol"]), torch.tensor(G["tr_layer_offset"], dtype=torch.int32, device="cuda"),
        torch.tensor(G["tr_layer_count"], dtype=torch.int32, device="cuda"), f32(G["tr_layer_thickness"]),
        f32(G["tr_layer_eps_r"]), f32(G["tr_layer_sigma_e"]), f32(G["tr_layer_mu_r"]))
    a = field_transmission_sequence(*args(G["tr_normals"], G["tr_material"], valid), frequency_hz=28e9)
    b = field_transmission_sequence(*args(normals, mids, moved), frequency_hz=28e9)
    torch.testing.assert_close(a["path_field"], b["path_field"], rtol=0, atol=0)
    assert float(a["path_gain"][3]) == 0.0


def test_validation_errors():
    x = f32(np.zeros((2, 3)))
    with pytest.raises(ValueError):
        field_free_space(x, x, f32([1.0, 1.0]), x, x, frequency_hz=-1.0)
    with pytest.raises(ValueError):
        field_free_space(x, f32(np.zeros((3, 3))), f32([1.0, 1.0]), x, x, frequency_hz=1e9)
    with pytest.raises(TypeError):
        field_free_space(x.double(), x, f32([1.0, 1.0]), x, x, frequency_hz=1e9)
