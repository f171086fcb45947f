"""CFR of exported paths on the GPU against the FP64 restatement of the
reference's ``PathResult.cfr`` (``oracle/channel.py``).  Tolerance: 1e-4 of
the link's sum of |a_p| (FP32 accumulation; the phase is reduced in FP64 and
advanced by a renormalised rotation)."""

from __future__ import annotations

import numpy as np
import pytest
import torch

from oracle import channel as och
from tests import scenes as sc
from witwin_channel_b200 import Config, solve
from witwin_channel_b200.channel import cfr, cir, taps

pytestmark = pytest.mark.gpu


def _paths():
    scene, freq = sc.small_city(n_boxes=4, seed=7, grid=(8, 6))
    res = solve(scene, Config(components={"los", "reflection", "diffraction"}, max_depth=2, export_paths=True),
                reference_frequency_hz=freq)
    return res.paths, 1, 48


def _check(p, T, R, freqs, normalize):
    got = cfr(p, freqs, num_tx=T, num_rx=R, normalize_delays=normalize).cpu().numpy()
    a = (p.field_real.double() + 1j * p.field_imag.double()).cpu().numpy()
    want = och.cfr(p.tx_id.cpu(), p.rx_id.cpu(), p.delay_s.double().cpu(), a, np.asarray(freqs), T, R, normalize)
    scale = np.zeros((T, R))
    np.add.at(scale, (p.tx_id.cpu().numpy(), p.rx_id.cpu().numpy()), np.abs(a))
    err = np.abs(got - want).max(axis=-1)
    assert np.all(err <= 1e-4 * scale + 1e-30), (err / np.maximum(scale, 1e-300)).max()


@pytest.mark.parametrize("normalize", [True, False])
def test_cfr_1024_subcarriers_over_400_mhz(normalize):
    p, T, R = _paths()
    freqs = (np.arange(1024) - 512) * 390.625e3
    _check(p, T, R, freqs, normalize)


def test_cfr_non_uniform_grid_and_single_subcarrier():
    p, T, R = _paths()
    rng = np.random.default_rng(0)
    _check(p, T, R, np.sort(rng.uniform(-2e8, 2e8, 77)), True)
    _check(p, T, R, np.array([1.5e6]), True)


def test_cfr_at_zero_offset_is_the_coherent_sum():
    p, T, R = _paths()
    h0 = cfr(p, [0.0], num_tx=T, num_rx=R)[..., 0]
    a = torch.complex(p.field_real, p.field_imag)
    want = torch.zeros(T * R, dtype=torch.complex64, device=a.device)
    want.index_add_(0, (p.tx_id * R + p.rx_id).long(), a)
    torch.testing.assert_close(h0.reshape(-1), want, rtol=1e-5, atol=1e-12)


def test_cir_and_taps():
    p, T, R = _paths()
    a, tau = cir(p)
    assert float(tau.min()) == 0.0
    tp = taps(p, 400e6, 64, num_tx=T, num_rx=R)
    # the taps of a link sum to its coefficients that fall inside the window
    idx = torch.round(tau.double() * 400e6).long()
    keep = idx < 64
    want = torch.zeros(T * R, dtype=torch.complex64, device=a.device)
    want.index_add_(0, (p.tx_id * R + p.rx_id).long()[keep], a[keep])
    torch.testing.assert_close(tp.sum(-1).reshape(-1), want, rtol=1e-5, atol=1e-12)
