"""Field operators through the C ABI against closed forms and the FP64 oracle.

Closed forms restate tests/kernels/test_field_transport.py:13-175 of the
reference (free-space phase/power contract, rotation invariance, lossy slab
reflection); the random cases compare with oracle/em.py (the complex128
mirror of tests/ad/_reference_fields.py)."""

from __future__ import annotations

import cmath
import math

import numpy as np
import pytest
import torch

from oracle import em
from witwin_channel_b200 import _native
from witwin_channel_b200.compiler import MaterialTables

pytestmark = pytest.mark.gpu
DEV = "cuda"


def _alloc(n, *shape, complex_=False):
    if complex_:
        return torch.zeros((n, *shape), dtype=torch.complex64, device=DEV)
    return torch.zeros((n, *shape), dtype=torch.float32, device=DEV)


def _free_space(source, target, power, tx_pol, rx_pol, freq):
    n = source.shape[0]
    out = dict(field_vector=_alloc(n, 3, complex_=True), coefficient=_alloc(n, complex_=True),
               path_field=_alloc(n, complex_=True), path_gain=_alloc(n), path_length=_alloc(n), delay=_alloc(n),
               direction=_alloc(n, 3))
    lib = _native.load()
    _native.check(lib.wcb_field_free_space(n, *(t.data_ptr() for t in (source, target, power, tx_pol, rx_pol)), freq,
                                           *(out[k].data_ptr() for k in out), _native.stream_handle()), "free_space")
    torch.cuda.synchronize()
    return out


def _reflection(source, target, pos, nrm, power, tx_pol, rx_pol, eps, sig, mu, gain, th, freq):
    n, d = pos.shape[0], pos.shape[1]
    out = dict(field_vector=_alloc(n, 3, complex_=True), coefficient=_alloc(n, complex_=True),
               path_field=_alloc(n, complex_=True), path_gain=_alloc(n), path_length=_alloc(n), delay=_alloc(n),
               direction=_alloc(n, 3))
    lib = _native.load()
    args = (source, target, pos, nrm, power, tx_pol, rx_pol, eps, sig, mu, gain, th)
    _native.check(lib.wcb_field_reflection_sequence(n, d, *(t.contiguous().data_ptr() for t in args), freq,
                                                    *(out[k].data_ptr() for k in out), _native.stream_handle()),
                  "reflection")
    torch.cuda.synchronize()
    return out


def t32(x):
    return torch.tensor(np.asarray(x), dtype=torch.float32, device=DEV)


def test_free_space_matches_analytic_phase_and_power_contract():
    freq, dist = 3.0e9, 10.0
    s = t32([[0.0, 0.0, 0.0]])
    t = t32([[dist, 0.0, 0.0]])
    pol = t32([[0.0, 0.0, 1.0]])
    unit = _free_space(s, t, t32([1.0]), pol, pol, freq)
    powered = _free_space(s, t, t32([4.0]), pol, pol, freq)
    lam = 299792458.0 / freq
    expected = lam / (4 * math.pi * dist) * cmath.exp(-1j * 2 * math.pi * dist / lam)
    et = torch.tensor([expected], dtype=torch.complex64, device=DEV)
    torch.testing.assert_close(unit["coefficient"], et, rtol=1e-4, atol=1e-8)
    assert torch.angle(unit["coefficient"] / et).abs().item() <= 1e-3
    torch.testing.assert_close(powered["path_field"], 2.0 * unit["path_field"])
    torch.testing.assert_close(powered["path_gain"], 4.0 * unit["path_gain"])
    torch.testing.assert_close(unit["field_vector"][:, 2], unit["coefficient"])
    torch.testing.assert_close(unit["field_vector"][:, :2], torch.zeros_like(unit["field_vector"][:, :2]))


def test_free_space_rotation_invariance():
    s = t32([[0.0, 0.0, 0.0]])
    t = t32([[3.0, 4.0, 1.0]])
    pz = t32([[0.0, 0.0, 1.0]])
    rot = t32([[0.0, -1.0, 0.0], [1.0, 0.0, 0.0], [0.0, 0.0, 1.0]])
    base = _free_space(s, t, t32([1.0]), pz, pz, 28e9)
    rotd = _free_space(s @ rot.T, (t @ rot.T).contiguous(), t32([1.0]), (pz @ rot.T).contiguous(),
                       (pz @ rot.T).contiguous(), 28e9)
    torch.testing.assert_close(rotd["coefficient"], base["coefficient"])
    torch.testing.assert_close(rotd["field_vector"], base["field_vector"] @ rot.T.to(torch.complex64))


def _slab(eps_r, sigma_e, mu_r, gain, thickness, frequency):
    eps0 = 8.8541878128e-12
    omega = 2 * math.pi * frequency
    lam = 299792458.0 / frequency
    eta = complex(eps_r, -sigma_e / (omega * eps0))
    root = cmath.sqrt(mu_r * eta)
    inter = (mu_r - root) / (mu_r + root)
    q = 2 * math.pi * thickness / lam * root
    ph = cmath.exp(-2j * q)
    return gain * inter * (1 - ph) / (1 - inter * inter * ph)


def test_lossy_slab_reflection_matches_complex_reference():
    f = 3.5e9
    out = _reflection(t32([[0.0, 0.0, 1.0]]), t32([[0.0, 0.0, 2.0]]), t32([[[0.0, 0.0, 0.0]]]),
                      t32([[[0.0, 0.0, 1.0]]]), t32([1.0]), t32([[1.0, 0.0, 0.0]]), t32([[1.0, 0.0, 0.0]]),
                      t32([[4.0]]), t32([[0.025]]), t32([[1.0]]), t32([[0.8]]), t32([[0.12]]), f)
    L = 3.0
    lam = 299792458.0 / f
    expected = lam / (4 * math.pi * L) * cmath.exp(-2j * math.pi * L / lam) * _slab(4.0, 0.025, 1.0, 0.8, 0.12, f)
    et = torch.tensor([expected], dtype=torch.complex64, device=DEV)
    torch.testing.assert_close(out["coefficient"], et, rtol=1e-4, atol=1e-8)
    assert torch.angle(out["coefficient"] / et).abs().item() <= 1e-3


def test_reflection_sequence_random_matches_oracle():
    rng = np.random.default_rng(5)
    n, d = 64, 3
    src = rng.uniform(-5, 5, (n, 3))
    tgt = rng.uniform(-5, 5, (n, 3)) + 20.0
    pos = rng.uniform(-3, 3, (n, d, 3)) + np.linspace(2, 18, d)[None, :, None]
    nrm = rng.normal(size=(n, d, 3))
    nrm /= np.linalg.norm(nrm, axis=-1, keepdims=True)
    tp = rng.normal(size=(n, 3))
    rp = rng.normal(size=(n, 3))
    eps = rng.uniform(2, 8, (n, d))
    sig = rng.uniform(0, 0.5, (n, d))
    mu = np.ones((n, d))
    gain = rng.uniform(0.5, 1.0, (n, d))
    th = rng.uniform(0.05, 0.4, (n, d))
    P = rng.uniform(0.5, 2.0, n)
    f = 28e9
    arrs = [np.asarray(a, dtype=np.float32).astype(np.float64) for a in (src, tgt, pos, nrm, P, tp, rp, eps, sig, mu, gain, th)]
    ref = em.reflection_sequence(*arrs, f)
    got = _reflection(*(t32(a) for a in arrs), f)
    _check_field(got, ref)


def _check_field(got, ref):
    """Field vector within 1e-3 relative of its norm (0.01 dB, 1e-3 rad);
    the projected coefficient to the same absolute bound (a near-orthogonal
    receiver polarization cancels the projection itself)."""
    fv = got["field_vector"].cpu().numpy().astype(np.complex128)
    rv = ref["field_vector"]
    scale = np.linalg.norm(rv, axis=-1)
    assert np.all(np.linalg.norm(fv - rv, axis=-1) <= 1e-3 * scale)
    gc = got["coefficient"].cpu().numpy().astype(np.complex128)
    assert np.all(np.abs(gc - ref["coefficient"]) <= 1e-3 * scale)


def test_transmission_sequence_random_matches_oracle():
    rng = np.random.default_rng(9)
    n, d = 48, 3
    f = 28e9
    src = rng.uniform(-1, 1, (n, 3))
    tgt = rng.uniform(-1, 1, (n, 3)) + np.array([12.0, 0.0, 0.0])
    nrm = rng.normal(size=(n, d, 3)) * 0.2 + np.array([1.0, 0.0, 0.0])
    counts = rng.integers(1, d + 1, n)
    mids = rng.integers(0, 2, (n, d))
    tp = rng.normal(size=(n, 3))
    rp = rng.normal(size=(n, 3))
    P = rng.uniform(0.5, 2.0, n)
    layers = [
        (np.array([0.006, 0.006]), np.array([6.27, 6.27]), np.array([0.2287, 0.2287]), np.array([1.0, 1.0])),
        (np.array([0.1]), np.array([4.0]), np.array([0.02]), np.array([1.0])),
    ]
    arrs = [np.asarray(a, dtype=np.float32).astype(np.float64) for a in (src, tgt, nrm, P, tp, rp)]
    ref = em.transmission_sequence(arrs[0], arrs[1], arrs[2], mids, counts, arrs[3], arrs[4], arrs[5], layers, f)
    mt = MaterialTables(
        eps_r=t32([[6.27, 4.0]]), sigma_e=t32([[0.2287, 0.02]]), mu_r=t32([[1.0, 1.0]]), gain=t32([[1.0, 1.0]]),
        thickness=t32([[0.006, 0.1]]), volumetric=torch.zeros(2, dtype=torch.int32, device=DEV),
        layer_offset=torch.tensor([0, 2], dtype=torch.int32, device=DEV),
        layer_count=torch.tensor([2, 1], dtype=torch.int32, device=DEV),
        layer_thickness=t32([[0.006, 0.006, 0.1]]), layer_eps_r=t32([[6.27, 6.27, 4.0]]),
        layer_sigma_e=t32([[0.2287, 0.2287, 0.02]]), layer_mu_r=t32([[1.0, 1.0, 1.0]]))
    out = dict(field_vector=_alloc(n, 3, complex_=True), coefficient=_alloc(n, complex_=True),
               path_field=_alloc(n, complex_=True), path_gain=_alloc(n), path_length=_alloc(n), delay=_alloc(n),
               direction=_alloc(n, 3))
    lib = _native.load()
    ms = mt.as_struct()
    args = [t32(arrs[0]), t32(arrs[1]), t32(arrs[2]),
            torch.tensor(mids, dtype=torch.int32, device=DEV), torch.tensor(counts, dtype=torch.int32, device=DEV),
            t32(arrs[3]), t32(arrs[4]), t32(arrs[5])]
    _native.check(lib.wcb_field_transmission_sequence(n, d, *(a.contiguous().data_ptr() for a in args),
                                                      _native.ctypes.byref(ms), f, *(out[k].data_ptr() for k in out),
                                                      _native.stream_handle()), "transmission")
    torch.cuda.synchronize()
    _check_field(out, ref)
