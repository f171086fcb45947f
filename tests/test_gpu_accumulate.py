"""Flat accumulation on the GPU: bit-exact against the reference's frozen
SHA-256 outputs (``tests/ad/test_deterministic_accum_ad.py:37-129``) and the
oracle, plus the adjoint (strict float64 gradcheck) and JVP/VJP duality."""

from __future__ import annotations

import hashlib
import json
from pathlib import Path

import numpy as np
import pytest
import torch

from oracle import accumulate as oacc
from witwin_channel_b200.kernels import (
    ACCUM_FIELDS,
    deterministic_accumulate_flat,
    deterministic_accumulate_flat_ad,
)

pytestmark = pytest.mark.gpu

REF = json.loads((Path(__file__).resolve().parent / "golden" / "reference_goldens.json").read_text())["accumulate_flat"]


def _fixture(dtype):
    g = torch.Generator(device="cpu").manual_seed(REF["seed"])
    n = len(REF["tx_id"])
    dev = torch.device("cuda")
    gain = (torch.rand((n,), generator=g, dtype=torch.float64) + 0.25).to(device=dev, dtype=dtype)
    real = torch.randn((n,), generator=g, dtype=torch.float64).to(device=dev, dtype=dtype)
    imag = torch.randn((n,), generator=g, dtype=torch.float64).to(device=dev, dtype=dtype)
    valid = torch.ones(n, dtype=torch.bool, device=dev)
    ids = [torch.tensor(REF[k], dtype=torch.int32, device=dev) for k in ("tx_id", "rx_id", "component_id")]
    return (valid, *ids, gain, real, imag)


def _sha(out):
    return hashlib.sha256(b"".join(out[k].detach().contiguous().cpu().numpy().tobytes()
                                   for k in ACCUM_FIELDS)).hexdigest()


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
@pytest.mark.parametrize("coherent", [True, False])
def test_reproduces_reference_frozen_sha256(dtype, coherent):
    fx = _fixture(dtype)
    if dtype == torch.float32:
        out = deterministic_accumulate_flat(*fx, num_tx=REF["num_tx"], num_rx=REF["num_rx"], coherent=coherent)
    else:
        out = deterministic_accumulate_flat_ad(*fx, num_tx=REF["num_tx"], num_rx=REF["num_rx"], coherent=coherent)
    name = f"{'float32' if dtype == torch.float32 else 'float64'}_{'coherent' if coherent else 'incoherent'}"
    assert _sha(out) == REF["sha256"][name]


def _random_paths(n, num_tx, num_rx, dtype, seed):
    rng = np.random.default_rng(seed)
    valid = rng.random(n) < 0.95
    tx = rng.integers(-1, num_tx + 1, n).astype(np.int32)
    rx = rng.integers(-1, num_rx + 1, n).astype(np.int32)
    cid = rng.integers(-1, 9, n).astype(np.int32)
    gain = rng.random(n).astype(dtype)
    real = rng.normal(size=n).astype(dtype)
    imag = rng.normal(size=n).astype(dtype)
    return valid, tx, rx, cid, gain, real, imag


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("coherent,domain", [(True, 0), (False, 0), (True, 1), (False, 1)])
def test_bit_exact_against_oracle(dtype, coherent, domain):
    num_tx, num_rx = 3, 40
    host = _random_paths(4000, num_tx, num_rx, dtype, seed=int(coherent) * 2 + domain)
    want = oacc.accumulate_flat(*host, num_tx=num_tx, num_rx=num_rx, coherent=coherent,
                                scattering_coherent=bool(domain), dtype=dtype)
    dev = [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in host]
    out = deterministic_accumulate_flat_ad(*dev, num_tx=num_tx, num_rx=num_rx, coherent=coherent,
                                           scattering_combine_domain=domain)
    for k in ACCUM_FIELDS:
        assert np.array_equal(out[k].cpu().numpy(), want[k]), k


def test_empty_and_zero_cells():
    dev = torch.device("cuda")
    e_i = torch.empty(0, dtype=torch.int32, device=dev)
    e_f = torch.empty(0, dtype=torch.float32, device=dev)
    out = deterministic_accumulate_flat(torch.empty(0, dtype=torch.bool, device=dev), e_i, e_i, e_i, e_f, e_f, e_f,
                                        num_tx=2, num_rx=3, coherent=True)
    for k in ACCUM_FIELDS:
        assert bool((out[k] == 0).all())
    out = deterministic_accumulate_flat(torch.empty(0, dtype=torch.bool, device=dev), e_i, e_i, e_i, e_f, e_f, e_f,
                                        num_tx=0, num_rx=3, coherent=False)
    assert tuple(out["component_power"].shape) == (6, 0, 3)


def test_validation_errors_match_reference():
    fx = list(_fixture(torch.float32))
    with pytest.raises(ValueError):
        deterministic_accumulate_flat(*fx, num_tx=2, num_rx=2, coherent=True, scattering_combine_domain=2)
    bad = list(fx)
    bad[4] = bad[4].double()
    with pytest.raises(TypeError):
        deterministic_accumulate_flat(*bad, num_tx=2, num_rx=2, coherent=True)
    bad = list(fx)
    bad[1] = bad[1][:-1]
    with pytest.raises(ValueError):
        deterministic_accumulate_flat(*bad, num_tx=2, num_rx=2, coherent=True)
    with pytest.raises(ValueError):
        deterministic_accumulate_flat(*fx, num_tx=-1, num_rx=2, coherent=True)


@pytest.mark.parametrize("coherent", [True, False])
@pytest.mark.parametrize("domain", [0, 1])
def test_gradcheck_strict_float64(coherent, domain):
    valid, tx, rx, cid, gain, real, imag = _fixture(torch.float64)

    def func(g, r, i):
        out = deterministic_accumulate_flat_ad(valid, tx, rx, cid, g, r, i, num_tx=2, num_rx=2, coherent=coherent,
                                               scattering_combine_domain=domain)
        return tuple(out[k] for k in ACCUM_FIELDS)

    leaves = tuple(v.clone().requires_grad_(True) for v in (gain, real, imag))
    assert torch.autograd.gradcheck(func, leaves, eps=1e-6, atol=1e-9, rtol=1e-5, nondet_tol=1e-10)
    assert torch.autograd.gradcheck(func, leaves, eps=1e-6, atol=1e-9, rtol=1e-5, nondet_tol=1e-10,
                                    check_forward_ad=True, check_backward_ad=False, check_undefined_grad=False,
                                    check_batched_grad=False)


@pytest.mark.parametrize("coherent", [True, False])
def test_jvp_vjp_duality(coherent):
    valid, tx, rx, cid, gain, real, imag = _fixture(torch.float64)
    g = torch.Generator(device="cpu").manual_seed(11)
    tangents = tuple(torch.randn(v.shape, generator=g, dtype=torch.float64).cuda() for v in (gain, real, imag))
    leaves = tuple(v.clone().requires_grad_(True) for v in (gain, real, imag))
    out = deterministic_accumulate_flat_ad(valid, tx, rx, cid, *leaves, num_tx=2, num_rx=2, coherent=coherent)
    cots = {k: torch.randn(out[k].shape, generator=g, dtype=torch.float64).cuda() for k in ACCUM_FIELDS}
    sum((cots[k] * out[k]).sum() for k in ACCUM_FIELDS).backward()
    vjp = sum((leaf.grad * t).sum() for leaf, t in zip(leaves, tangents))
    with torch.autograd.forward_ad.dual_level():
        duals = tuple(torch.autograd.forward_ad.make_dual(v.clone(), t) for v, t in zip((gain, real, imag), tangents))
        dout = deterministic_accumulate_flat_ad(valid, tx, rx, cid, *duals, num_tx=2, num_rx=2, coherent=coherent)
        jvp = sum((cots[k] * torch.autograd.forward_ad.unpack_dual(dout[k]).tangent).sum() for k in ACCUM_FIELDS)
    torch.testing.assert_close(jvp, vjp, rtol=1e-10, atol=1e-12)
