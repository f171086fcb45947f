"""Generate tests/golden/field_vectors.npz from the reference's complex128 field mirror.

The reference ships pure-torch complex128 mirrors of its field kernels in
``tests/ad/_reference_fields.py`` (free space, slab reflection chains, the
thin-sheet transmission stack).  This script imports that file from a
checkout of witwin-ai/witwin-channel, evaluates it on seeded random inputs and
stores inputs and outputs, so the oracle and the CUDA field operators can be
checked against the reference without the reference present.

Usage: python tests/golden/make_field_vectors.py [path/to/witwin-channel]
"""

from __future__ import annotations

import importlib.util
import sys
from pathlib import Path

import numpy as np
import torch

OUT = Path(__file__).with_name("field_vectors.npz")


def _load_mirror(root: Path):
    path = root / "tests" / "ad" / "_reference_fields.py"
    spec = importlib.util.spec_from_file_location("_reference_fields", path)
    mod = importlib.util.module_from_spec(spec)
    sys.modules["_reference_fields"] = mod
    spec.loader.exec_module(mod)
    return mod


def _f32(x):
    """Inputs representable in float32, the CUDA operators' input type."""
    return np.asarray(x, dtype=np.float32).astype(np.float64)


def _unit(rng, n):
    v = rng.normal(size=(n, 3))
    return _f32(v / np.linalg.norm(v, axis=1, keepdims=True))


def _t(x):
    return torch.as_tensor(np.asarray(x), dtype=torch.float64)


def _np(out):
    return {k: v.detach().numpy() for k, v in out.items()}


def main(root: Path) -> None:
    ref = _load_mirror(root)
    rng = np.random.default_rng(0)
    data = {}

    # free space: 64 cases, two carriers
    n = 64
    src = _f32(rng.uniform(-50, 50, size=(n, 3)))
    tgt = _f32(src + _unit(rng, n) * rng.uniform(0.5, 400.0, size=(n, 1)))
    pw = _f32(rng.uniform(0.1, 4.0, size=n))
    tpol, rpol = _unit(rng, n), _unit(rng, n)
    freq = np.where(np.arange(n) % 2 == 0, 3.5e9, 28.0e9)
    data.update(fs_source=src, fs_target=tgt, fs_power=pw, fs_tx_pol=tpol, fs_rx_pol=rpol, fs_freq=freq)
    for key in ("field_vector", "coefficient", "path_field", "path_gain"):
        data[f"fs_{key}"] = np.stack([
            _np(ref.free_space_reference(_t(src[i:i + 1]), _t(tgt[i:i + 1]), _t(pw[i:i + 1]), _t(tpol[i:i + 1]),
                                         _t(rpol[i:i + 1]), _t(freq[i])))[key][0] for i in range(n)])

    # specular chains of depth 1..3 at 28 GHz: random bounce points and normals
    for depth in (1, 2, 3):
        n = 32
        src = _f32(rng.uniform(-30, 30, size=(n, 3)))
        pos = _f32(src[:, None, :] + np.cumsum(rng.uniform(-20, 20, size=(n, depth, 3)), axis=1))
        tgt = _f32(pos[:, -1] + rng.uniform(-20, 20, size=(n, 3)))
        nrm = rng.normal(size=(n, depth, 3))
        nrm = _f32(nrm / np.linalg.norm(nrm, axis=2, keepdims=True))
        eps = _f32(rng.uniform(1.5, 9.0, size=(n, depth)))
        sig = _f32(rng.uniform(0.0, 1.0, size=(n, depth)))
        mu = np.ones((n, depth))
        gain = _f32(rng.uniform(0.5, 1.0, size=(n, depth)))
        th = _f32(rng.uniform(0.05, 0.4, size=(n, depth)))
        pw = _f32(rng.uniform(0.1, 4.0, size=n))
        tpol, rpol = _unit(rng, n), _unit(rng, n)
        f = 28.0e9
        out = _np(ref.reflection_sequence_reference(_t(src), _t(tgt), _t(pos), _t(nrm), _t(pw), _t(tpol), _t(rpol),
                                                    _t(eps), _t(sig), _t(mu), _t(gain), _t(th), _t(f)))
        p = f"rf{depth}_"
        data.update({p + "source": src, p + "target": tgt, p + "positions": pos, p + "normals": nrm, p + "eps_r": eps,
                     p + "sigma_e": sig, p + "mu_r": mu, p + "gain": gain, p + "thickness": th, p + "power": pw,
                     p + "tx_pol": tpol, p + "rx_pol": rpol, p + "freq": np.float64(f)})
        for key in ("field_vector", "coefficient", "path_field", "path_gain"):
            data[p + key] = out[key]

    # thin-sheet transmission: up to 3 walls, materials with 1 or 2 layers
    n, depth = 32, 3
    layer_offset = np.array([0, 1, 3])
    layer_count = np.array([1, 2, 1])
    layer_th = _f32([0.2, 0.006, 0.006, 0.1])
    layer_eps = _f32([5.24, 6.27, 6.27, 3.0])
    layer_sig = _f32([0.626, 0.2287, 0.2287, 0.05])
    layer_mu = np.ones(4)
    src = _f32(rng.uniform(-30, 30, size=(n, 3)))
    tgt = _f32(src + _unit(rng, n) * rng.uniform(2.0, 200.0, size=(n, 1)))
    nrm = rng.normal(size=(n, depth, 3))
    nrm = _f32(nrm / np.linalg.norm(nrm, axis=2, keepdims=True))
    mids = rng.integers(0, 3, size=(n, depth))
    count = rng.integers(1, depth + 1, size=n)
    valid = np.arange(depth)[None, :] < count[:, None]
    pw = _f32(rng.uniform(0.1, 4.0, size=n))
    tpol, rpol = _unit(rng, n), _unit(rng, n)
    f = 28.0e9
    out = _np(ref.transmission_sequence_reference(
        _t(src), _t(tgt), _t(nrm), torch.as_tensor(mids), torch.as_tensor(valid), _t(pw), _t(tpol), _t(rpol),
        torch.as_tensor(layer_offset), torch.as_tensor(layer_count), _t(layer_th), _t(layer_eps), _t(layer_sig),
        _t(layer_mu), _t(f)))
    data.update(tr_source=src, tr_target=tgt, tr_normals=nrm, tr_material=mids, tr_count=count, tr_power=pw,
                tr_tx_pol=tpol, tr_rx_pol=rpol, tr_freq=np.float64(f), tr_layer_offset=layer_offset,
                tr_layer_count=layer_count, tr_layer_thickness=layer_th, tr_layer_eps_r=layer_eps,
                tr_layer_sigma_e=layer_sig, tr_layer_mu_r=layer_mu)
    for key in ("field_vector", "coefficient", "path_field", "path_gain"):
        data["tr_" + key] = out[key]

    np.savez_compressed(OUT, **data)
    print(f"wrote {OUT} ({OUT.stat().st_size} bytes, {len(data)} arrays)")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python make_field_vectors.py <path to the reference checkout>")
    main(Path(sys.argv[1]))
