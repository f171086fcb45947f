"""Forward-mode AD (``ad_mode="jvp"``) of the deterministic solve.

The reference runs its dual companions inside the forward when
``ad_mode="jvp"`` (``witwin/channel/deterministic.py:733-742``): the scene
values are ``torch.autograd.forward_ad`` dual tensors and the outputs carry
the directional derivative.  Checked on the two-wall, wedge and thin-wall
scenes of the VJP tests:

* against central finite differences along the same direction of the
  oracle's FP64 fixed-topology re-evaluation (Richardson-extrapolated, steps
  1e-4 relative), within 1e-4 relative;
* against the VJP by duality, <v, J t> = <J^T v, t>, within 1e-5 relative
  (the output tangents are float32 like the outputs).
"""

from __future__ import annotations

import dataclasses

import numpy as np
import pytest
import torch
import torch.autograd.forward_ad as fwAD

from oracle import adjoint as oadj
from oracle import solve as osolve
from tests.test_gpu_vjp import thin_walls, two_wall, wedge
from witwin_channel_b200 import Config, solve

pytestmark = pytest.mark.gpu

CASES = [
    (two_wall, {"los", "reflection"}, 2, 3.0e9),
    (wedge, {"diffraction"}, 1, 3.0e9),
    (thin_walls, {"los", "transmission", "reflection"}, 2, 28.0e9),
]


def _materials(scene):
    mats = []
    for st in scene.structures:
        if all(st.material is not m for m in mats):
            mats.append(st.material)
    return mats


def _direction(scene, seed):
    """A random tangent for every differentiable scene value."""
    g = torch.Generator().manual_seed(seed)
    # coincident vertices of different structures (a merged shared edge) move
    # together: moving one copy alone would break the merge, a topology change
    shared: dict[tuple, torch.Tensor] = {}
    verts = []
    for st in scene.structures:
        tv = torch.randn(st.vertices.shape, generator=g, dtype=torch.float32)
        for v in range(st.vertices.shape[0]):
            key = tuple(round(float(x), 6) for x in st.vertices[v].detach())
            tv[v] = shared.setdefault(key, tv[v].clone())
        verts.append(tv)
    t = {"vertices": verts,
         "eps_r": [float(torch.randn((), generator=g)) for _ in _materials(scene)],
         "sigma_e": [float(torch.randn((), generator=g)) * 0.01 for _ in _materials(scene)],
         "frequency": float(torch.randn((), generator=g)) * 1e6,
         "tx": [torch.randn(3, generator=g, dtype=torch.float32) for _ in scene.transmitters],
         "rx": [torch.randn(3, generator=g, dtype=torch.float32) for _ in scene.receivers]}
    return t


def _weights(T, R, seed=3):
    rng = np.random.default_rng(seed)
    return rng.uniform(0.5, 1.5, (T, R)), rng.normal(size=(T, R)), rng.normal(size=(T, R))


@pytest.mark.parametrize("case", range(len(CASES)))
def test_jvp_matches_directional_fd_and_vjp(case):
    make, comps, depth, freq = CASES[case]
    # plain forward (for the weights' scales and the frozen path table)
    base = make()
    ref = solve(base, Config(components=comps, max_depth=depth, export_paths=True), reference_frequency_hz=freq)
    T, R = ref.path_gain.shape
    w, a, b = _weights(T, R)
    scale = float(ref.path_gain.max())
    fscale = float(ref.field.abs().max())
    tan = _direction(base, seed=11 + case)

    # forward mode
    scene = make()
    mats = _materials(scene)
    with fwAD.dual_level():
        for st, tv in zip(scene.structures, tan["vertices"]):
            st.geometry.vertices = fwAD.make_dual(st.vertices.detach(), tv)
        # materials are immutable records: replace each by a copy holding dual values
        for m, te, ts in zip(mats, tan["eps_r"], tan["sigma_e"]):
            dual = dataclasses.replace(
                m, eps_r=fwAD.make_dual(torch.as_tensor(m.eps_r).detach().double(), torch.tensor(te, dtype=torch.float64)),
                sigma_e=fwAD.make_dual(torch.as_tensor(m.sigma_e).detach().double(), torch.tensor(ts, dtype=torch.float64)))
            for st in scene.structures:
                if st.material is m:
                    st.material = dual
        for a_, tp in zip(scene.transmitters, tan["tx"]):
            a_.position = fwAD.make_dual(a_.position.detach(), tp)
        for a_, tp in zip(scene.receivers, tan["rx"]):
            a_.position = fwAD.make_dual(a_.position.detach(), tp)
        f_dual = fwAD.make_dual(torch.tensor(freq, dtype=torch.float64), torch.tensor(tan["frequency"],
                                                                                       dtype=torch.float64))
        res = solve(scene, Config(components=comps, max_depth=depth, ad_mode="jvp"), reference_frequency_hz=f_dual)
        d_pg = fwAD.unpack_dual(res.path_gain).tangent
        d_f = fwAD.unpack_dual(res.field).tangent
    assert d_pg is not None and d_f is not None
    jvp = float((torch.tensor(w, device="cuda") * d_pg.double()).sum() / scale +
                (torch.tensor(a, device="cuda") * d_f.real.double() +
                 torch.tensor(b, device="cuda") * d_f.imag.double()).sum() / fscale)
    torch.testing.assert_close(res.path_gain.detach(), ref.path_gain, rtol=1e-4, atol=1e-12)

    # directional FD of the oracle's fixed-topology re-evaluation
    p = ref.paths
    table = {"tx_id": p.tx_id.cpu().numpy(), "rx_id": p.rx_id.cpu().numpy(),
             "component_id": p.component_id.cpu().numpy(), "depth": p.depth.cpu().numpy(),
             "primitive_sequence": p.primitive_sequence.cpu().numpy(), "edge_id": p.edge_id.cpu().numpy()}
    arrays = osolve.scene_arrays(base, freq)
    tv = np.concatenate([t.double().numpy().reshape(-1, 3) for t in tan["vertices"]])
    bmats = _materials(base)

    def moved(h):
        a2 = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in arrays.items()}
        a2["face_mats"] = {k: v.copy() for k, v in arrays["face_mats"].items()}
        a2["material_layers"] = list(arrays["material_layers"])
        a2["vertices"] = arrays["vertices"] + h * tv
        for mi in range(len(bmats)):
            faces = a2["face_material"] == mi
            a2["face_mats"]["eps_r"][faces] += h * tan["eps_r"][mi]
            a2["face_mats"]["sigma_e"][faces] += h * tan["sigma_e"][mi]
            th, er, sg, mr = a2["material_layers"][mi]
            a2["material_layers"][mi] = (th, er + np.r_[h * tan["eps_r"][mi], np.zeros(len(er) - 1)],
                                         sg + np.r_[h * tan["sigma_e"][mi], np.zeros(len(sg) - 1)], mr)
        a2["tx_pos"] = arrays["tx_pos"] + h * np.stack([t.double().numpy() for t in tan["tx"]])
        a2["rx_pos"] = arrays["rx_pos"] + h * np.stack([t.double().numpy() for t in tan["rx"]])
        return a2, freq + h * tan["frequency"]

    def loss(h):
        a2, f2 = moved(h)
        fields = oadj.fixed_topology_fields(a2, table, f2)
        pg = oadj.cell_path_gain(fields, table, T, R)
        acc = np.zeros((T, R), dtype=np.complex128)
        np.add.at(acc, (table["tx_id"], table["rx_id"]), fields)
        return float((w * pg).sum() / scale + (a * acc.real + b * acc.imag).sum() / fscale)

    hstep = 1e-4

    def central(hh):
        return (loss(hh) - loss(-hh)) / (2 * hh)

    d1, d2, d4 = central(hstep), central(hstep / 2), central(hstep / 4)
    r1, r2 = (4 * d2 - d1) / 3, (4 * d4 - d2) / 3
    assert abs(r1 - r2) <= 1e-3 * abs(r2), "finite differences are not smooth here"
    assert abs(jvp - r2) <= 1e-4 * abs(r2), (jvp, r2)

    # duality with the VJP on the same loss
    scene2 = make()
    ft = torch.tensor(freq, dtype=torch.float64, requires_grad=True)
    res2 = solve(scene2, Config(components=comps, max_depth=depth, ad_mode="vjp"), reference_frequency_hz=ft)
    l2 = (torch.tensor(w, device="cuda") * res2.path_gain.double()).sum() / scale + \
        (torch.tensor(a, device="cuda") * res2.field.real.double() +
         torch.tensor(b, device="cuda") * res2.field.imag.double()).sum() / fscale
    l2.backward()
    dual = 0.0
    for st, t in zip(scene2.structures, tan["vertices"]):
        dual += float((st.vertices.grad.double() * t.double()).sum())
    for m, te, ts in zip(_materials(scene2), tan["eps_r"], tan["sigma_e"]):
        dual += float(m.eps_r.grad) * te + float(m.sigma_e.grad) * ts
    dual += float(ft.grad) * tan["frequency"]
    for a_, t in zip(scene2.transmitters, tan["tx"]):
        dual += float((a_.position.grad.double() * t.double()).sum())
    for a_, t in zip(scene2.receivers, tan["rx"]):
        dual += float((a_.position.grad.double() * t.double()).sum())
    assert abs(jvp - dual) <= 1e-5 * abs(dual), (jvp, dual)
