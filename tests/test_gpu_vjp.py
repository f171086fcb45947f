"""Fixed-topology VJP (``ad_mode="vjp"``) against central finite differences.

The reference's deterministic AD differentiates with every path's
interaction sequence frozen; ``oracle/adjoint.py`` re-evaluates a frozen
path table in FP64 from raw arrays with the same definition, so central
differences of it (relative step 1e-4, FP64) are the derivative to match.
Central differences are Richardson-extrapolated (steps h, h/2, h/4 with
h the relative step 1e-4): at 28 GHz a 1e-4 relative step of a 6 m coordinate
moves the carrier phase by 0.35 rad, and the plain central difference is then
off by ~(k h)^2/6 = 2%.  The two extrapolations (h, h/2) and (h/2, h/4) must
agree within 1e-3, which also shows the loss is smooth there (receivers sit
away from shadow boundaries).  Tolerance: 1e-4
relative per parameter whose FD gradient is above 1e-3 of the largest, 1e-7
of the largest in absolute terms otherwise.
"""

from __future__ import annotations

import copy

import numpy as np
import pytest
import torch

from oracle import adjoint as oadj
from oracle import solve as osolve
from witwin_channel_b200 import Config, solve
from witwin_channel_b200.scene import (
    PhysicalMaterial,
    Scene,
    make_mesh_structure,
    make_receiver,
    make_receiver_grid,
    make_transmitter,
)

pytestmark = pytest.mark.gpu
REL = 1.0e-4


def _leaf(x):
    return torch.tensor(x, dtype=torch.float32, requires_grad=True)


def _tx(pos):
    a = make_transmitter(pos)
    a.position = _leaf(pos)  # keep the leaf itself so its .grad is populated
    return a


def _rx(pos):
    a = make_receiver(pos)
    a.position = _leaf(pos)
    return a


def _mat(eps, sig, **kw):
    return PhysicalMaterial(eps_r=torch.tensor(eps, dtype=torch.float64, requires_grad=True),
                            sigma_e=torch.tensor(sig, dtype=torch.float64, requires_grad=True), **kw)


def two_wall():
    wx = make_mesh_structure(vertices=_leaf([[2.0, -1.0, 0.0], [2.0, 3.0, 0.0], [2.0, -1.0, 2.0], [2.0, 3.0, 2.0]]),
                             faces=torch.tensor([[0, 1, 2], [1, 3, 2]]), material=_mat(3.0, 0.005), surface_id=10)
    wy = make_mesh_structure(vertices=_leaf([[0.0, 2.0, 0.0], [3.0, 2.0, 0.0], [0.0, 2.0, 2.0], [3.0, 2.0, 2.0]]),
                             faces=torch.tensor([[0, 2, 1], [1, 2, 3]]), material=_mat(4.0, 0.01), surface_id=11)
    return Scene(structures=[wx, wy], endpoints=[_tx(([0.0, 0.0, 1.0])),
                                                  _rx(([0.0, 1.0, 1.0])),
                                                  _rx(([0.5, 1.2, 1.3]))])


def wedge():
    a = make_mesh_structure(vertices=_leaf([[2.0, 0.0, -1.0], [2.0, 0.0, 2.0], [2.0, 2.0, -1.0]]),
                            faces=torch.tensor([[0, 1, 2]]), material=_mat(5.0, 0.05), surface_id=2)
    b = make_mesh_structure(vertices=_leaf([[2.0, 0.0, -1.0], [2.0, 0.0, 2.0], [4.0, 0.0, -1.0]]),
                            faces=torch.tensor([[0, 2, 1]]), material=_mat(3.0, 0.02), surface_id=3)
    return Scene(structures=[a, b], endpoints=[_tx(([0.0, -1.0, 0.5])),
                                                _rx(([3.13, 1.07, 0.53])),
                                                _rx(([3.52, 0.81, 0.22]))])


def thin_walls():
    w = make_mesh_structure(vertices=_leaf([[2.0, -4.0, -4.0], [2.0, 4.0, -4.0], [2.0, -4.0, 4.0], [2.0, 4.0, 4.0]]),
                            faces=torch.tensor([[0, 1, 2], [1, 3, 2]]), material=_mat(6.27, 0.2287, thickness_m=0.012),
                            surface_id=1)
    w2 = make_mesh_structure(vertices=_leaf([[4.0, -4.0, -4.0], [4.0, 4.0, -4.0], [4.0, -4.0, 4.0], [4.0, 4.0, 4.0]]),
                             faces=torch.tensor([[0, 1, 2], [1, 3, 2]]), material=_mat(4.0, 0.02, thickness_m=0.1),
                             surface_id=2)
    return Scene(structures=[w, w2], endpoints=[_tx(([0.0, 0.3, 0.2])),
                                                 _rx(([6.0, -0.5, 0.4])),
                                                 _rx(([3.0, 1.0, -0.3])),
                                                 _rx(([1.0, 0.5, 0.35]))])


def _params(scene):
    """Every scalar checked by FD.  Coincident vertices of different structures
    (a shared boundary edge merges them) move together as one parameter."""
    out = []
    groups: dict[tuple, list] = {}
    for s, st in enumerate(scene.structures):
        for v in range(st.vertices.shape[0]):
            key = tuple(round(float(x), 6) for x in st.vertices[v].detach())
            groups.setdefault(key, []).append((s, v))
    for members in groups.values():
        for c in range(3):
            out.append(("vertex", (tuple(members), c)))
    mats = []
    for st in scene.structures:
        if all(st.material is not m for m in mats):
            mats.append(st.material)
    for m in range(len(mats)):
        out.append(("eps_r", m))
        out.append(("sigma_e", m))
    out.append(("frequency", None))
    for t in range(len(scene.transmitters)):
        for c in range(3):
            out.append(("tx", (t, c)))
    for r in range(len(scene.receivers)):
        for c in range(3):
            out.append(("rx", (r, c)))
    return out, mats


def _perturb(arrays, scene, mats, key, h, freq):
    a = copy.deepcopy(arrays)
    kind, idx = key
    f = freq
    if kind == "vertex":
        members, c = idx
        for s, v in members:
            off = sum(st.vertices.shape[0] for st in scene.structures[:s])
            a["vertices"][off + v, c] += h
    elif kind in ("eps_r", "sigma_e"):
        m = idx
        faces = a["face_material"] == m
        a["face_mats"][kind][faces] += h
        th, er, sg, mr = a["material_layers"][m]
        if kind == "eps_r":
            er = er.copy(); er[0] += h
        else:
            sg = sg.copy(); sg[0] += h
        a["material_layers"][m] = (th, er, sg, mr)
    elif kind == "frequency":
        f = freq + h
    elif kind == "tx":
        t, c = idx
        a["tx_pos"][t, c] += h
    elif kind == "rx":
        r, c = idx
        a["rx_pos"][r, c] += h
    return a, f


def _value(arrays, scene, mats, key, freq):
    kind, idx = key
    if kind == "vertex":
        members, c = idx
        s, v = members[0]
        off = sum(st.vertices.shape[0] for st in scene.structures[:s])
        return arrays["vertices"][off + v, c]
    if kind in ("eps_r", "sigma_e"):
        return arrays["material_layers"][idx][1 if kind == "eps_r" else 2][0]
    if kind == "frequency":
        return freq
    if kind == "tx":
        return arrays["tx_pos"][idx]
    return arrays["rx_pos"][idx]


def _grad_of(scene, mats, key, freq_t):
    kind, idx = key
    if kind == "vertex":
        members, c = idx
        total = 0.0
        for s, v in members:
            g = scene.structures[s].vertices.grad
            total += 0.0 if g is None else float(g[v, c])
        return total
    if kind in ("eps_r", "sigma_e"):
        g = getattr(mats[idx], kind).grad
        return 0.0 if g is None else float(g)
    if kind == "frequency":
        return 0.0 if freq_t.grad is None else float(freq_t.grad)
    if kind == "tx":
        g = scene.transmitters[idx[0]].position.grad
        return 0.0 if g is None else float(g[idx[1]])
    g = scene.receivers[idx[0]].position.grad
    return 0.0 if g is None else float(g[idx[1]])


def _check_against_fd(scene, components, max_depth, freq):
    freq_t = torch.tensor(freq, dtype=torch.float64, requires_grad=True)
    cfg = Config(components=components, max_depth=max_depth, ad_mode="vjp", export_paths=True)
    res = solve(scene, cfg, reference_frequency_hz=freq_t)
    T, R = res.path_gain.shape
    rng = np.random.default_rng(3)
    w = rng.uniform(0.5, 1.5, (T, R))
    a = rng.normal(size=(T, R))
    b = rng.normal(size=(T, R))
    scale = float(res.path_gain.detach().max())
    fscale = float(res.field.detach().abs().max())
    loss = (torch.tensor(w, device="cuda") * res.path_gain.double()).sum() / scale + \
        (torch.tensor(a, device="cuda") * res.field.real.double() +
         torch.tensor(b, device="cuda") * res.field.imag.double()).sum() / fscale
    loss.backward()
    p = res.paths
    table = {"tx_id": p.tx_id.cpu().numpy(), "rx_id": p.rx_id.cpu().numpy(),
             "component_id": p.component_id.cpu().numpy(), "depth": p.depth.cpu().numpy(),
             "primitive_sequence": p.primitive_sequence.cpu().numpy(), "edge_id": p.edge_id.cpu().numpy()}
    arrays = osolve.scene_arrays(scene, freq)

    def oracle_loss(arr, f):
        fields = oadj.fixed_topology_fields(arr, table, f)
        pg = oadj.cell_path_gain(fields, table, T, R)
        acc = np.zeros((T, R), dtype=np.complex128)
        np.add.at(acc, (table["tx_id"], table["rx_id"]), fields)
        return float((w * pg).sum() / scale + (a * acc.real + b * acc.imag).sum() / fscale)

    keys, mats = _params(scene)
    fd, ours, rough = [], [], []
    for key in keys:
        x = float(_value(arrays, scene, mats, key, freq))
        h = REL * max(abs(x), 1.0)

        def central(step):
            ap, fp = _perturb(arrays, scene, mats, key, step, freq)
            am, fm = _perturb(arrays, scene, mats, key, -step, freq)
            return (oracle_loss(ap, fp) - oracle_loss(am, fm)) / (2 * step)

        d1, d2, d4 = central(h), central(h / 2), central(h / 4)
        r1, r2 = (4.0 * d2 - d1) / 3.0, (4.0 * d4 - d2) / 3.0
        fd.append(r2)
        rough.append(abs(r1 - r2))
        ours.append(_grad_of(scene, mats, key, freq_t))
    fd, ours, rough = np.array(fd), np.array(ours), np.array(rough)
    big = np.abs(fd).max()
    strong = np.abs(fd) > 1e-3 * big
    assert np.all(rough[strong] <= 1e-3 * np.abs(fd[strong])), "finite differences are not smooth here"
    bad = [(keys[i], ours[i], fd[i]) for i in range(len(keys))
           if (strong[i] and abs(ours[i] - fd[i]) > REL * abs(fd[i])) or
           (not strong[i] and abs(ours[i] - fd[i]) > 1e-7 * big)]
    assert not bad, bad[:8]
    assert strong.sum() >= 10
    return res


def test_vjp_reflection_and_los_match_fd():
    _check_against_fd(two_wall(), {"los", "reflection"}, 2, 3.0e9)


def test_vjp_diffraction_matches_fd():
    _check_against_fd(wedge(), {"diffraction"}, 1, 3.0e9)


def test_vjp_transmission_matches_fd():
    _check_against_fd(thin_walls(), {"los", "transmission", "reflection"}, 2, 28.0e9)


def test_vjp_is_deterministic_and_matches_forward():
    scene = two_wall()
    freq_t = torch.tensor(3.0e9, dtype=torch.float64, requires_grad=True)
    cfg = Config(components={"los", "reflection"}, max_depth=2, ad_mode="vjp")
    grads = []
    for _ in range(2):
        for st in scene.structures:
            st.vertices.grad = None
        res = solve(scene, cfg, reference_frequency_hz=freq_t)
        res.path_gain.sum().backward()
        grads.append(torch.cat([st.vertices.grad.reshape(-1) for st in scene.structures]).clone())
    assert torch.equal(grads[0], grads[1])
    plain = solve(scene, Config(components={"los", "reflection"}, max_depth=2), reference_frequency_hz=3.0e9)
    torch.testing.assert_close(res.path_gain.detach(), plain.path_gain, rtol=1e-4, atol=1e-12)


@pytest.mark.parametrize("make, comps, depth", [(two_wall, {"los", "reflection"}, 2),
                                                (wedge, {"diffraction"}, 1),
                                                (thin_walls, {"los", "transmission", "reflection"}, 2)])
def test_fp64_record_search_gives_the_same_records_and_gradients(make, comps, depth):
    """``precision="fp64"`` with ``ad_mode="vjp"`` (the plain all-FP64 form):
    the record search runs in FP64, the values and derivatives are FP64 in
    both forms, so the same records give the same gradients."""
    out = []
    for prec in ("mixed", "fp64"):
        scene = make()
        freq_t = torch.tensor(3.0e9, dtype=torch.float64, requires_grad=True)
        res = solve(scene, Config(components=comps, max_depth=depth, ad_mode="vjp", export_paths=True),
                    reference_frequency_hz=freq_t, precision=prec)
        (res.path_gain.double().sum() * 1e6).backward()
        g = torch.cat([st.vertices.grad.reshape(-1) for st in scene.structures] + [freq_t.grad.reshape(1)])
        out.append((res, g))
    (a, ga), (b, gb) = out
    for name in ("tx_id", "rx_id", "component_id", "depth", "edge_id", "primitive_sequence"):
        assert torch.equal(getattr(a.paths, name), getattr(b.paths, name)), name
    torch.testing.assert_close(a.path_gain, b.path_gain, rtol=1e-6, atol=0.0)
    torch.testing.assert_close(ga, gb, rtol=1e-9, atol=1e-12 * float(ga.abs().max()))
