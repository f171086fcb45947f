"""First-order AD of the consumer's scalar coefficient on the GPU (reference
``propagation/consumer.py`` ``ad_mode="vjp"`` / ``"jvp"``; tests after the
reference's ``tests/propagation/consumer/test_*ad*.py``).

Checked, on a two-wall scene (LoS and reflections up to depth 2) and on the
small city (LoS, reflection, diffraction):

* reverse mode against central finite differences of the frozen-topology
  replay (the topology held fixed, as the derivative is defined) for source
  and sink positions, a wall's vertices, a material's permittivity and
  conductivity and the frequency;
* forward mode against reverse mode (<v, J u> = <J^T v, u>);
* the discovery route and the replay route give the same gradients for the
  same rows;
* rows that stopped existing in a replay carry no derivative;
* refusals before any native work: primal-only inputs carrying AD,
  responses other than scalar_transport, a forward dual under ``vjp``,
  wideband offsets with AD.
"""

from __future__ import annotations

import dataclasses

import pytest
import torch

from tests import scenes
from witwin_channel_b200.compiler import compile_scene
from witwin_channel_b200.propagation import consumer as c
from witwin_channel_b200.scene import PhysicalMaterial, Scene, make_mesh_structure

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda", 0)
FREQ = 2.4e9


def _batch(positions, ids, powers=None, pol=(0.0, 0.0, 1.0)):
    pos = torch.as_tensor(positions, dtype=torch.float32).reshape(-1, 3).to(DEV).contiguous()
    n = pos.shape[0]
    return c.EndpointBatch(stable_ids=torch.arange(n, dtype=torch.int64, device=DEV) + ids, positions_m=pos,
                           polarizations=torch.tensor([pol] * n, dtype=torch.float32, device=DEV),
                           powers_w=None if powers is None else torch.full((n,), powers, dtype=torch.float32,
                                                                           device=DEV))


def _walls(eps=None, sigma=None):
    """The two-wall scene with an optional tensor-valued wall material."""
    base = scenes.two_wall_scene()
    if eps is not None:
        st = base.structures[0]
        base.structures[0] = make_mesh_structure(vertices=st.vertices, faces=st.faces,
                                                 material=PhysicalMaterial(eps_r=eps, sigma_e=sigma), surface_id=10)
    return base


def _request(sources, sinks, freq=FREQ, ad="vjp", comps=("los", "reflection"), depth=2, **kw):
    return c.PropagationRequest(sources=sources, sinks=sinks, reference_frequency_hz=freq,
                                components=frozenset(comps), max_depth=depth, response="scalar_transport",
                                topology_mode="discover", ad_mode=ad, **kw)


def _replay(compiled, sources, sinks, prepared, freq=FREQ, ad="vjp"):
    return c.reevaluate(compiled, c.FixedTopologyRequest(
        sources=sources, sinks=sinks, reference_frequency_hz=freq, topology=prepared, response="scalar_transport",
        ad_mode=ad, world_motion="fixed_winner_replay"))


SRC = [[0.0, 0.0, 1.0]]
SNK = [[0.0, 1.0, 1.0], [0.4, 1.3, 0.7], [-0.5, 0.8, 1.2]]


def _unanchored(prepared):
    """The same frozen rows without world provenance: the finite differences
    replay them on scenes compiled from perturbed copies of the world."""
    topology = dataclasses.replace(prepared.topology, provenance=None)
    return c.PreparedFixedTopology(topology=topology, buckets=prepared.buckets, prepare_d2h_copies=0,
                                   prepare_d2h_bytes=0, prepare_synchronizations=0,
                                   execution_order=prepared.execution_order)


def _weights(K, seed=5):
    g = torch.Generator().manual_seed(seed)
    return torch.complex(torch.randn(K, generator=g), torch.randn(K, generator=g)).to(DEV)


def _loss(coef, w, mask=None, scale=None):
    """A real loss of the coefficients: a weighted sum plus their power, over
    the rows in ``mask``; ``scale`` (default: this call's largest magnitude)
    normalises the power term."""
    if mask is not None:
        coef = coef * mask.to(device=coef.device, dtype=coef.real.dtype)
    if scale is None:
        scale = coef.abs().max().detach().clamp_min(1e-30)
    return (coef * w).real.sum() + 0.3 * (coef.abs() ** 2).sum() / scale


def _stable_rows(replay, points):
    """Rows valid at every perturbed point (a finite difference across a
    row's birth or death is not a derivative of the frozen topology)."""
    stable = None
    for point in points:
        _coef, valid = replay(*point)
        stable = valid if stable is None else stable & valid
    return stable


def test_positions_vjp_matches_replay_finite_differences():
    scene = _walls()
    compiled = compile_scene(scene, DEV)
    sources, sinks = _batch(SRC, 0, powers=1.0), _batch(SNK, 10)
    found = c.evaluate(compiled, _request(sources, sinks, ad="none"))
    K = found.paths.path_count
    assert K >= 6
    w = _weights(K)
    prepared = c.prepare_fixed_topology(found.paths.topology)
    scale = float(found.paths.transport.coefficient.abs().max())

    def replay(src, snk):
        with torch.no_grad():
            out = _replay(compiled, _batch(src, 0, powers=1.0), _batch(snk, 10), prepared, ad="none")
            return out.paths.transport.coefficient.to(torch.complex128), out.row_valid

    h = 1e-3
    base = torch.tensor(SRC + SNK)
    points = []
    for idx in range(base.numel()):
        for sign in (1.0, -1.0):
            p = base.clone().reshape(-1)
            p[idx] += sign * h
            p = p.reshape(base.shape)
            points.append((p[:1], p[1:]))
    stable = _stable_rows(replay, points)
    assert int(stable.sum()) >= K - 2
    # reverse mode on the discovery route, the loss over the stable rows
    src_pos = torch.tensor(SRC, device=DEV, requires_grad=True)
    snk_pos = torch.tensor(SNK, device=DEV, requires_grad=True)
    sources_ad = c.EndpointBatch(stable_ids=sources.stable_ids, positions_m=src_pos,
                                 polarizations=sources.polarizations, powers_w=sources.powers_w)
    sinks_ad = c.EndpointBatch(stable_ids=sinks.stable_ids, positions_m=snk_pos, polarizations=sinks.polarizations)
    out = c.evaluate(compiled, _request(sources_ad, sinks_ad))
    _loss(out.paths.transport.coefficient, w, stable, scale).backward()
    grad = torch.cat([src_pos.grad, snk_pos.grad]).cpu()
    w64 = w.to(torch.complex128)
    fd = torch.zeros_like(base)
    for idx in range(base.numel()):
        plus, minus = points[2 * idx], points[2 * idx + 1]
        fd.reshape(-1)[idx] = (float(_loss(replay(*plus)[0], w64, stable, scale))
                               - float(_loss(replay(*minus)[0], w64, stable, scale))) / (2 * h)
    torch.testing.assert_close(grad, fd.float(), rtol=0, atol=float(2e-3 * fd.abs().max()))


def test_material_vertex_and_frequency_vjp_matches_finite_differences():
    eps = torch.tensor(3.0, requires_grad=True)
    sigma = torch.tensor(0.005, requires_grad=True)
    scene = _walls(eps, sigma)
    scene.structures[1].geometry.vertices = scene.structures[1].vertices.clone().requires_grad_(True)
    freq = torch.tensor(FREQ, dtype=torch.float64, requires_grad=True)
    compiled = compile_scene(scene, DEV)
    sources, sinks = _batch(SRC, 0, powers=1.0), _batch(SNK, 10)
    found = c.evaluate(compiled, _request(sources, sinks, freq=freq))
    K = found.paths.path_count
    w = _weights(K, seed=7)
    scale = float(found.paths.transport.coefficient.abs().max())
    prepared = _unanchored(c.prepare_fixed_topology(found.paths.topology))
    v0 = scenes.two_wall_scene().structures[1].vertices.detach().clone()

    def replay(eps_v=3.0, sigma_v=0.005, f=FREQ, verts=None):
        sc = _walls(torch.tensor(eps_v), torch.tensor(sigma_v))
        if verts is not None:
            sc.structures[1].geometry.vertices = verts
        comp = compile_scene(sc, DEV)
        with torch.no_grad():
            out = _replay(comp, sources, sinks, prepared, freq=f, ad="none")
            return out.paths.transport.coefficient.to(torch.complex128), out.row_valid

    h = 1e-3
    vertex_points = []
    for idx in range(v0.numel()):
        for sign in (1.0, -1.0):
            p = v0.clone().reshape(-1)
            p[idx] += sign * h
            vertex_points.append(p.reshape(v0.shape))
    stable = _stable_rows(lambda v: replay(verts=v), [(v,) for v in vertex_points])
    assert int(stable.sum()) >= K - 2
    _loss(found.paths.transport.coefficient, w, stable, scale).backward()
    grads = {"eps": eps.grad, "sigma": sigma.grad, "freq": freq.grad,
             "vert": scene.structures[1].vertices.grad.clone()}
    assert all(g is not None for g in grads.values())
    w64 = w.to(torch.complex128)
    L = lambda **kw: float(_loss(replay(**kw)[0], w64, stable, scale))
    for name, step, kw in (("eps", 1e-3, "eps_v"), ("sigma", 5e-4, "sigma_v")):
        base = 3.0 if name == "eps" else 0.005
        fd = (L(**{kw: base + step}) - L(**{kw: base - step})) / (2 * step)
        assert abs(float(grads[name]) - fd) <= 2e-3 * abs(fd) + 1e-9, (name, float(grads[name]), fd)
    df = 2e4
    fd = (L(f=FREQ + df) - L(f=FREQ - df)) / (2 * df)
    assert abs(float(grads["freq"]) - fd) <= 5e-3 * abs(fd) + 1e-15, (float(grads["freq"]), fd)
    gv = grads["vert"].reshape(-1)
    for idx in range(v0.numel()):
        fd = (L(verts=vertex_points[2 * idx]) - L(verts=vertex_points[2 * idx + 1])) / (2 * h)
        assert abs(float(gv[idx]) - fd) <= 3e-3 * float(gv.abs().max()) + 1e-12, (idx, float(gv[idx]), fd)


def test_forward_mode_is_the_adjoint_of_reverse_mode():
    scene, freq = scenes.small_city()
    compiled = compile_scene(scene, DEV)
    grid = scene.receivers[0].points()[:12].float()
    tx = scene.transmitters[0].position.float().reshape(1, 3)
    g = torch.Generator().manual_seed(11)
    u_src = torch.randn((1, 3), generator=g).to(DEV)
    u_snk = torch.randn((12, 3), generator=g).to(DEV)
    comps = ("los", "reflection", "diffraction")
    # reverse
    src_pos = tx.to(DEV).clone().requires_grad_(True)
    snk_pos = grid.to(DEV).clone().requires_grad_(True)
    mk = lambda sp, kp: (c.EndpointBatch(stable_ids=torch.zeros(1, dtype=torch.int64, device=DEV), positions_m=sp,
                                         polarizations=torch.tensor([[0.0, 0.0, 1.0]], device=DEV),
                                         powers_w=torch.ones(1, device=DEV)),
                         c.EndpointBatch(stable_ids=torch.arange(12, device=DEV), positions_m=kp,
                                         polarizations=torch.tensor([[0.0, 0.0, 1.0]] * 12, device=DEV)))
    out = c.evaluate(compiled, _request(*mk(src_pos, snk_pos), freq=freq, comps=comps, depth=2))
    K = out.paths.path_count
    assert bool((out.paths.topology.component_id == 2).any())
    v = _weights(K, seed=13)
    (out.paths.transport.coefficient * v.conj()).real.sum().backward()
    reverse = float((src_pos.grad * u_src).sum() + (snk_pos.grad * u_snk).sum())
    # forward
    import torch.autograd.forward_ad as fwAD

    with fwAD.dual_level():
        sp = fwAD.make_dual(tx.to(DEV).clone(), u_src)
        kp = fwAD.make_dual(grid.to(DEV).clone(), u_snk)
        out_f = c.evaluate(compiled, _request(*mk(sp, kp), freq=freq, comps=comps, depth=2, ad="jvp"))
        tangent = fwAD.unpack_dual(out_f.paths.transport.coefficient).tangent
    assert tangent is not None and out_f.paths.path_count == K
    forward = float((tangent * v.conj()).real.sum())
    assert abs(forward - reverse) <= 1e-4 * abs(reverse) + 1e-12, (forward, reverse)


def test_discovery_and_replay_give_the_same_gradients():
    scene = _walls()
    compiled = compile_scene(scene, DEV)

    def grads(replay):
        snk_pos = torch.tensor(SNK, device=DEV, requires_grad=True)
        sinks = c.EndpointBatch(stable_ids=torch.arange(3, device=DEV) + 10, positions_m=snk_pos,
                                polarizations=torch.tensor([[0.0, 0.0, 1.0]] * 3, device=DEV))
        sources = _batch(SRC, 0, powers=1.0)
        out = c.evaluate(compiled, _request(sources, sinks, ad="vjp" if not replay else "none"))
        if replay:
            out = _replay(compiled, sources, sinks, c.prepare_fixed_topology(out.paths.topology))
        w = _weights(out.paths.path_count, seed=3)
        _loss(out.paths.transport.coefficient, w).backward()
        return snk_pos.grad

    torch.testing.assert_close(grads(False), grads(True), rtol=1e-6, atol=1e-9)


def test_rows_that_stop_existing_carry_no_derivative():
    scene = _walls()
    compiled = compile_scene(scene, DEV)
    sources = _batch(SRC, 0, powers=1.0)
    found = c.evaluate(compiled, _request(sources, _batch(SNK[:1], 10), ad="none"))
    prepared = c.prepare_fixed_topology(found.paths.topology)
    behind = torch.tensor([[4.0, 1.0, 1.0]], device=DEV, requires_grad=True)  # behind the wall at x = 2
    sinks = c.EndpointBatch(stable_ids=torch.tensor([10], device=DEV), positions_m=behind,
                            polarizations=torch.tensor([[0.0, 0.0, 1.0]], device=DEV))
    out = _replay(compiled, sources, sinks, prepared)
    assert not bool(out.row_valid.all())
    coef = out.paths.transport.coefficient
    dead = ~out.row_valid
    (coef[dead].abs() ** 2).sum().backward(retain_graph=True)
    assert behind.grad is None or float(behind.grad.abs().max()) == 0.0


def test_ad_refusals_before_native_work():
    eps = torch.tensor(3.0)
    scene = Scene(structures=[make_mesh_structure(
        vertices=torch.tensor([[2.0, -1.0, 0.0], [2.0, 3.0, 0.0], [2.0, -1.0, 2.0]]), faces=torch.tensor([[0, 1, 2]]),
        material=PhysicalMaterial(eps_r=eps, sigma_e=0.01, thickness_m=torch.tensor(0.2, requires_grad=True)))],
        endpoints=[])
    compiled = compile_scene(scene, DEV)
    sources, sinks = _batch(SRC, 0, powers=1.0), _batch(SNK, 10)
    before = c._native.launch_count()
    with pytest.raises(NotImplementedError, match="thickness_m is primal-only"):
        c.evaluate(compiled, _request(sources, sinks))
    powered = c.EndpointBatch(stable_ids=sources.stable_ids, positions_m=sources.positions_m,
                              polarizations=sources.polarizations,
                              powers_w=torch.ones(1, device=DEV, requires_grad=True))
    plain = compile_scene(_walls(), DEV)
    with pytest.raises(NotImplementedError, match="powers_w is primal-only"):
        c.evaluate(plain, _request(powered, sinks))
    with pytest.raises(NotImplementedError):
        c.evaluate(plain, c.PropagationRequest(sources=sources, sinks=sinks, reference_frequency_hz=FREQ,
                                               components=frozenset({"los"}), max_depth=0,
                                               response="polarimetric_transport", topology_mode="discover",
                                               ad_mode="vjp"))
    import torch.autograd.forward_ad as fwAD

    with fwAD.dual_level():
        dual = fwAD.make_dual(sinks.positions_m.clone(), torch.ones_like(sinks.positions_m))
        dual_sinks = c.EndpointBatch(stable_ids=sinks.stable_ids, positions_m=dual, polarizations=sinks.polarizations)
        with pytest.raises(NotImplementedError, match="second-order"):
            c.evaluate(plain, _request(sources, dual_sinks, ad="vjp"))
    assert c._native.launch_count() == before
    found = c.evaluate(plain, _request(sources, sinks, ad="none"))
    with pytest.raises(NotImplementedError, match="wideband"):
        c.reevaluate(plain, c.FixedTopologyRequest(
            sources=sources, sinks=sinks, reference_frequency_hz=FREQ,
            topology=c.prepare_fixed_topology(found.paths.topology), response="scalar_transport", ad_mode="vjp",
            frequency_offsets_hz=(1.0e6,)))


def test_complex3_field_vjp_matches_replay_finite_differences():
    """The complex3 field (each world component through the native VJP with
    that axis as the sink polarization) against central differences of the
    replayed complex3 field, for the sink positions."""
    scene = _walls()
    compiled = compile_scene(scene, DEV)
    sources, sinks = _batch(SRC, 0, powers=1.0), _batch(SNK, 10)

    def request3(snk, ad):
        return c.PropagationRequest(sources=sources, sinks=snk, reference_frequency_hz=FREQ,
                                    components=frozenset({"los", "reflection"}), max_depth=2,
                                    response="complex3_transport", topology_mode="discover", ad_mode=ad)

    found = c.evaluate(compiled, request3(sinks, "none"))
    prepared = c.prepare_fixed_topology(found.paths.topology)
    K = found.paths.path_count
    g = torch.Generator().manual_seed(17)
    w = torch.complex(torch.randn((K, 3), generator=g), torch.randn((K, 3), generator=g)).to(DEV)
    scale = float(found.paths.transport.field.abs().max())

    def loss3(field, mask):
        m = mask.to(device=field.device, dtype=field.real.dtype).view(-1, 1)
        return (field * m * w.to(field.dtype)).real.sum() / scale

    def replay(snk_pos):
        with torch.no_grad():
            out = c.reevaluate(compiled, c.FixedTopologyRequest(
                sources=sources, sinks=_batch(snk_pos, 10), reference_frequency_hz=FREQ, topology=prepared,
                response="complex3_transport", ad_mode="none"))
            return out.paths.transport.field.to(torch.complex128), out.row_valid

    h = 1e-3
    base = torch.tensor(SNK)
    points = []
    for idx in range(base.numel()):
        for sign in (1.0, -1.0):
            p = base.clone().reshape(-1)
            p[idx] += sign * h
            points.append(p.reshape(base.shape))
    stable = _stable_rows(replay, [(p,) for p in points])
    snk_pos = torch.tensor(SNK, device=DEV, requires_grad=True)
    sinks_ad = c.EndpointBatch(stable_ids=sinks.stable_ids, positions_m=snk_pos, polarizations=sinks.polarizations)
    out = c.evaluate(compiled, request3(sinks_ad, "vjp"))
    loss3(out.paths.transport.field, stable).backward()
    fd = torch.zeros_like(base)
    for idx in range(base.numel()):
        fd.reshape(-1)[idx] = (float(loss3(replay(points[2 * idx])[0], stable))
                               - float(loss3(replay(points[2 * idx + 1])[0], stable))) / (2 * h)
    torch.testing.assert_close(snk_pos.grad.cpu(), fd.float(), rtol=0, atol=float(2e-3 * fd.abs().max()))


def test_replayed_path_lengths_and_delays_carry_geometry_derivatives():
    """Replay path lengths (and delays) differentiate in the sink positions and
    a wall's vertices: against central differences of the replayed lengths."""
    scene = _walls()
    scene.structures[1].geometry.vertices = scene.structures[1].vertices.clone().requires_grad_(True)
    compiled = compile_scene(scene, DEV)
    sources, sinks = _batch(SRC, 0, powers=1.0), _batch(SNK, 10)
    found = c.evaluate(compiled, _request(sources, sinks, ad="none"))
    prepared = _unanchored(c.prepare_fixed_topology(found.paths.topology))
    K = found.paths.path_count
    w = torch.rand(K, generator=torch.Generator().manual_seed(23)).to(DEV)
    v0 = scene.structures[1].vertices.detach().clone()

    def replay(snk, verts=None):
        sc = _walls()
        if verts is not None:
            sc.structures[1].geometry.vertices = verts
        comp = compile_scene(sc, DEV)
        with torch.no_grad():
            out = _replay(comp, sources, _batch(snk, 10), prepared, ad="none")
            return out.paths.geometry.path_length_m.double(), out.row_valid

    h = 1e-3
    base = torch.tensor(SNK)
    snk_points, vert_points = [], []
    for idx in range(base.numel()):
        for sign in (1.0, -1.0):
            p = base.clone().reshape(-1)
            p[idx] += sign * h
            snk_points.append(p.reshape(base.shape))
    for idx in range(v0.numel()):
        for sign in (1.0, -1.0):
            p = v0.clone().reshape(-1)
            p[idx] += sign * h
            vert_points.append(p.reshape(v0.shape))
    stable = _stable_rows(lambda s: replay(s), [(p,) for p in snk_points])
    stable = stable & _stable_rows(lambda v: replay(base, v), [(v,) for v in vert_points])
    m = stable.double()
    snk_pos = torch.tensor(SNK, device=DEV, requires_grad=True)
    sinks_ad = c.EndpointBatch(stable_ids=sinks.stable_ids, positions_m=snk_pos, polarizations=sinks.polarizations)
    out = _replay(compiled, sources, sinks_ad, prepared)
    L = out.paths.geometry.path_length_m
    assert L.requires_grad and out.paths.geometry.delay_s.requires_grad
    torch.testing.assert_close(out.paths.geometry.delay_s, L / 299_792_458.0, rtol=1e-6, atol=0.0)
    (L.double() * w * m).sum().backward()
    loss = lambda lengths: float((lengths * w * m).sum())
    fd = torch.tensor([(loss(replay(snk_points[2 * i])[0]) - loss(replay(snk_points[2 * i + 1])[0])) / (2 * h)
                       for i in range(base.numel())], dtype=torch.float64).reshape(base.shape)
    torch.testing.assert_close(snk_pos.grad.cpu().double(), fd, rtol=0, atol=2e-3 * float(fd.abs().max()))
    gv = scene.structures[1].vertices.grad.reshape(-1).double().cpu()
    fdv = torch.tensor([(loss(replay(base, vert_points[2 * i])[0]) - loss(replay(base, vert_points[2 * i + 1])[0]))
                        / (2 * h) for i in range(v0.numel())], dtype=torch.float64)
    torch.testing.assert_close(gv, fdv, rtol=0, atol=3e-3 * float(fdv.abs().max()) + 1e-9)
