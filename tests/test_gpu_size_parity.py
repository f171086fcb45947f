"""GPU parity on the benchmark workloads at their real sizes.

* two-ray ground check (64x64 grid at 2 m, 3.5 GHz): every cell against the
  closed-form two-ray field (free-space LoS plus one half-space Fresnel
  bounce of the z-polarised dipole), not against the ray-tracing oracle;
* urban canyon (64 boxes, 256x256 grid, 28 GHz, depth 3 + UTD): the full
  262,144-ray discovery on the GPU against the oracle's FP64 discovery of the
  same directions, then path records and cell fields on 256 strided cells;
* specular chains of depth 4 and 5: a closed room (exhaustive chains) and a
  16-box city (discovered chains);
* gradient run (canyon, eps_r x1.10 and 8 displaced boxes): the VJP of the
  log-gain MSE over sampled cells against Richardson-extrapolated central
  differences of the oracle's FP64 fixed-topology re-evaluation, for 22
  parameters (eps_r, sigma_e, frequency, Tx x/y/z and 16 box-vertex
  coordinates).

Tolerances as in the other parity tests: identical path records, gains
0.01 dB, phases 1e-3 rad, gradients 1e-4 relative of the finite difference.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from oracle import adjoint as oadj
from oracle import parallel as opar
from oracle import solve as osolve
from tests import scenes
from tests.test_gpu_parity import _check_cells, _db, _rows_key
from witwin_channel_b200 import Config, solve
from witwin_channel_b200.workloads import gradient_run, log_mse, two_ray_scene, urban_canyon_scene

pytestmark = pytest.mark.gpu

C0 = 299792458.0
EPS0 = 8.8541878128e-12


def _cell_index(x: torch.Tensor, shape) -> np.ndarray:
    """(T, shape[1], shape[0]) grid output -> (T, rows*cols) in point order."""
    rows, cols = shape
    return x.transpose(1, 2).reshape(x.shape[0], rows * cols).cpu().numpy()


# ---------------------------------------------------------------- two-ray
def _two_ray_closed_form(points: np.ndarray, tx: np.ndarray, f: float, eps_r: float, sigma: float):
    """LoS + ground bounce of a z-polarised isotropic dipole received on z.
    Amplitude lambda/(4 pi d) e^{-jkd}; the transmit and receive axes are the
    unnormalised transverse projections of z; the bounce multiplies the
    in-plane (TM) component by the half-space Fresnel coefficient."""
    k = 2 * np.pi * f / C0
    z = np.array([0.0, 0.0, 1.0])
    d_vec = points - tx
    d = np.linalg.norm(d_vec, axis=1)
    khat = d_vec / d[:, None]
    cz = khat @ z
    los = (1.0 / (2 * k * d)) * np.exp(-1j * k * d) * (1.0 - cz * cz)
    image = tx * np.array([1.0, 1.0, -1.0])
    r_vec = points - image
    dr = np.linalg.norm(r_vec, axis=1)
    rhat = r_vec / dr[:, None]  # reflected direction (ground point -> receiver)
    ihat = rhat * np.array([1.0, 1.0, -1.0])  # incident direction (Tx -> ground point)
    cos_t = np.abs(ihat[:, 2])
    sin2 = 1.0 - cos_t ** 2
    eta = eps_r - 1j * sigma / (2 * np.pi * f * EPS0)
    root = np.sqrt(eta - sin2)
    gamma_tm = (eta * cos_t - root) / (eta * cos_t + root)
    # p-axes: s = normalize(z x i); p_in = normalize(s x i); p_out = normalize(s x r)
    s = np.cross(np.broadcast_to(z, ihat.shape), ihat)
    s /= np.linalg.norm(s, axis=1)[:, None]
    p_in = np.cross(s, ihat)
    p_in /= np.linalg.norm(p_in, axis=1)[:, None]
    p_out = np.cross(s, rhat)
    p_out /= np.linalg.norm(p_out, axis=1)[:, None]
    tx_axis = z - (ihat @ z)[:, None] * ihat
    rx_axis = z - (rhat @ z)[:, None] * rhat
    e_p = np.sum(tx_axis * p_in, axis=1)
    refl = gamma_tm * e_p * np.sum(rx_axis * p_out, axis=1) * (1.0 / (2 * k * dr)) * np.exp(-1j * k * dr)
    return los, refl, d, dr


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_two_ray_full_grid_closed_form(precision):
    scene, f = two_ray_scene()
    # the FP64 form is a cell-mode solve (no path export)
    res = solve(scene, Config(components={"los", "reflection"}, max_depth=1, export_paths=precision == "mixed"),
                reference_frequency_hz=f, precision=precision)
    grid = scene.receivers[0]
    pts = grid.points().double().numpy()
    sigma = 0.0462 * (f / 1e9) ** 0.7822
    los, refl, d, dr = _two_ray_closed_form(pts, np.array([0.0, 0.0, 10.0]), f, 5.24, sigma)
    total = los + refl
    got_field = _cell_index(res.field, grid.shape)[0]
    got_gain = _cell_index(res.path_gain, grid.shape)[0].astype(np.float64)
    assert got_gain.shape == (4096,)
    tol_db = 0.01 if precision == "mixed" else 1e-4
    want_gain = np.abs(total) ** 2
    # cells away from two-ray interference nulls: dB bound; near a null the
    # field error is bounded by the constituent magnitudes
    scale = np.abs(los) + np.abs(refl)
    deep = np.abs(total) < 0.05 * scale
    assert np.all(_db(got_gain[~deep], want_gain[~deep]) <= tol_db)
    _check_cells(got_field, total, scale * (1.0 if precision == "mixed" else 1e-2))
    if precision != "mixed":
        return
    # per-path: LoS and reflection gains and delays (1 ps)
    p = res.paths
    rx = p.rx_id.cpu().numpy()
    cid = p.component_id.cpu().numpy()
    gain = p.path_gain.double().cpu().numpy()
    delay = p.delay_s.double().cpu().numpy()
    assert np.array_equal(np.sort(rx[cid == 0]), np.arange(4096))
    assert np.array_equal(np.sort(rx[cid == 1]), np.arange(4096))
    lo, rf = cid == 0, cid == 1
    assert np.all(_db(gain[lo], np.abs(los[rx[lo]]) ** 2) <= tol_db)
    assert np.all(_db(gain[rf], np.abs(refl[rx[rf]]) ** 2) <= tol_db)
    assert np.all(np.abs(delay[lo] - d[rx[lo]] / C0) <= 1e-12)
    assert np.all(np.abs(delay[rf] - dr[rx[rf]] / C0) <= 1e-12)


# ------------------------------------------------------------ urban canyon
def test_canyon_full_discovery_sampled_cells():
    scene, f = urban_canyon_scene()
    comps = {"los", "reflection", "diffraction"}
    res = solve(scene, Config(components=comps, max_depth=3, export_paths=True), reference_frequency_hz=f)
    grid = scene.receivers[0]
    n = grid.shape[0] * grid.shape[1]
    cells = (np.arange(256) * 257 + 13) % n  # 256 cells spread over rows and columns
    arrays = osolve.scene_arrays(scene, f)
    discovered = opar.discover(arrays, max_depth=3, rays=osolve.DISCOVERY_RAYS)
    assert discovered is not None  # 385 groups: the depth-2/3 chains come from discovery
    edge_visible = osolve.tx_edge_masks(arrays, f)
    chunks = opar.solve_cells(arrays, cells, discovered=discovered, edge_visible=edge_visible, components=comps,
                              max_depth=3, frequency=f)
    # oracle rows in canonical order for the sampled cells
    parts = []
    for sub_cells, out in chunks:
        r = out["rows"]
        for i in range(len(r["tx_id"])):
            parts.append((int(sub_cells[int(r["rx_id"][i])]), int(r["tx_id"][i]), int(r["component_id"][i]),
                          int(r["depth"][i]), tuple(int(x) for x in r["primitive_sequence"][i]),
                          int(r["edge_id"][i]), float(r["path_gain"][i]), complex(r["path_field"][i])))
    parts.sort(key=lambda x: x[0])  # canonical order is rx-major; within a cell it is already canonical
    p = res.paths
    rx = p.rx_id.cpu().numpy()
    sel = np.isin(rx, cells)
    got = _rows_key(p.tx_id.cpu().numpy()[sel], rx[sel], p.component_id.cpu().numpy()[sel], p.depth.cpu().numpy()[sel],
                    p.primitive_sequence.cpu().numpy()[sel], p.edge_id.cpu().numpy()[sel])
    want = [(t, r, c, d, s, e) for (r, t, c, d, s, e, _, _) in parts]
    assert len(want) > 500 and sum(1 for k in want if k[3] >= 2) > 20 and sum(1 for k in want if k[2] == 2) > 50
    extra, missing = sorted(set(got) - set(want)), sorted(set(want) - set(got))
    # Two kinds of row may differ between the FP32 solve and the FP64 oracle,
    # at most 2 rows or one per 500:
    # * a row at the existence floor (path gain below 1e-24 in the solver that
    #   keeps it, ~200 dB under the cells' paths): a UTD tail term whose
    #   stationary point lies far outside its edge, where FP32 cannot resolve
    #   the 1e-30 floor decision;
    # * a row whose visibility is marginal (the oracle's own blocked decision
    #   changes when a segment endpoint moves by 0.5 mm).
    differing = extra + missing
    assert len(differing) <= max(2, len(want) // 500), (extra[:6], missing[:6])
    gpu_gain = {k: float(x) for k, x in zip(got, p.path_gain.double().cpu().numpy()[sel])}
    oracle_gain = {(t, r, c, d, s, e): gn for (r, t, c, d, s, e, gn, _) in parts}
    for key in differing:
        g_key = gpu_gain.get(key, oracle_gain.get(key))
        assert g_key < 1e-24 or _marginal_visibility(arrays, key), ("not a floor or marginal case", key, g_key)
    keep_keys = set(got) & set(want)
    got_idx = [i for i, k in enumerate(got) if k in keep_keys]
    want_idx = [i for i, k in enumerate(want) if k in keep_keys]
    assert [got[i] for i in got_idx] == [want[i] for i in want_idx]
    parts = [parts[i] for i in want_idx]
    g = p.path_gain.double().cpu().numpy()[sel][got_idx]
    w = np.array([x[6] for x in parts])
    strong = w >= 1e-6 * w.max()
    assert np.all(_db(g[strong], w[strong]) <= 0.01)
    pf = torch.complex(p.field_real, p.field_imag).cpu().numpy()[sel][got_idx]
    wf = np.array([x[7] for x in parts])
    big = np.abs(wf) > 1e-3 * np.abs(wf).max()
    assert np.all(np.abs(np.angle(pf[big] / wf[big])) <= 1e-3)
    # coherent cell fields at the sampled cells without a differing row
    ok_cells = np.array([c for c in cells if all(k[1] != c for k in differing)])
    cells = ok_cells
    field = _cell_index(res.field, grid.shape)[0][cells]
    want_field = np.zeros(len(cells), dtype=np.complex128)
    scale = np.zeros(len(cells))
    pos = {int(c): i for i, c in enumerate(cells)}
    for (r, _, _, _, _, _, _, fld) in parts:
        if r in pos:
            want_field[pos[r]] += fld
            scale[pos[r]] += abs(fld)
    _check_cells(field, want_field, scale)


def _marginal_visibility(arrays, key, step=5e-4) -> bool:
    """True when one of the row's visibility segments changes its blocked
    decision if an endpoint moves by `step` along a coordinate axis (LoS and
    diffraction rows; the oracle's own geometry)."""
    from oracle import geom, utd

    t, r, c, d, seq, e = key
    S, R = arrays["tx_pos"][t], arrays["rx_pos"][r]
    tris = geom.Triangles(arrays["vertices"], arrays["faces"])
    F = tris.count
    if c == 0:
        segs = [(S, R, np.zeros(F, bool))]
    elif c == 2:
        eg = osolve.edge_table(arrays)
        out = utd.diffraction_field(S, R, arrays["tx_pol"][t], eg, e, arrays["face_mats"], 28e9)
        if out is None:
            return True
        qv = out[2]
        ign = np.zeros(F, bool)
        ign[eg["face0"][e]] = True
        if eg["face1"][e] >= 0:
            ign[eg["face1"][e]] = True
        segs = [(S, qv, ign), (qv, R, ign)]
    else:
        return False
    for p0, p1, ign in segs:
        base = geom.segment_blocked(tris, p0[None], p1[None], ign[None])[0]
        for end in (0, 1):
            for ax in range(3):
                for sgn in (-1.0, 1.0):
                    q0, q1 = p0.copy(), p1.copy()
                    (q0 if end == 0 else q1)[ax] += sgn * step
                    if geom.segment_blocked(tris, q0[None], q1[None], ign[None])[0] != base:
                        return True
    return False


# --------------------------------------------------------- depth 4 and 5
def _room():
    """A closed 8 x 6 x 4 m room (12 triangles, 6 walls), Tx and a few
    receivers inside: every chain up to depth 5 is enumerated exhaustively."""
    import torch as _t

    from witwin_channel_b200.scene import PhysicalMaterial, Scene, make_mesh_structure, make_receiver, make_transmitter
    from witwin_channel_b200.workloads import box_mesh

    v, fc = box_mesh(0.0, 0.0, 8.0, 6.0, 4.0)
    v = _t.as_tensor(v, dtype=_t.float32)
    fc = _t.as_tensor(fc, dtype=_t.int64)
    fc = fc[:, [0, 2, 1]]  # normals into the room
    room = make_mesh_structure(vertices=v, faces=fc, material=PhysicalMaterial(eps_r=4.0, sigma_e=0.02, thickness_m=0.2),
                               surface_id=1)
    return Scene(structures=[room], endpoints=[make_transmitter([2.1, 1.7, 1.3]), make_receiver([6.2, 4.1, 1.1]),
                                               make_receiver([5.3, 1.2, 2.7]), make_receiver([1.4, 4.6, 0.8])])


@pytest.mark.parametrize("depth", [4, 5])
def test_closed_room_depth_4_and_5(depth):
    scene = _room()
    f = 3.5e9
    res = solve(scene, Config(components={"los", "reflection"}, max_depth=depth, export_paths=True),
                reference_frequency_hz=f)
    ref = osolve.solve(osolve.scene_arrays(scene, f), components={"los", "reflection"}, max_depth=depth, frequency=f)
    from tests.test_gpu_parity import _compare_paths
    _compare_paths(res, ref)
    d = res.paths.depth.cpu().numpy()
    assert (d == depth).sum() > 0 and (d == depth - 1).sum() > 0


def test_discovered_chains_depth_5():
    scene, f = scenes.small_city(n_boxes=16, seed=5, grid=(5, 4), spacing=9.0)
    from witwin_channel_b200 import engine
    from witwin_channel_b200.compiler import compile_scene
    from witwin_channel_b200.deterministic import _endpoints

    rays = 16384
    device = torch.device("cuda", torch.cuda.current_device())
    compiled = compile_scene(scene, device)
    ep = _endpoints(scene, device)
    mats = compiled.material_tables([f], device)
    out = engine.run_solve(compiled, ep, mats, [f], components=engine.component_bits({"reflection"}), max_depth=5,
                           coherent=True, want_rows=True, discovery_rays=rays)
    sel = engine.select_rows(out["rows"], 5, None, "global")
    dec = engine.decode_rows(out["rows"], sel)
    got = _rows_key(dec["tx_id"].cpu(), dec["rx_id"].cpu(), dec["component_id"].cpu(), dec["depth"].cpu(),
                    dec["seq"][:, :5].cpu(), dec["edge_id"].cpu())
    arrays = osolve.scene_arrays(scene, f)
    discovered = opar.discover(arrays, max_depth=5, rays=rays)
    ref = osolve.solve(arrays, components={"reflection"}, max_depth=5, frequency=f, discovered=discovered)
    r = ref["rows"]
    want = _rows_key(r["tx_id"], r["rx_id"], r["component_id"], r["depth"], r["primitive_sequence"], r["edge_id"])
    assert sum(1 for k in want if k[3] >= 4) > 0
    assert got == want


# ---------------------------------------------------------- gradient run
def test_gradient_run_sampled_cells_fd():
    run = gradient_run()
    scene, freq_t, target = run["scene"], run["frequency"], run["target"]
    grid = scene.receivers[0]
    n = grid.shape[0] * grid.shape[1]
    res = solve(scene, Config(components=run["components"], max_depth=3, ad_mode="vjp", export_paths=True),
                reference_frequency_hz=freq_t)
    # cells with paths in both maps (gain above 1e-20, i.e. not made of tail
    # terms at the existence floor) and no strong coherent cancellation
    # (|sum f| >= 0.5 sum |f|: the log-gain loss divides by the cell gain),
    # spread over the grid
    pg_flat = _cell_index(res.path_gain.detach(), grid.shape)[0]
    tg_flat = _cell_index(target, grid.shape)[0]
    p0 = res.paths
    fr = torch.complex(p0.field_real, p0.field_imag).detach().cpu().numpy().astype(np.complex128)
    rx0 = p0.rx_id.cpu().numpy()
    coh = np.zeros(n, dtype=np.complex128)
    mag = np.zeros(n)
    np.add.at(coh, rx0, fr)
    np.add.at(mag, rx0, np.abs(fr))
    ratio = np.abs(coh) / np.maximum(mag, 1e-300)
    cand = np.nonzero((pg_flat > 1e-20) & (tg_flat > 1e-20) & (ratio >= 0.5))[0]
    cells = cand[np.linspace(0, len(cand) - 1, 48).astype(np.int64)]
    # the sub-loss over those cells (grid layout: (T, cols, rows) with cell = row*cols + col)
    rows, cols = grid.shape
    ri, ci = cells // cols, cells % cols
    sub = res.path_gain[0, ci, ri]
    tsub = target[0, ci, ri]
    loss = log_mse(sub, tsub)
    loss.backward()
    lv = run["leaves"]
    p = res.paths
    keep = np.isin(p.rx_id.cpu().numpy(), cells)
    table = {"tx_id": p.tx_id.cpu().numpy()[keep], "rx_id": p.rx_id.cpu().numpy()[keep],
             "component_id": p.component_id.cpu().numpy()[keep], "depth": p.depth.cpu().numpy()[keep],
             "primitive_sequence": p.primitive_sequence.cpu().numpy()[keep], "edge_id": p.edge_id.cpu().numpy()[keep]}
    f0 = float(freq_t.detach())
    arrays = osolve.scene_arrays(scene, f0)
    tgt = tg_flat[cells].astype(np.float64)
    # the differentiable concrete (the boxes' shared material; the ground has its own)
    mi = int(arrays["face_material"][arrays["face_structure"] == 1][0])

    def oracle_pg(arr, f):
        fields = oadj.fixed_topology_fields(arr, table, f)
        return oadj.cell_path_gain(fields, table, 1, n)[0][cells]

    def oracle_loss(arr, f):
        dlt = np.log10(oracle_pg(arr, f)) - np.log10(tgt)
        return float(np.mean(dlt * dlt))

    # the two losses are the same function of the same cells: equal at the base point
    pg_gpu = sub.detach().double().cpu().numpy()
    pg_ora = oracle_pg(arrays, f0)
    np.testing.assert_allclose(pg_ora, pg_gpu, rtol=1e-4)
    np.testing.assert_allclose(oracle_loss(arrays, f0), float(loss), rtol=1e-4)

    # parameters: materials, frequency, Tx, and the 16 moved-box vertex
    # coordinates with the largest gradients
    vert_off = {}
    off = 0
    for s, st in enumerate(scene.structures):
        vert_off[s] = off
        off += st.vertices.shape[0]
    vgrads = []
    for s in run["moved_structures"]:
        g = scene.structures[s].vertices.grad
        for v in range(g.shape[0]):
            for c in range(3):
                vgrads.append((abs(float(g[v, c])), s, v, c, float(g[v, c])))
    vgrads.sort(reverse=True)
    params = [("eps_r", float(lv["eps_r"].grad)), ("sigma_e", float(lv["sigma_e"].grad)),
              ("frequency", float(freq_t.grad))]
    params += [(("tx", c), float(lv["tx"].grad[c])) for c in range(3)]
    params += [(("vertex", s, v, c), gv) for (_, s, v, c, gv) in vgrads[:16]]
    assert len(params) >= 22

    def perturb(key, h):
        a = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in arrays.items()}
        a["face_mats"] = {k: v.copy() for k, v in arrays["face_mats"].items()}
        a["material_layers"] = list(arrays["material_layers"])
        fq = f0
        if key in ("eps_r", "sigma_e"):
            a["face_mats"][key][a["face_material"] == mi] += h
            th, er, sg, mr = a["material_layers"][mi]
            if key == "eps_r":
                er = er.copy(); er[0] += h
            else:
                sg = sg.copy(); sg[0] += h
            a["material_layers"][mi] = (th, er, sg, mr)
        elif key == "frequency":
            fq = f0 + h
            a = osolve.scene_arrays(scene, fq)  # the ground's conductivity follows the frequency
        elif key[0] == "tx":
            a["tx_pos"] = a["tx_pos"].copy(); a["tx_pos"][0, key[1]] += h
        else:
            _, s, v, c = key
            a["vertices"] = a["vertices"].copy(); a["vertices"][vert_off[s] + v, c] += h
        return a, fq

    def value(key):
        if key in ("eps_r", "sigma_e"):
            return arrays["face_mats"][key][arrays["face_material"] == mi][0]
        if key == "frequency":
            return f0
        if key[0] == "tx":
            return arrays["tx_pos"][0, key[1]]
        _, s, v, c = key
        return arrays["vertices"][vert_off[s] + v, c]

    bad = []
    strong = 0
    report = []
    for key, ours in params:
        def central(step):
            ap, fp = perturb(key, step)
            am, fm = perturb(key, -step)
            return (oracle_loss(ap, fp) - oracle_loss(am, fm)) / (2 * step)

        # relative step 1e-4, then 1e-5 and 1e-6 where the loss is not smooth
        # over the larger step (a centimetre move of a 100 m coordinate can
        # carry a sampled cell's path across a shadow boundary or the UTD
        # window cutoff)
        smooth = False
        for rel in (1e-4, 1e-5, 1e-6):
            h = rel * max(abs(float(value(key))), 1.0)
            d1, d2, d4 = central(h), central(h / 2), central(h / 4)
            r1, r2 = (4 * d2 - d1) / 3, (4 * d4 - d2) / 3
            if np.isfinite([d1, d2, d4]).all() and abs(r1 - r2) <= 1e-3 * abs(r2) + 1e-12:
                smooth = True
                break
        report.append((key, ours, r2, abs(r1 - r2), rel))
        if not smooth:
            # a path of a sampled cell appears or vanishes within every step
            # (a topology change): not a derivative check
            continue
        if abs(r2) > 0:
            strong += 1
        if abs(ours - r2) > 1e-4 * abs(r2) + 1e-9 * max(abs(x[1]) for x in params):
            bad.append((key, ours, r2))
    assert not bad, (bad[:6], report)
    assert strong >= 18, report
