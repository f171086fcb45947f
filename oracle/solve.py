"""End-to-end FP64 deterministic solve (oracle).

Follows ``witwin/channel/propagation/enumerated.py:549-836`` (component order
LoS -> reflection order 1 -> reflection depth 2..D -> diffraction ->
transmission), ``propagation/topology.py:408-466`` plus
``native/channel/kernels/evaluated_paths.cu:560-760`` (canonical sort, dedup,
max_paths), ``propagation/fields.py:949-1236`` (field evaluation) and
``native/channel/kernels/deterministic.cu:829-970`` (accumulation).

Test infrastructure only: the tests, the smoke check and the benchmark's CPU
baseline call it as the checker; the product path never does.
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import em, geom, utd

ORDER1_EXHAUSTIVE_GROUP_LIMIT = 4096  # interactions/reflection.py:30
MAX_MULTIBOUNCE_FACE_SEQUENCES = 100_000  # interactions/reflection.py:31
DISCOVERY_RAYS = 262_144  # interactions/reflection.py:34
PEC_SIGMA = 1.0e9


def _value(v, f):
    if callable(v) and not hasattr(v, "detach"):
        v = v(f)
    if hasattr(v, "detach"):
        v = float(v.detach())
    return float(v)


def scene_arrays(scene, frequency: float) -> dict:
    """Flatten a (duck-typed) scene into float64 arrays at ``frequency``."""
    verts, faces, fstruct, fsurf, fmat = [], [], [], [], []
    materials = []
    mat_index: dict[int, int] = {}
    offset = 0
    for s_idx, st in enumerate(scene.structures):
        v = st.vertices.detach().cpu().numpy().astype(np.float32).astype(np.float64)
        f = st.faces.detach().cpu().numpy().astype(np.int64) + offset
        verts.append(v)
        faces.append(f)
        fstruct.append(np.full(f.shape[0], s_idx))
        sid = st.surface_id if st.surface_id is not None else s_idx
        fsurf.append(np.full(f.shape[0], int(sid)))
        key = id(st.material)
        if key not in mat_index:
            mat_index[key] = len(materials)
            materials.append(st.material)
        fmat.append(np.full(f.shape[0], mat_index[key]))
        offset += v.shape[0]
    m = len(materials)
    tab = {k: np.zeros(m) for k in ("eps_r", "sigma_e", "mu_r", "gain", "thickness")}
    layers = []
    volumetric = np.zeros(m, dtype=bool)
    for i, mat in enumerate(materials):
        pec = getattr(mat, "conductor_model", None) == "perfect"
        stack = mat.stack() if hasattr(mat, "stack") else mat.layers
        th = np.array([_value(l.thickness_m, frequency) for l in stack])
        er = np.array([_value(l.eps_r, frequency) for l in stack])
        sg = np.array([PEC_SIGMA if pec else _value(l.sigma_e, frequency) for l in stack])
        mr = np.array([_value(l.mu_r, frequency) for l in stack])
        if pec:
            sg = np.maximum(sg, PEC_SIGMA)
        layers.append((th, er, sg, mr))
        tab["eps_r"][i] = er[0]
        tab["sigma_e"][i] = sg[0]
        tab["mu_r"][i] = mr[0]
        tab["thickness"][i] = th[0]
        tab["gain"][i] = _value(mat.gain, frequency)
        volumetric[i] = getattr(mat, "geometry_mode", "thin_sheet") == "volumetric"
    V = np.concatenate(verts) if verts else np.zeros((0, 3))
    Fc = np.concatenate(faces) if faces else np.zeros((0, 3), dtype=np.int64)
    fm = np.concatenate(fmat) if fmat else np.zeros(0, dtype=np.int64)
    face_tab = {k: v[fm] for k, v in tab.items()}
    tx = scene.transmitters
    rx = scene.receivers
    tx_pos = np.stack([t.position.detach().cpu().numpy() for t in tx]).astype(np.float32).astype(np.float64) if tx else np.zeros((0, 3))
    tx_pow = np.array([_value(t.power_w, frequency) for t in tx])
    tx_pol = np.stack([t.polarization.detach().cpu().numpy() for t in tx]).astype(np.float32).astype(np.float64) if tx else np.zeros((0, 3))
    rx_pos, rx_pol = [], []
    for r in rx:
        if hasattr(r, "points") and hasattr(r, "shape") and hasattr(r, "spacing"):
            pts = _grid_points_f32(r)
        else:
            pts = r.position.detach().cpu().numpy().reshape(1, 3).astype(np.float32)
        rx_pos.append(pts.astype(np.float64))
        rx_pol.append(np.broadcast_to(r.polarization.detach().cpu().numpy().astype(np.float32).astype(np.float64), pts.shape))
    return {
        "vertices": V,
        "faces": Fc,
        "face_structure": np.concatenate(fstruct) if fstruct else np.zeros(0, dtype=np.int64),
        "face_surface": np.concatenate(fsurf) if fsurf else np.zeros(0, dtype=np.int64),
        "face_material": fm,
        "face_mats": face_tab,
        "material_layers": layers,
        "material_volumetric": volumetric,
        "tx_pos": tx_pos,
        "tx_power": tx_pow,
        "tx_pol": tx_pol,
        "rx_pos": np.concatenate(rx_pos) if rx_pos else np.zeros((0, 3)),
        "rx_pol": np.concatenate(rx_pol) if rx_pol else np.zeros((0, 3)),
        "edge_policy": scene.metadata.get("imported_edge_policy") if hasattr(scene, "metadata") else None,
    }


def _grid_points_f32(grid) -> np.ndarray:
    """Float32 grid points exactly as ``los.cu:391-420`` forms them."""
    rows, cols = grid.shape
    o = grid.origin.detach().cpu().numpy().astype(np.float32)
    xa = grid.x_axis.detach().cpu().numpy().astype(np.float32)
    ya = grid.y_axis.detach().cpu().numpy().astype(np.float32)
    s0, s1 = np.float32(grid.spacing[0]), np.float32(grid.spacing[1])
    r = np.repeat(np.arange(rows, dtype=np.float32), cols) * s0
    c = np.tile(np.arange(cols, dtype=np.float32), rows) * s1
    pts = o[None, :] + xa[None, :] * r[:, None]
    pts = pts.astype(np.float32) + ya[None, :] * c[:, None]
    return pts.astype(np.float32)


@dataclass
class Rows:
    tx: list = field(default_factory=list)
    rx: list = field(default_factory=list)
    cid: list = field(default_factory=list)
    depth: list = field(default_factory=list)
    seq: list = field(default_factory=list)
    edge: list = field(default_factory=list)
    hits: list = field(default_factory=list)
    normals: list = field(default_factory=list)
    field_xyz: list = field(default_factory=list)  # diffraction only (unit excitation)
    length: list = field(default_factory=list)

    def add(self, **kw):
        for k, v in kw.items():
            getattr(self, k).append(v)


def _face_sequence_count(g: int, d: int) -> int:
    if d > 1:
        return 0 if g <= 1 else g * (g - 1) ** (d - 1)
    return g


def _exhaustive_chains(g: int, d: int) -> list[tuple[int, ...]]:
    """Adjacent-distinct sequences in the order of ``paths.cu:364-406``."""
    out = []
    total = _face_sequence_count(g, d)
    base = g - 1 if d > 1 else g
    for value in range(total):
        div = base ** (d - 1) if d > 1 else 1
        prev = -1
        digits = []
        v = value
        for col in range(d):
            if d > 1:
                raw = v // div
                v -= raw * div
                div = div // base if div > 1 else 1
                digit = raw if col == 0 else (raw if raw < prev else raw + 1)
                prev = digit
            else:
                digit = v
            digits.append(digit)
        out.append(tuple(digits))
    return out


def discovery_groups(arrays: dict, *, max_depth: int) -> np.ndarray | None:
    """Face -> coplanar group map when the chain plan needs discovery at some
    depth (``interactions/reflection.py:186-293``), else ``None``."""
    V, Fc = arrays["vertices"], arrays["faces"]
    if Fc.shape[0] == 0 or max_depth < 1:
        return None
    groups = geom.coplanar_groups(V[Fc[:, 0]], geom.face_normals_f32(V, Fc), arrays["face_surface"])
    G = groups["group_count"]
    need = G > ORDER1_EXHAUSTIVE_GROUP_LIMIT or (max_depth >= 2 and not all(
        _face_sequence_count(G, d) <= MAX_MULTIBOUNCE_FACE_SEQUENCES for d in range(2, max_depth + 1)))
    return groups["face_group_id"] if need else None


def discover_directions(arrays: dict, face_group_id: np.ndarray, tx: int, directions: np.ndarray, *,
                        max_depth: int) -> np.ndarray:
    """Group chains of the bounce paths launched from transmitter ``tx`` along
    ``directions`` (``(N, max_depth)``, ``-1`` after a miss)."""
    V, Fc = arrays["vertices"], arrays["faces"]
    prims = geom.trace_reflections(geom.Triangles(V, Fc), geom.face_normals(V, Fc), arrays["tx_pos"][tx], directions,
                                   max(max_depth, 1))
    return np.where(prims >= 0, face_group_id[np.maximum(prims, 0)], -1)


def discover(arrays: dict, *, max_depth: int, discovery_rays: int = DISCOVERY_RAYS) -> list | None:
    """Per-transmitter discovered group chains (``interactions/reflection.py:541-569``),
    or ``None`` when the exhaustive plan applies at every depth."""
    face_group_id = discovery_groups(arrays, max_depth=max_depth)
    if face_group_id is None:
        return None
    dirs = geom.fibonacci_directions(discovery_rays)
    return [discover_directions(arrays, face_group_id, t, dirs, max_depth=max_depth)
            for t in range(arrays["tx_pos"].shape[0])]


def solve(arrays: dict, *, components, max_depth: int, coherent: bool = True, max_paths=None,
          max_paths_scope: str = "global", frequency: float, discovery_rays: int = DISCOVERY_RAYS,
          edge_policy=None, discovered: list | None = None, edge_visible: list | None = None) -> dict:
    """Full deterministic solve.  ``discovered`` (per transmitter, from
    ``discover``) and ``edge_visible`` (per transmitter, from
    ``tx_edge_masks``) let a caller compute the per-transmitter work once and
    reuse it across receiver subsets."""
    V, Fc = arrays["vertices"], arrays["faces"]
    fm = arrays["face_mats"]
    tx_pos, tx_pow, tx_pol = arrays["tx_pos"], arrays["tx_power"], arrays["tx_pol"]
    rx_pos, rx_pol = arrays["rx_pos"], arrays["rx_pol"]
    T, R = tx_pos.shape[0], rx_pos.shape[0]
    F = Fc.shape[0]
    components = set(components)
    width = max(int(max_depth), 0)
    tris = geom.Triangles(V, Fc)
    normals = geom.face_normals(V, Fc) if F else np.zeros((0, 3))
    rows = Rows()
    has_struct = F > 0
    groups = geom.coplanar_groups(V[Fc[:, 0]], geom.face_normals_f32(V, Fc), arrays["face_surface"]) if F else None
    k = em.wave_number(frequency)

    def group_planes(chain):
        return [(V[Fc[groups["representative_faces"][g], 0]], normals[groups["representative_faces"][g]]) for g in chain]

    # ---- LoS -------------------------------------------------------------
    if "los" in components:
        for t in range(T):
            p0 = np.repeat(tx_pos[t][None], R, axis=0)
            blocked = geom.segment_blocked(tris, p0, rx_pos) if has_struct else np.zeros(R, dtype=bool)
            for r in np.nonzero(~blocked)[0]:
                rows.add(tx=t, rx=int(r), cid=0, depth=0, seq=(), edge=-1, hits=(), normals=(), field_xyz=None,
                         length=float(np.linalg.norm(rx_pos[r] - tx_pos[t])))

    # ---- reflection --------------------------------------------------------
    discovered_all = discovered
    if "reflection" in components and max_depth >= 1 and has_struct and R > 0:
        G = groups["group_count"]
        face_group = groups["face_group_id"]
        for t in range(T):
            S = tx_pos[t]
            discovered = None
            need_disc_o1 = G > ORDER1_EXHAUSTIVE_GROUP_LIMIT
            need_disc_mb = max_depth >= 2 and not all(
                _face_sequence_count(G, d) <= MAX_MULTIBOUNCE_FACE_SEQUENCES for d in range(2, max_depth + 1))
            chain_sets = {}
            if need_disc_o1 or need_disc_mb:
                if discovered_all is not None:
                    discovered = discovered_all[t]
                else:
                    dirs = geom.fibonacci_directions(discovery_rays)
                    prims = geom.trace_reflections(tris, normals, S, dirs, max(max_depth, 1))
                    discovered = np.where(prims >= 0, face_group[np.maximum(prims, 0)], -1)
            if need_disc_o1:
                firsts = np.unique(discovered[discovered[:, 0] >= 0, 0])
                chain_sets[1] = [(int(g),) for g in firsts]
            else:
                chain_sets[1] = [(g,) for g in range(G)]
            for d in range(2, max_depth + 1):
                if need_disc_mb:
                    reached = discovered[:, d - 1] >= 0
                    uniq = np.unique(discovered[reached][:, :d], axis=0) if reached.any() else np.zeros((0, d), dtype=np.int64)
                    chain_sets[d] = [tuple(int(x) for x in c) for c in uniq]
                else:
                    chain_sets[d] = _exhaustive_chains(G, d)
            for d in range(1, max_depth + 1):
                for chain in chain_sets[d]:
                    planes = group_planes(chain)
                    images = geom.image_chain(S, planes)
                    for r in range(R):
                        hits = geom.back_project(rx_pos[r], images, planes)
                        if hits is None:
                            continue
                        faces_res = []
                        for kk, g in enumerate(chain):
                            found = -1
                            for f in groups["members"][g]:
                                if geom.point_in_face(hits[kk], V, Fc, normals, f):
                                    found = f
                                    break
                            if found < 0:
                                break
                            faces_res.append(found)
                        if len(faces_res) != d:
                            continue
                        pts = [S] + list(hits) + [rx_pos[r]]
                        ok = True
                        for sidx in range(d + 1):
                            ign = np.zeros((1, F), dtype=bool)
                            if sidx > 0:
                                ign[0, face_group == chain[sidx - 1]] = True
                            if sidx < d:
                                ign[0, face_group == chain[sidx]] = True
                            if np.linalg.norm(pts[sidx + 1] - pts[sidx]) <= 0.0:
                                ok = False
                                break
                            if geom.segment_blocked(tris, pts[sidx][None], pts[sidx + 1][None], ign)[0]:
                                ok = False
                                break
                        if not ok:
                            continue
                        length = float(np.linalg.norm(rx_pos[r] - images[-1]))
                        rows.add(tx=t, rx=r, cid=1, depth=d, seq=tuple(faces_res), edge=-1,
                                 hits=tuple(hits), normals=tuple(normals[f] for f in faces_res), field_xyz=None,
                                 length=length)

    # ---- diffraction --------------------------------------------------------
    diff_vector = np.zeros((T, R, 3), dtype=np.complex128)
    if "diffraction" in components and max_depth >= 1 and has_struct and R > 0:
        eg = edge_table(arrays, edge_policy)
        wavelength = em.SPEED_OF_LIGHT / frequency
        for t in range(T):
            S = tx_pos[t]
            for e in np.nonzero(eg["selected"])[0]:
                inside, _ = utd.source_exterior(S, eg, e)
                if not inside:
                    continue
                if edge_visible is not None:
                    if not edge_visible[t][e]:
                        continue
                elif not tx_edge_visible(tris, S, eg, e, wavelength):
                    continue
                for r in range(R):
                    out = utd.diffraction_field(S, rx_pos[r], tx_pol[t], eg, e, fm, frequency)
                    if out is None:
                        continue
                    fxyz, q, q_vis, s_p, s = out
                    powered = fxyz * np.sqrt(max(tx_pow[t], 0.0))
                    if float(np.sum(np.abs(powered) ** 2)) < utd.GAIN_FLOOR:
                        continue
                    ign = np.zeros((1, F), dtype=bool)
                    ign[0, eg["face0"][e]] = True
                    if eg["face1"][e] >= 0:
                        ign[0, eg["face1"][e]] = True
                    if geom.segment_blocked(tris, S[None], q_vis[None], ign)[0]:
                        continue
                    if geom.segment_blocked(tris, q_vis[None], rx_pos[r][None], ign)[0]:
                        continue
                    rows.add(tx=t, rx=r, cid=2, depth=1, seq=(), edge=int(e), hits=(q,), normals=(np.zeros(3),),
                             field_xyz=fxyz, length=float(s_p + s))
                    diff_vector[t, r] += powered

    # ---- transmission ---------------------------------------------------------
    overflow = 0
    if "transmission" in components and max_depth >= 1 and has_struct and R > 0:
        for t in range(T):
            p0 = np.repeat(tx_pos[t][None], R, axis=0)
            all_hits = geom.segment_hits(tris, p0, rx_pos, groups["face_group_id"])
            for r in range(R):
                hits = all_hits[r]
                if not hits:
                    continue
                if len(hits) > max_depth:
                    overflow += 1
                    continue
                if any(arrays["material_volumetric"][arrays["face_material"][f]] for _, f in hits):
                    continue
                d = rx_pos[r] - tx_pos[t]
                pts = tuple(tx_pos[t] + tt * d for tt, _ in hits)
                rows.add(tx=t, rx=r, cid=5, depth=len(hits), seq=tuple(f for _, f in hits), edge=-1,
                         hits=pts, normals=tuple(normals[f] for _, f in hits), field_xyz=None,
                         length=float(np.linalg.norm(d)))

    table = _finish(rows, arrays, width, frequency, max_paths, max_paths_scope, T, R)
    acc = accumulate(table, T, R, coherent)
    acc["diffraction_vector_power"] = np.sum(np.abs(diff_vector) ** 2, axis=-1)
    acc["transmission_overflow"] = overflow
    acc["rows"] = table
    return acc


def edge_table(arrays: dict, edge_policy=None) -> dict:
    """Selected diffraction edges with their geometry (``diffraction.cu:803-900``,
    ``scene/resources.py:356-405``)."""
    V, Fc = arrays["vertices"], arrays["faces"]
    rec = geom.edge_records(Fc, arrays["face_structure"])
    pol = edge_policy
    return geom.edge_geometry(
        V, Fc, geom.face_normals(V, Fc), rec,
        boundary_policy=getattr(pol, "boundary_edge_policy", "half_plane") or "half_plane",
        vertical_only=getattr(pol, "edge_selection_mode", "all_edges") == "vertical_only",
        vertical_ratio=getattr(pol, "vertical_ratio", 0.7),
    )


def tx_edge_masks(arrays: dict, frequency: float, edge_policy=None) -> list:
    """Per transmitter, the Tx-visibility prefilter of every edge (False for
    unselected edges)."""
    V, Fc = arrays["vertices"], arrays["faces"]
    tris = geom.Triangles(V, Fc)
    eg = edge_table(arrays, edge_policy)
    wavelength = em.SPEED_OF_LIGHT / frequency
    out = []
    for t in range(arrays["tx_pos"].shape[0]):
        mask = np.zeros(len(eg["selected"]), dtype=bool)
        for e in np.nonzero(eg["selected"])[0]:
            if utd.source_exterior(arrays["tx_pos"][t], eg, e)[0]:
                mask[e] = tx_edge_visible(tris, arrays["tx_pos"][t], eg, e, wavelength)
        out.append(mask)
    return out


def tx_edge_visible(tris, S, eg, e, wavelength) -> bool:
    """Tx-visible edge prefilter: any of ``clamp(ceil(L/lambda), 4, 16)``
    sample points on the edge (offset along the exterior bisector) is
    unoccluded from the source (``rayd/diffraction.cpp:380-403``; count per
    the reference's design doc F6)."""
    L = eg["length"][e]
    n = int(min(max(np.ceil(L / wavelength), 4), 16))
    e_hat, t0, _ = utd.edge_frame(eg, e)
    bis = utd.exterior_bisector(eg, e)
    c = eg["edge_pos"][e]
    ts = -0.5 * L + (np.arange(n) + 0.5) / n * L
    pts = c[None] + ts[:, None] * e_hat[None] + utd.RAY_BIAS * bis[None]
    F = tris.count
    ign = np.zeros((n, F), dtype=bool)
    ign[:, eg["face0"][e]] = True
    if eg["face1"][e] >= 0:
        ign[:, eg["face1"][e]] = True
    blocked = geom.segment_blocked(tris, np.repeat(S[None], n, axis=0), pts, ign)
    return bool((~blocked).any())


def _finish(rows: Rows, arrays, width, frequency, max_paths, scope, T, R) -> dict:
    K = len(rows.tx)
    tx = np.asarray(rows.tx, dtype=np.int64)
    rx = np.asarray(rows.rx, dtype=np.int64)
    cid = np.asarray(rows.cid, dtype=np.int64)
    depth = np.asarray(rows.depth, dtype=np.int64)
    edge = np.asarray(rows.edge, dtype=np.int64)
    seq = np.full((K, width), -1, dtype=np.int64)
    for i, s in enumerate(rows.seq):
        seq[i, : len(s)] = s
    prim = np.where(np.isin(cid, (1, 5)), seq[:, 0] if width > 0 else -1, -1) if K else np.zeros(0, dtype=np.int64)
    length = np.asarray(rows.length, dtype=np.float64)
    keep = select_records(tx, rx, cid, depth, edge, seq, length, max_paths=max_paths, scope=scope)
    out = _evaluate(rows, keep, arrays, width, frequency)
    out.update({
        "tx_id": tx[keep], "rx_id": rx[keep], "component_id": cid[keep], "depth": depth[keep],
        "edge_id": edge[keep], "primitive_id": prim[keep], "primitive_sequence": seq[keep],
    })
    fmid = arrays["face_material"]
    ms = np.where(out["primitive_sequence"] >= 0, fmid[np.maximum(out["primitive_sequence"], 0)] if fmid.size else -1, -1)
    out["material_sequence"] = ms
    out["material_id"] = np.where(out["primitive_id"] >= 0, fmid[np.maximum(out["primitive_id"], 0)] if fmid.size else -1, -1)
    return out


def select_records(tx, rx, cid, depth, edge, seq, length, *, max_paths=None, scope="global") -> np.ndarray:
    """Canonical order, identity dedup and max_paths over path records
    (int64 arrays; ``seq`` is ``(K, width)`` with -1 padding).  Returns the
    kept record indices in canonical order.

    * order: (rx, tx, depth, component, seq[0..w-1], primitive, edge)
      ascending, stable (``evaluated_paths.cu:669-710``);
    * dedup: rows with one identity (tx, rx, per-slot event type and object
      id) keep the shortest, the first on ties; a NaN length drops the group
      (``evaluated_paths.cu:127-309``);
    * max_paths: a global prefix, or the first max_paths rows of each
      (rx, tx) pair."""
    K = len(tx)
    width = seq.shape[1] if seq.ndim == 2 else 0
    prim = np.where(np.isin(cid, (1, 5)), seq[:, 0] if width > 0 else -1, -1) if K else np.zeros(0, dtype=np.int64)
    keys = [edge, prim] + [seq[:, c] for c in range(width - 1, -1, -1)] + [cid, depth, tx, rx]
    order = np.lexsort(keys) if K else np.zeros(0, dtype=np.int64)
    keep = []
    i = 0
    while i < len(order):
        j = i
        ident = _identity(order[i], tx, rx, cid, depth, edge, seq, width)
        while j + 1 < len(order) and _identity(order[j + 1], tx, rx, cid, depth, edge, seq, width) == ident:
            j += 1
        grp = order[i: j + 1]
        lens = length[grp]
        if not np.any(np.isnan(lens)):
            keep.append(grp[int(np.argmin(lens))])
        i = j + 1
    keep = np.asarray(keep, dtype=np.int64)
    if max_paths is not None:
        if scope == "global":
            keep = keep[:max_paths]
        else:
            sel = []
            counts = {}
            for r in keep:
                key = (rx[r], tx[r])
                counts[key] = counts.get(key, 0) + 1
                if counts[key] <= max_paths:
                    sel.append(r)
            keep = np.asarray(sel, dtype=np.int64)
    return keep


def _identity(r, tx, rx, cid, depth, edge, seq, width):
    """(tx, rx, per-slot event type and object id): evaluated_paths.cu:127-209."""
    c, d = int(cid[r]), int(depth[r])
    slots = []
    for s in range(width):
        if c == 1 and s < d:
            et = 1
        elif c == 2 and d > 0 and s == 0:
            et = 2
        elif c == 5 and s < d:
            et = 4
        else:
            et = 0
        if et == 0:
            obj = -1
        elif c == 2 and s == 0:
            obj = int(edge[r])
        else:
            obj = int(seq[r, s])
        slots.append((et, obj))
    return (int(tx[r]), int(rx[r]), tuple(slots))


def _evaluate(rows: Rows, keep, arrays, width, frequency) -> dict:
    K = len(keep)
    fm = arrays["face_mats"]
    tx_pos, tx_pow, tx_pol = arrays["tx_pos"], arrays["tx_power"], arrays["tx_pol"]
    rx_pos, rx_pol = arrays["rx_pos"], arrays["rx_pol"]
    out = {
        "path_length_m": np.zeros(K), "delay_s": np.zeros(K), "path_gain": np.zeros(K),
        "path_field": np.zeros(K, dtype=np.complex128), "coefficient": np.zeros(K, dtype=np.complex128),
        "field_xyz": np.zeros((K, 3), dtype=np.complex128), "field_direction": np.zeros((K, 3)),
        "interaction_positions": np.zeros((K, width, 3)), "interaction_normals": np.zeros((K, width, 3)),
    }
    for i, r in enumerate(keep):
        t, x, c, d = rows.tx[r], rows.rx[r], rows.cid[r], rows.depth[r]
        S, Rx = tx_pos[t][None], rx_pos[x][None]
        P = np.array([tx_pow[t]])
        pt, pr = tx_pol[t][None], rx_pol[x][None]
        for s in range(min(len(rows.hits[r]), width)):
            out["interaction_positions"][i, s] = rows.hits[r][s]
            out["interaction_normals"][i, s] = rows.normals[r][s]
        if c == 0:
            ev = em.free_space(S, Rx, P, pt, pr, frequency)
        elif c == 1:
            f = np.asarray(rows.seq[r])
            pos = np.asarray(rows.hits[r])[None]
            nrm = np.asarray(rows.normals[r])[None]
            ev = em.reflection_sequence(S, Rx, pos, nrm, P, pt, pr, fm["eps_r"][f][None], fm["sigma_e"][f][None],
                                        fm["mu_r"][f][None], fm["gain"][f][None], fm["thickness"][f][None], frequency)
            # the path length is the image distance (FP64), equal to the segment sum
            ev["path_length_m"] = np.array([rows.length[r]])
            ev["delay_s"] = ev["path_length_m"] / em.SPEED_OF_LIGHT
        elif c == 5:
            f = np.asarray(rows.seq[r])
            nrm = np.asarray(rows.normals[r])[None]
            mid = arrays["face_material"][f][None]
            ev = em.transmission_sequence(S, Rx, nrm, mid, np.array([d]), P, pt, pr, arrays["material_layers"], frequency)
        elif c == 2:
            q = rows.hits[r][0]
            arrival = em.safe_normalize((Rx - q[None]), np.array([[0.0, 0.0, 1.0]]))
            powered = rows.field_xyz[r][None] * np.sqrt(max(tx_pow[t], 0.0))
            pj = em.project_complex3(powered, arrival, pr)
            amp = np.sqrt(max(tx_pow[t], 1e-30))
            ev = {
                "field_vector": powered / amp,
                "coefficient": pj["coefficient"] / amp,
                "path_field": pj["coefficient"],
                "path_gain": pj["path_gain"],
                "path_length_m": np.array([rows.length[r]]),
                "delay_s": np.array([rows.length[r] / em.SPEED_OF_LIGHT]),
                "direction": arrival,
            }
        out["path_length_m"][i] = ev["path_length_m"][0]
        out["delay_s"][i] = ev["delay_s"][0]
        out["path_gain"][i] = ev["path_gain"][0]
        out["path_field"][i] = ev["path_field"][0]
        out["coefficient"][i] = ev["coefficient"][0]
        out["field_xyz"][i] = ev["field_vector"][0]
        out["field_direction"][i] = ev["direction"][0]
    out["phase_rad"] = np.mod(-np.angle(out["path_field"]), 2.0 * np.pi)
    return out


SLOT = {0: 0, 1: 1, 2: 2, 5: 3}


def accumulate(table: dict, T: int, R: int, coherent: bool) -> dict:
    """Six-slot accumulation and finalisation (``deterministic.cu:829-970``)."""
    power = np.zeros((6, T, R))
    fieldc = np.zeros((6, T, R), dtype=np.complex128)
    for i in range(len(table["tx_id"])):
        s = SLOT[int(table["component_id"][i])]
        t, r = int(table["tx_id"][i]), int(table["rx_id"][i])
        power[s, t, r] += table["path_gain"][i]
        fieldc[s, t, r] += table["path_field"][i]
    total_field = fieldc.sum(axis=0)
    if coherent:
        comp_power = np.abs(fieldc) ** 2
        comp_power[4] = power[4]
        path_gain = np.abs(fieldc[[0, 1, 2, 3, 5]].sum(axis=0)) ** 2 + power[4]
        field_total = fieldc[[0, 1, 2, 3, 5]].sum(axis=0)
    else:
        comp_power = power
        path_gain = power.sum(axis=0)
        field_total = np.sqrt(np.maximum(path_gain, 0.0)) + 0.0j
    del total_field
    return {
        "path_gain": path_gain,
        "field": field_total,
        "component_power": comp_power,
        "component_field": fieldc,
    }
