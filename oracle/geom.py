"""Scene geometry for the oracle: normals, coplanar groups, edges, brute-force
ray queries, the image-method path solve and the discovery trace.

Ray/segment queries test every triangle (no BVH) in float64.

Test infrastructure only: the tests, the smoke check and the benchmark's CPU
baseline call it as the checker; the product path never does.
"""

from __future__ import annotations

import numpy as np

PLANE_GROUP_QUANTIZATION = 1.0e-4  # propagation/geometry.py:113
PLANE_TOLERANCE = 1.0e-3  # rayd/reflection.cpp:50 (request.plane_tolerance)
BARY_EPS = 1.0e-7
SEGMENT_T_EPS = 1.0e-6
EDGE_PLANE_TOL = 1.34e-5  # propagation/geometry.py:37 (_RAYD_EDGE_INFO_PLANE_TOL)
ENDPOINT_QUANTIZATION = 1.0e-4  # scene/resources.py:296

# Rays traced (segment queries and discovery bounces), for throughput figures.
RAY_COUNTER = [0]
NORMAL_COS_TOL = 1.0 - 1.0e-5  # scene/resources.py:297


def face_normals(vertices: np.ndarray, faces: np.ndarray) -> np.ndarray:
    """Unit geometric normals ``normalize(cross(v1-v0, v2-v0))`` in float64."""
    v0 = vertices[faces[:, 0]]
    n = np.cross(vertices[faces[:, 1]] - v0, vertices[faces[:, 2]] - v0)
    length = np.sqrt(np.sum(n * n, axis=-1))
    return n / np.maximum(length, 1.0e-6)[:, None]


def face_normals_f32(vertices: np.ndarray, faces: np.ndarray) -> np.ndarray:
    v = vertices.astype(np.float32)
    v0 = v[faces[:, 0]]
    n = np.cross(v[faces[:, 1]] - v0, v[faces[:, 2]] - v0).astype(np.float32)
    length = np.sqrt(np.sum(n * n, axis=-1, dtype=np.float32)).astype(np.float32)
    return (n / np.maximum(length, np.float32(1.0e-6))[:, None]).astype(np.float32)


def _llround(x: np.ndarray) -> np.ndarray:
    return (np.sign(x) * np.floor(np.abs(x) + 0.5)).astype(np.int64)


def coplanar_groups(tri_a: np.ndarray, normals: np.ndarray, surface_ids: np.ndarray) -> dict:
    """Coplanar face groups (``paths.cu:3168-3190`` keys; ``paths.cu:3768-3912`` order).

    Key = (surface_id, round(n*1e4) with the sign fixed so the largest-magnitude
    component is positive, round(offset*1e4)); groups are numbered in key order,
    the representative is the lowest face index of each group.
    """
    face_count = tri_a.shape[0]
    n = normals.astype(np.float32)
    norm = np.sqrt(np.sum(n * n, axis=-1, dtype=np.float32)).astype(np.float32)
    inv = np.where(norm > np.float32(1e-6), np.float32(1.0) / norm, np.float32(0.0)).astype(np.float32)
    n = (n * inv[:, None]).astype(np.float32)
    major = n[:, 0].copy()
    ab = np.abs(n[:, 0])
    ay = np.abs(n[:, 1])
    major = np.where(ay > ab, n[:, 1], major)
    ab = np.maximum(ab, ay)
    az = np.abs(n[:, 2])
    major = np.where(az > ab, n[:, 2], major)
    sign = np.where(major < 0, np.float32(-1.0), np.float32(1.0)).astype(np.float32)
    n = (n * sign[:, None]).astype(np.float32)
    p = tri_a.astype(np.float32)
    offset = (n[:, 0] * p[:, 0] + n[:, 1] * p[:, 1] + n[:, 2] * p[:, 2]).astype(np.float32)
    scale = np.float32(1.0 / PLANE_GROUP_QUANTIZATION)
    keys = np.stack(
        [
            surface_ids.astype(np.int64),
            _llround((n[:, 0] * scale).astype(np.float32)),
            _llround((n[:, 1] * scale).astype(np.float32)),
            _llround((n[:, 2] * scale).astype(np.float32)),
            _llround((offset * scale).astype(np.float32)),
        ],
        axis=1,
    )
    order = np.lexsort(keys[:, ::-1].T) if face_count else np.zeros(0, dtype=np.int64)
    face_group = np.zeros(face_count, dtype=np.int64)
    reps = []
    members: list[list[int]] = []
    prev = None
    for f in order:
        k = tuple(keys[f])
        if k != prev:
            reps.append(int(f))
            members.append([])
            prev = k
        face_group[f] = len(reps) - 1
        members[-1].append(int(f))
    return {
        "face_group_id": face_group,
        "representative_faces": np.asarray(reps, dtype=np.int64),
        "members": [sorted(m) for m in members],
        "group_count": len(reps),
    }


def edge_records(faces: np.ndarray, face_structure: np.ndarray) -> dict:
    """Per-structure unique undirected edges, numbered structure by structure
    in ascending ``(min vertex, max vertex)`` order; ``face0``/``face1`` are the
    two lowest face indices that use the edge (``-1`` when on a boundary).

    This numbering reproduces the reference's single-wedge edge ids
    (``tests/deterministic/test_diffraction_single_wedge.py:44-53``).
    """
    v0s, v1s, f0s, f1s = [], [], [], []
    for s in np.unique(face_structure):
        fidx = np.nonzero(face_structure == s)[0]
        table: dict[tuple[int, int], list[int]] = {}
        for f in fidx:
            a, b, c = (int(x) for x in faces[f])
            for u, v in ((a, b), (b, c), (c, a)):
                key = (min(u, v), max(u, v))
                table.setdefault(key, []).append(int(f))
        for key in sorted(table):
            fl = sorted(table[key])
            v0s.append(key[0])
            v1s.append(key[1])
            f0s.append(fl[0])
            f1s.append(fl[1] if len(fl) > 1 else -1)
    return {
        "edge_v0": np.asarray(v0s, dtype=np.int64),
        "edge_v1": np.asarray(v1s, dtype=np.int64),
        "face0": np.asarray(f0s, dtype=np.int64),
        "face1": np.asarray(f1s, dtype=np.int64),
    }


def _unsigned_angle(a, b, axis):
    c = np.cross(a, b)
    sn = np.sign(np.dot(c, axis)) * np.linalg.norm(c)
    ang = np.arctan2(sn, np.dot(a, b))
    return ang + 2 * np.pi if ang < 0 else ang


def _normalize(v, eps=1e-6):
    length = np.linalg.norm(v)
    return v / max(length, eps)


def _opposite(faces, f, a, b):
    for v in faces[f]:
        if v != a and v != b:
            return int(v)
    return int(faces[f][2])


def edge_geometry(vertices: np.ndarray, faces: np.ndarray, normals: np.ndarray, records: dict,
                  *, boundary_policy: str = "half_plane", vertical_only: bool = False,
                  vertical_ratio: float = 0.7) -> dict:
    """Edge selection, ordered wedge normals and exterior angle
    (``diffraction.cu:803-900``) followed by the shared-boundary merge and
    policy filter (``scene/resources.py:306-405``)."""
    ne = records["edge_v0"].shape[0]
    sel = np.zeros(ne, dtype=bool)
    pos = np.zeros((ne, 3))
    dirs = np.zeros((ne, 3))
    length = np.zeros(ne)
    n0o = np.zeros((ne, 3))
    n1o = np.zeros((ne, 3))
    opp0 = np.zeros((ne, 3))
    mat0 = np.zeros(ne, dtype=np.int64)
    mat1 = np.zeros(ne, dtype=np.int64)
    ext = np.zeros(ne)
    for e in range(ne):
        v0, v1 = int(records["edge_v0"][e]), int(records["edge_v1"][e])
        f0, f1 = int(records["face0"][e]), int(records["face1"][e])
        boundary = f0 >= 0 and f1 < 0
        interior = f0 >= 0 and f1 >= 0
        s0, s1 = max(f0, 0), max(f1, 0)
        start, end = vertices[v0], vertices[v1]
        vec = end - start
        L = max(np.linalg.norm(vec), 1e-12)
        d = vec / L
        n0c = _normalize(normals[s0])
        n1c = _normalize(normals[s1])
        to1 = _normalize(np.cross(n0c, d))
        tn1 = _normalize(np.cross(n1c, d))
        choose_first = _unsigned_angle(to1, tn1, d) < _unsigned_angle(tn1, to1, d)
        on0 = n0c if choose_first else n1c
        on1 = n1c if choose_first else n0c
        out0 = on0 if interior else n0c
        out1 = on1 if interior else n1c
        if f1 < 0:
            out1 = -n0c
        inter = np.arccos(np.clip(-np.dot(out0, out1), -1.0, 1.0))
        ext[e] = (2 * np.pi - inter) if interior else 2 * np.pi
        coplanar = False
        if interior:
            aligned = abs(np.dot(n0c, n1c)) >= NORMAL_COS_TOL
            pa = vertices[_opposite(faces, s0, v0, v1)]
            pb = vertices[_opposite(faces, s1, v0, v1)]
            da = abs(np.dot(pa - start, n0c))
            db = abs(np.dot(pb - start, n0c))
            coplanar = aligned and da <= EDGE_PLANE_TOL and db <= EDGE_PLANE_TOL
        wedge_ok = boundary or (interior and np.dot(n0c, n1c) < 1.0)
        sel[e] = (interior or boundary) and (not coplanar) and L > 1e-6 and wedge_ok
        swapped = interior and not choose_first
        opp0[e] = vertices[_opposite(faces, s1 if swapped else s0, v0, v1)]
        mat0[e] = f1 if swapped else f0
        mat1[e] = f0 if swapped else f1
        pos[e] = 0.5 * (start + end)
        dirs[e] = d
        length[e] = L
        n0o[e] = out0
        n1o[e] = out1
    face0 = records["face0"].copy()
    face1 = records["face1"].copy()
    boundary = face1 < 0
    # shared boundary merge (scene/resources.py:322-353, 369-386)
    cand = np.nonzero(sel & boundary)[0]
    if cand.size >= 2:
        p0 = np.round(vertices[records["edge_v0"][cand]] / ENDPOINT_QUANTIZATION).astype(np.int64)
        p1 = np.round(vertices[records["edge_v1"][cand]] / ENDPOINT_QUANTIZATION).astype(np.int64)
        keys = []
        for a, b in zip(p0, p1):
            ta, tb = tuple(a), tuple(b)
            keys.append(ta + tb if ta <= tb else tb + ta)
        groups: dict[tuple, list[int]] = {}
        for idx, k in zip(cand, keys):
            groups.setdefault(k, []).append(int(idx))
        for k in groups:
            g = groups[k]
            if len(g) >= 2:
                a, b = g[0], g[1]
                nd = np.clip(np.dot(n0o[a], n0o[b]), -1.0, 1.0)
                interior_angle = np.arccos(np.clip(-nd, -1.0, 1.0))
                merged = 2 * np.pi - interior_angle
                copl = abs(nd) >= NORMAL_COS_TOL
                sel[a] = (merged > np.pi * (1.0 + 1e-6)) and not copl
                sel[b] = False
                n1o[a] = n0o[b]
                face1[a] = face0[b]
                mat1[a] = mat0[b]
                ext[a] = merged
                boundary[a] = False
                for extra in g[2:]:
                    sel[extra] = False
    if boundary_policy != "half_plane":
        sel &= ~boundary
    if vertical_only:
        delta = vertices[records["edge_v1"]] - vertices[records["edge_v0"]]
        lz = np.maximum(np.linalg.norm(delta, axis=1), 1e-6)
        sel &= (np.abs(delta[:, 2]) / lz) > vertical_ratio
    return {
        "selected": sel,
        "edge_pos": pos,
        "edge_dir": dirs,
        "length": length,
        "line_min": -0.5 * length,
        "line_max": 0.5 * length,
        "n0": n0o,
        "n1": n1o,
        "face0": face0,
        "face1": face1,
        "exterior_angle": ext,
        "opp0": opp0,
        "wedge_face0": mat0,
        "wedge_face1": mat1,
    }


# --------------------------------------------------------------------------
# brute-force ray queries
# --------------------------------------------------------------------------


class Triangles:
    def __init__(self, vertices: np.ndarray, faces: np.ndarray):
        self.v0 = vertices[faces[:, 0]].astype(np.float64)
        self.e1 = vertices[faces[:, 1]].astype(np.float64) - self.v0
        self.e2 = vertices[faces[:, 2]].astype(np.float64) - self.v0
        self.count = faces.shape[0]

    def intersect(self, origin: np.ndarray, direction: np.ndarray):
        """Moller-Trumbore against all triangles.  ``origin``/``direction``
        are ``(N, 3)``; returns ``t (N, F)`` (inf where missed)."""
        n = origin.shape[0]
        if self.count == 0 or n == 0:
            return np.full((n, self.count), np.inf)
        d = direction[:, None, :]
        pvec = np.cross(d, self.e2[None, :, :])
        det = np.sum(self.e1[None] * pvec, axis=-1)
        ok = np.abs(det) > 1e-300
        inv = np.where(ok, 1.0 / np.where(ok, det, 1.0), 0.0)
        tvec = origin[:, None, :] - self.v0[None]
        u = np.sum(tvec * pvec, axis=-1) * inv
        qvec = np.cross(tvec, self.e1[None])
        v = np.sum(d * qvec, axis=-1) * inv
        t = np.sum(self.e2[None] * qvec, axis=-1) * inv
        hit = ok & (u >= -BARY_EPS) & (v >= -BARY_EPS) & (u + v <= 1.0 + BARY_EPS)
        return np.where(hit, t, np.inf)


def segment_blocked(tris: Triangles, p0: np.ndarray, p1: np.ndarray, ignore: np.ndarray | None = None,
                    chunk: int = 4096) -> np.ndarray:
    """True where segment p0->p1 hits a triangle at ``t`` in
    ``[SEGMENT_T_EPS, 1 - SEGMENT_T_EPS]``; ``ignore`` is an ``(N, F)`` bool mask."""
    out = np.zeros(p0.shape[0], dtype=bool)
    RAY_COUNTER[0] += int(p0.shape[0])
    for s in range(0, p0.shape[0], chunk):
        e = min(s + chunk, p0.shape[0])
        t = tris.intersect(p0[s:e], p1[s:e] - p0[s:e])
        if ignore is not None:
            t = np.where(ignore[s:e], np.inf, t)
        out[s:e] = np.any((t >= SEGMENT_T_EPS) & (t <= 1.0 - SEGMENT_T_EPS), axis=1)
    return out


def segment_hits(tris: Triangles, p0: np.ndarray, p1: np.ndarray, groups: np.ndarray | None = None
                 ) -> list[list[tuple[float, int]]]:
    """All hits ``(t, face)`` per segment, ascending in ``t``."""
    t = tris.intersect(p0, p1 - p0)
    RAY_COUNTER[0] += int(p0.shape[0])
    out = []
    for row in t:
        idx = np.nonzero((row >= SEGMENT_T_EPS) & (row <= 1.0 - SEGMENT_T_EPS))[0]
        hits = sorted((float(row[i]), int(i)) for i in idx)
        if groups is not None:
            # one crossing per plane: a shared diagonal reports both triangles
            kept = []
            for tt, f in hits:
                if any(groups[g] == groups[f] and abs(tt - t2) < 1e-7 for t2, g in kept):
                    continue
                kept.append((tt, f))
            hits = kept
        out.append(hits)
    return out


# --------------------------------------------------------------------------
# image method
# --------------------------------------------------------------------------


def point_in_face(point: np.ndarray, vertices: np.ndarray, faces: np.ndarray, normals: np.ndarray, f: int) -> bool:
    a, b, c = (vertices[int(i)].astype(np.float64) for i in faces[f])
    n = normals[f]
    if abs(np.dot(point - a, n)) > PLANE_TOLERANCE:
        return False
    q = point - np.dot(point - a, n) * n
    e1, e2, w = b - a, c - a, q - a
    d11, d12, d22 = np.dot(e1, e1), np.dot(e1, e2), np.dot(e2, e2)
    w1, w2 = np.dot(w, e1), np.dot(w, e2)
    den = d11 * d22 - d12 * d12
    if den <= 0.0:
        return False
    v = (d22 * w1 - d12 * w2) / den
    u = (d11 * w2 - d12 * w1) / den
    return v >= -BARY_EPS and u >= -BARY_EPS and u + v <= 1.0 + BARY_EPS


def reflect_point(p: np.ndarray, a: np.ndarray, n: np.ndarray) -> np.ndarray:
    return p - 2.0 * np.dot(p - a, n) * n


def image_chain(source: np.ndarray, planes: list[tuple[np.ndarray, np.ndarray]]) -> list[np.ndarray]:
    images = []
    p = source
    for a, n in planes:
        p = reflect_point(p, a, n)
        images.append(p)
    return images


def back_project(receiver: np.ndarray, images: list[np.ndarray], planes) -> list[np.ndarray] | None:
    """Hit points of the specular chain or ``None`` when a back-projected line
    does not cross its plane strictly between its ends."""
    d = len(planes)
    hits: list[np.ndarray] = [None] * d  # type: ignore[list-item]
    x = receiver
    for k in range(d - 1, -1, -1):
        a, n = planes[k]
        img = images[k]
        denom = np.dot(img - x, n)
        if denom == 0.0:
            return None
        t = np.dot(a - x, n) / denom
        if not (t > SEGMENT_T_EPS and t < 1.0 - SEGMENT_T_EPS):
            return None
        x = x + t * (img - x)
        hits[k] = x
    return hits


def fibonacci_directions(count: int) -> np.ndarray:
    """FP64 Fibonacci sphere rounded to float32 (``montecarlo.cu:713-731``)."""
    golden = 1.618033988749894848204586834365638118
    idx = np.arange(count, dtype=np.float64)
    az = idx / golden
    az_u = az - np.floor(az)
    ev = np.zeros(count) if count == 1 else idx / float(count - 1)
    phi = 2.0 * np.pi * az_u
    z = 1.0 - 2.0 * ev
    radial = np.sqrt(np.maximum(1.0 - z * z, 0.0))
    out = np.stack([radial * np.cos(phi), radial * np.sin(phi), z], axis=1)
    return out.astype(np.float32)


def trace_reflections(tris: Triangles, normals: np.ndarray, origin: np.ndarray, directions: np.ndarray,
                      max_depth: int, chunk: int = 2048) -> np.ndarray:
    """Specular bounce chains from ``origin``: closest hit with ``t > 1e-6``
    (the face just left is skipped), mirror the direction about the face
    normal, continue.  Returns ``(N, max_depth)`` face ids, ``-1`` after a miss."""
    n = directions.shape[0]
    out = np.full((n, max_depth), -1, dtype=np.int64)
    for s in range(0, n, chunk):
        e = min(s + chunk, n)
        o = np.broadcast_to(origin.astype(np.float64), (e - s, 3)).copy()
        d = directions[s:e].astype(np.float64)
        last = np.full(e - s, -1, dtype=np.int64)
        alive = np.ones(e - s, dtype=bool)
        for depth in range(max_depth):
            RAY_COUNTER[0] += int(alive.sum())
            t = tris.intersect(o, d)
            rows = np.arange(e - s)
            t[rows[last >= 0], last[last >= 0]] = np.inf
            t = np.where(t > 1e-6, t, np.inf)
            f = np.argmin(t, axis=1)
            tmin = t[rows, f]
            hit = alive & np.isfinite(tmin)
            out[s:e, depth] = np.where(hit, f, -1)
            nn = normals[f]
            # misses step by 0 (not inf * 0): the origin is kept exactly
            o = o + np.where(hit, tmin, 0.0)[:, None] * d
            d = np.where(hit[:, None], d - 2.0 * np.sum(d * nn, axis=1)[:, None] * nn, d)
            last = np.where(hit, f, -1)
            alive = hit
    return out
