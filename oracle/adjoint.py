"""Fixed-topology re-evaluation of path fields, FP64 (test infrastructure only).

The reference differentiates its deterministic solve with every path's
interaction sequence frozen (``witwin/channel/propagation/geometry.py:214-286``:
the frozen-winner re-solve gathers the winner faces' anchor and normal, so a
reflection's hit points follow the planes of the faces it was resolved to;
``kernels/fields.py`` then differentiates the field algebra).  This module
re-evaluates a frozen path table from raw arrays (vertices, materials,
frequency, endpoints) with exactly that definition, so central finite
differences of it are the reference's fixed-topology derivative.
"""

from __future__ import annotations

import numpy as np

from . import em, geom, utd
from .solve import edge_table


def _face_planes(V, Fc):
    n = geom.face_normals(V, Fc)
    return n, V[Fc[:, 0]]


def fixed_topology_fields(arrays: dict, table: dict, frequency: float) -> np.ndarray:
    """Powered complex path field of every row of ``table`` (keys ``tx_id``,
    ``rx_id``, ``component_id``, ``depth``, ``primitive_sequence``, ``edge_id``)."""
    V, Fc = arrays["vertices"], arrays["faces"]
    fm = arrays["face_mats"]
    tx_pos, tx_pow, tx_pol = arrays["tx_pos"], arrays["tx_power"], arrays["tx_pol"]
    rx_pos, rx_pol = arrays["rx_pos"], arrays["rx_pol"]
    normals, anchors = _face_planes(V, Fc) if Fc.shape[0] else (np.zeros((0, 3)), np.zeros((0, 3)))
    eg = None
    out = np.zeros(len(table["tx_id"]), dtype=np.complex128)
    for i in range(len(out)):
        t, r = int(table["tx_id"][i]), int(table["rx_id"][i])
        c, d = int(table["component_id"][i]), int(table["depth"][i])
        S, R = tx_pos[t], rx_pos[r]
        P = np.array([tx_pow[t]])
        pt, pr = tx_pol[t][None], rx_pol[r][None]
        if c == 0:
            ev = em.free_space(S[None], R[None], P, pt, pr, frequency)
        elif c == 1:
            faces = [int(x) for x in table["primitive_sequence"][i][:d]]
            planes = [(anchors[f], normals[f]) for f in faces]
            images = geom.image_chain(S, planes)
            x = R.copy()
            hits = [None] * d
            for k in range(d - 1, -1, -1):
                a, n = planes[k]
                img = images[k]
                tt = np.dot(a - x, n) / np.dot(img - x, n)
                x = x + (img - x) * tt
                hits[k] = x
            f = np.asarray(faces)
            ev = em.reflection_sequence(S[None], R[None], np.asarray(hits)[None], normals[f][None], P, pt, pr,
                                        fm["eps_r"][f][None], fm["sigma_e"][f][None], fm["mu_r"][f][None],
                                        fm["gain"][f][None], fm["thickness"][f][None], frequency)
        elif c == 5:
            f = np.asarray([int(x) for x in table["primitive_sequence"][i][:d]])
            ev = em.transmission_sequence(S[None], R[None], normals[f][None], arrays["face_material"][f][None],
                                          np.array([d]), P, pt, pr, arrays["material_layers"], frequency)
        elif c == 2:
            if eg is None:
                eg = edge_table(arrays, arrays.get("edge_policy"))
            e = int(table["edge_id"][i])
            res = utd.diffraction_field(S, R, tx_pol[t], eg, e, fm, frequency)
            if res is None:
                continue
            fxyz, q, _q_vis, _sp, _s = res
            arrival = em.safe_normalize((R - q)[None], np.array([[0.0, 0.0, 1.0]]))
            ev = em.project_complex3(fxyz[None] * np.sqrt(max(tx_pow[t], 0.0)), arrival, pr)
            ev = {"path_field": ev["coefficient"]}
        else:
            continue
        out[i] = ev["path_field"][0]
    return out


def cell_path_gain(fields: np.ndarray, table: dict, T: int, R: int, coherent: bool = True) -> np.ndarray:
    """Per-cell path gain of the rows: |sum of fields|^2 (coherent) or the sum of |field|^2."""
    pg = np.zeros((T, R))
    if coherent:
        acc = np.zeros((T, R), dtype=np.complex128)
        np.add.at(acc, (np.asarray(table["tx_id"]), np.asarray(table["rx_id"])), fields)
        pg = np.abs(acc) ** 2
    else:
        np.add.at(pg, (np.asarray(table["tx_id"]), np.asarray(table["rx_id"])), np.abs(fields) ** 2)
    return pg
