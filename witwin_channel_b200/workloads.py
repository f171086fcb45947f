"""Seeded synthetic scenes for the benchmark workloads.

No public dataset is involved: every scene is generated from
``numpy.random.default_rng(seed)`` with the shapes, sizes and material laws
of the five benchmark workloads (two-ray ground check; 64-box urban canyon;
gradient run on that canyon; eight uneven scenes batched over transmitters
and frequencies; a 2048-box city with subdivided roofs and glass sheets).
"""

from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np
import torch

from .scene import (
    MaterialLayer,
    PhysicalMaterial,
    Scene,
    make_mesh_structure,
    make_receiver_grid,
    make_transmitter,
)


def concrete(thickness_m: float = 0.3, name: str = "concrete") -> PhysicalMaterial:
    """ITU-R P.2040 concrete: eps_r 5.24, sigma = 0.0462 (f/1GHz)^0.7822 S/m."""
    return PhysicalMaterial(
        eps_r=5.24,
        sigma_e=lambda f: 0.0462 * (f / 1.0e9) ** 0.7822,
        thickness_m=thickness_m,
        name=name,
    )


def glass_two_layer() -> PhysicalMaterial:
    """Two 6 mm glass layers, eps_r 6.27, sigma = 0.0043 (f/1GHz)^1.1925 S/m."""
    sig = lambda f: 0.0043 * (f / 1.0e9) ** 1.1925  # noqa: E731
    layer = MaterialLayer(thickness_m=0.006, eps_r=6.27, sigma_e=sig)
    return PhysicalMaterial(eps_r=6.27, sigma_e=sig, thickness_m=0.006, layers=(layer, layer), name="glass")


def ground_structure(half: float, material: PhysicalMaterial, surface_id: int):
    v = torch.tensor([[-half, -half, 0.0], [half, -half, 0.0], [half, half, 0.0], [-half, half, 0.0]])
    f = torch.tensor([[0, 1, 2], [0, 2, 3]])
    return make_mesh_structure(vertices=v, faces=f, material=material, surface_id=surface_id, name="ground")


def box_mesh(x0: float, y0: float, x1: float, y1: float, h: float, roof_k: int = 1):
    """Closed box with outward-facing triangles (bottom included).

    With ``roof_k > 1`` the roof is split into ``roof_k x roof_k`` quads and
    each wall's top edge into ``roof_k`` pieces (walls become fans), so the
    mesh stays free of T-junctions: every roof/wall edge piece is a proper
    90-degree wedge and the extra triangles are coplanar with their face.
    """
    k = max(int(roof_k), 1)
    verts = [(x0, y0, 0.0), (x1, y0, 0.0), (x1, y1, 0.0), (x0, y1, 0.0)]
    top = {}

    def top_vertex(i: int, j: int) -> int:
        if (i, j) not in top:
            top[(i, j)] = len(verts)
            verts.append((x0 + (x1 - x0) * i / k, y0 + (y1 - y0) * j / k, h))
        return top[(i, j)]

    faces = [(0, 2, 1), (0, 3, 2)]  # bottom, normal -z
    # walls as fans from a bottom corner; top edge runs along the roof boundary
    # wall y = y0 (normal -y): polygon 0, 1, top(k,0) ... top(0,0)
    ring = [top_vertex(i, 0) for i in range(k, -1, -1)]
    faces += [(0, 1, ring[0])] + [(0, ring[q], ring[q + 1]) for q in range(k)]
    # wall x = x1 (normal +x): polygon 1, 2, top(k,k) ... top(k,0)
    ring = [top_vertex(k, j) for j in range(k, -1, -1)]
    faces += [(1, 2, ring[0])] + [(1, ring[q], ring[q + 1]) for q in range(k)]
    # wall y = y1 (normal +y): polygon 2, 3, top(0,k) ... top(k,k)
    ring = [top_vertex(i, k) for i in range(0, k + 1)]
    faces += [(2, 3, ring[0])] + [(2, ring[q], ring[q + 1]) for q in range(k)]
    # wall x = x0 (normal -x): polygon 3, 0, top(0,0) ... top(0,k)
    ring = [top_vertex(0, j) for j in range(0, k + 1)]
    faces += [(3, 0, ring[0])] + [(3, ring[q], ring[q + 1]) for q in range(k)]
    for i in range(k):
        for j in range(k):
            a, b, c, d = top_vertex(i, j), top_vertex(i + 1, j), top_vertex(i + 1, j + 1), top_vertex(i, j + 1)
            faces += [(a, b, c), (a, c, d)]  # roof, normal +z
    return torch.tensor(verts, dtype=torch.float32), torch.tensor(faces, dtype=torch.int64)


@dataclass
class CityLayout:
    lots: int            # lots per side
    lot_size: float
    boxes: list          # (x0, y0, x1, y1, h)

    @property
    def half(self) -> float:
        return 0.5 * self.lots * self.lot_size


def city_layout(n_boxes: int, seed: int, lot_size: float = 50.0, lots: int | None = None,
                footprint=(10.0, 40.0), height=(10.0, 60.0)) -> CityLayout:
    rng = np.random.default_rng(seed)
    side = lots if lots is not None else int(math.ceil(math.sqrt(n_boxes)))
    half = 0.5 * side * lot_size
    boxes = []
    for idx in range(n_boxes):
        i, j = idx % side, idx // side
        cx = -half + (i + 0.5) * lot_size
        cy = -half + (j + 0.5) * lot_size
        w, d = rng.uniform(footprint[0], footprint[1], size=2)
        h = rng.uniform(height[0], height[1])
        boxes.append((cx - w / 2, cy - d / 2, cx + w / 2, cy + d / 2, h))
    return CityLayout(lots=side, lot_size=lot_size, boxes=boxes)


def street_point(layout: CityLayout, rng: np.random.Generator, z: float) -> tuple[float, float, float]:
    """A point on a lot-gap centreline (between lots, clear of every box)."""
    k = int(rng.integers(1, layout.lots)) if layout.lots > 1 else 0
    along = float(rng.uniform(-layout.half, layout.half))
    line = -layout.half + k * layout.lot_size
    if rng.uniform() < 0.5:
        return (line, along, z)
    return (along, line, z)


def city_scene(layout: CityLayout, *, material: PhysicalMaterial | None = None, ground_half: float | None = None,
               roof_k=None, sheets: list | None = None) -> list:
    mat = material or concrete()
    structures = [ground_structure(ground_half or layout.half, concrete(10.0, "ground"), surface_id=0)]
    for b, (x0, y0, x1, y1, h) in enumerate(layout.boxes):
        k = roof_k(b) if callable(roof_k) else 1
        v, f = box_mesh(x0, y0, x1, y1, h, k)
        structures.append(make_mesh_structure(vertices=v, faces=f, material=mat, surface_id=b + 1, name=f"box{b}"))
    if sheets:
        glass = glass_two_layer()
        for s, (p0, p1, h) in enumerate(sheets):
            v = torch.tensor([[p0[0], p0[1], 0.0], [p1[0], p1[1], 0.0], [p1[0], p1[1], h], [p0[0], p0[1], h]])
            f = torch.tensor([[0, 1, 2], [0, 2, 3]])
            structures.append(make_mesh_structure(vertices=v, faces=f, material=glass,
                                                  surface_id=len(layout.boxes) + 1 + s, name=f"sheet{s}"))
    return structures


# ------------------------------------------------------------------ workloads
def two_ray_scene(shape=(64, 64), spacing=2.0) -> tuple[Scene, float]:
    """Ground of 2 triangles over [-100, 100]^2 at z=0 (concrete, 10 m slab so
    the Fabry-Perot term vanishes), Tx (0,0,10) z-polarised 1 W, a 64x64 grid
    at z=1.5 with 2 m spacing centred on the Tx, 3.5 GHz."""
    g = ground_structure(100.0, concrete(10.0, "ground"), surface_id=0)
    rows, cols = shape
    origin = (-(rows - 1) / 2.0 * spacing, -(cols - 1) / 2.0 * spacing, 1.5)
    grid = make_receiver_grid(origin=origin, x_axis=(1.0, 0.0, 0.0), y_axis=(0.0, 1.0, 0.0), shape=shape,
                              spacing=(spacing, spacing))
    return Scene(structures=[g], endpoints=[make_transmitter((0.0, 0.0, 10.0)), grid]), 3.5e9


def urban_canyon_scene(seed: int = 1, grid_side: int = 256, spacing: float = 1.5, n_boxes: int = 64,
                       tx_height: float = 25.0) -> tuple[Scene, float]:
    """64 boxes on 8x8 lots of 50 m, Tx at 25 m on a street, 256^2 grid at
    1.5 m height and spacing, 28 GHz."""
    layout = city_layout(n_boxes, seed)
    rng = np.random.default_rng(seed + 1000)
    tx = street_point(layout, rng, tx_height)
    structures = city_scene(layout)
    origin = (-(grid_side - 1) / 2.0 * spacing, -(grid_side - 1) / 2.0 * spacing, 1.5)
    grid = make_receiver_grid(origin=origin, x_axis=(1.0, 0.0, 0.0), y_axis=(0.0, 1.0, 0.0),
                              shape=(grid_side, grid_side), spacing=(spacing, spacing))
    return Scene(structures=structures, endpoints=[make_transmitter(tx), grid]), 28.0e9


BATCH_BOXES = (16, 32, 48, 64, 96, 128, 192, 256)
BATCH_GRID = (64, 96, 128, 192, 256, 320, 384, 512)
BATCH_SPACING = (4.0, 3.5, 3.0, 2.5, 2.0, 1.5, 1.25, 1.0)
BATCH_FREQS = (3.5e9, 6.0e9, 28.0e9, 39.0e9)


def batched_scenes() -> list[Scene]:
    """Eight scenes (boxes 16..256, seeds 3..10), four transmitters each at
    5-40 m on streets, grids 64^2..512^2 centred on the lot grid."""
    scenes = []
    for s, (n, side, sp) in enumerate(zip(BATCH_BOXES, BATCH_GRID, BATCH_SPACING)):
        seed = 3 + s
        layout = city_layout(n, seed)
        rng = np.random.default_rng(seed + 1000)
        txs = [make_transmitter(street_point(layout, rng, float(rng.uniform(5.0, 40.0)))) for _ in range(4)]
        origin = (-(side - 1) / 2.0 * sp, -(side - 1) / 2.0 * sp, 1.5)
        grid = make_receiver_grid(origin=origin, x_axis=(1.0, 0.0, 0.0), y_axis=(0.0, 1.0, 0.0), shape=(side, side),
                                  spacing=(sp, sp))
        scenes.append(Scene(structures=city_scene(layout), endpoints=txs + [grid]))
    return scenes


def large_city_scene(seed: int = 4, grid_side: int = 1024) -> tuple[Scene, float]:
    """2048 boxes on 46x46 lots, roofs subdivided k x k with k = 4 on even and
    5 on odd boxes (walls split to match so the mesh has no T-junctions:
    ~134k triangles), 25% of boxes with an interior two-layer glass sheet, 1 Tx
    at 25 m, 1024^2 grid at 1 m spacing, 28 GHz."""
    layout = city_layout(2048, seed, lots=46)
    rng = np.random.default_rng(seed + 2000)
    sheets = []
    for b, (x0, y0, x1, y1, h) in enumerate(layout.boxes):
        if rng.uniform() < 0.25:
            cx = 0.5 * (x0 + x1)
            sheets.append(((cx, y0 + 0.5), (cx, y1 - 0.5), 0.8 * h))
    structures = city_scene(layout, roof_k=lambda b: 4 if b % 2 == 0 else 5, sheets=sheets)
    tx = street_point(layout, np.random.default_rng(seed + 1000), 25.0)
    origin = (-(grid_side - 1) / 2.0, -(grid_side - 1) / 2.0, 1.5)
    grid = make_receiver_grid(origin=origin, x_axis=(1.0, 0.0, 0.0), y_axis=(0.0, 1.0, 0.0),
                              shape=(grid_side, grid_side), spacing=(1.0, 1.0))
    return Scene(structures=structures, endpoints=[make_transmitter(tx), grid]), 28.0e9


def gradient_run(seed: int = 1, grid_side: int = 256, moved_boxes: int = 8, displacement_m: float = 0.5,
                 eps_scale: float = 1.10) -> dict:
    """The gradient workload on the urban canyon: a differentiable scene
    (concrete eps_r and sigma_e as leaf tensors, the vertices of `moved_boxes`
    seeded boxes and the Tx position as leaves, the carrier frequency as a
    leaf) and a target radiomap solved on a perturbed copy (eps_r x1.10 and
    the same boxes' vertices displaced by N(0, 0.5 m)).  The loss is the MSE
    between log10 path-gain maps over the cells where both are positive."""
    from .deterministic import Config, solve

    freq = 28.0e9
    layout = city_layout(64, seed)
    rng = np.random.default_rng(seed + 1000)
    tx = street_point(layout, rng, 25.0)
    sigma = 0.0462 * (freq / 1.0e9) ** 0.7822
    eps = torch.tensor(5.24, dtype=torch.float64, requires_grad=True)
    sig = torch.tensor(sigma, dtype=torch.float64, requires_grad=True)
    mat = PhysicalMaterial(eps_r=eps, sigma_e=sig, thickness_m=0.3, name="concrete")
    structures = city_scene(layout, material=mat)
    pick = np.random.default_rng(seed + 3000).choice(len(layout.boxes), size=moved_boxes, replace=False)
    moved = []
    for b in sorted(int(x) for x in pick):
        st = structures[b + 1]
        leaf = st.vertices.detach().clone().requires_grad_(True)
        st.geometry.vertices = leaf
        moved.append(b + 1)
    txa = make_transmitter(tx)
    txa.position = torch.tensor(tx, dtype=torch.float32, requires_grad=True)
    spacing = 1.5
    origin = (-(grid_side - 1) / 2.0 * spacing, -(grid_side - 1) / 2.0 * spacing, 1.5)
    grid = make_receiver_grid(origin=origin, x_axis=(1.0, 0.0, 0.0), y_axis=(0.0, 1.0, 0.0),
                              shape=(grid_side, grid_side), spacing=(spacing, spacing))
    scene = Scene(structures=structures, endpoints=[txa, grid])
    # the target: a perturbed copy solved without gradients
    tmat = PhysicalMaterial(eps_r=5.24 * eps_scale, sigma_e=sigma, thickness_m=0.3, name="concrete")
    tstructs = city_scene(layout, material=tmat)
    drng = np.random.default_rng(seed + 4000)
    for idx in moved:
        v = tstructs[idx].vertices.detach().clone()
        tstructs[idx].geometry.vertices = v + torch.tensor(drng.normal(0.0, displacement_m, tuple(v.shape)),
                                                           dtype=torch.float32)
    tscene = Scene(structures=tstructs, endpoints=[make_transmitter(tx), grid])
    components = {"los", "reflection", "diffraction"}
    with torch.no_grad():
        target = solve(tscene, Config(components=components, max_depth=3), reference_frequency_hz=freq).path_gain
    freq_t = torch.tensor(freq, dtype=torch.float64, requires_grad=True)
    return {"scene": scene, "frequency": freq_t, "target": target, "components": components, "max_depth": 3,
            "leaves": {"eps_r": eps, "sigma_e": sig, "tx": txa.position,
                       "vertices": [structures[i].vertices for i in moved]},
            "moved_structures": moved}


def log_mse(path_gain, target):
    """MSE of log10 path gain over cells where both maps are positive."""
    mask = (path_gain > 0) & (target > 0)
    d = torch.log10(path_gain[mask].double()) - torch.log10(target[mask].double())
    return (d * d).mean()
