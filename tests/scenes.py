"""Small scenes shared by the tests (restated from the reference's fixtures:
tests/support/scenes.py:126-215, tests/deterministic/test_reflection_multibounce.py:126-161,
tests/deterministic/test_component_layout.py:15-30)."""

from __future__ import annotations

import numpy as np
import torch

from witwin_channel_b200.scene import (
    MaterialLayer,
    PhysicalMaterial,
    Scene,
    make_mesh_structure,
    make_receiver,
    make_receiver_grid,
    make_transmitter,
)
from witwin_channel_b200.workloads import city_layout, city_scene, street_point


def two_wall_scene() -> Scene:
    wall_x = make_mesh_structure(
        vertices=torch.tensor([[2.0, -1.0, 0.0], [2.0, 3.0, 0.0], [2.0, -1.0, 2.0], [2.0, 3.0, 2.0]]),
        faces=torch.tensor([[0, 1, 2], [1, 3, 2]]),
        material=PhysicalMaterial(eps_r=3.0, sigma_e=0.005), surface_id=10)
    wall_y = make_mesh_structure(
        vertices=torch.tensor([[0.0, 2.0, 0.0], [3.0, 2.0, 0.0], [0.0, 2.0, 2.0], [3.0, 2.0, 2.0]]),
        faces=torch.tensor([[0, 2, 1], [1, 2, 3]]),
        material=PhysicalMaterial(eps_r=4.0, sigma_e=0.01), surface_id=11)
    return Scene(structures=[wall_x, wall_y],
                 endpoints=[make_transmitter([0.0, 0.0, 1.0]), make_receiver([0.0, 1.0, 1.0])])


def wedge_scene(rx=(3.0, 1.0, 0.5)) -> Scene:
    pec = PhysicalMaterial.perfect_conductor()
    a = make_mesh_structure(vertices=torch.tensor([[2.0, 0.0, -1.0], [2.0, 0.0, 2.0], [2.0, 2.0, -1.0]]),
                            faces=torch.tensor([[0, 1, 2]]), material=pec, surface_id=2)
    b = make_mesh_structure(vertices=torch.tensor([[2.0, 0.0, -1.0], [2.0, 0.0, 2.0], [4.0, 0.0, -1.0]]),
                            faces=torch.tensor([[0, 2, 1]]), material=pec, surface_id=3)
    return Scene(structures=[a, b], endpoints=[make_transmitter([0.0, -1.0, 0.5]), make_receiver(list(rx))])


def los_grid_scene() -> Scene:
    return Scene(structures=[], endpoints=[
        make_transmitter([0.0, 0.0, 0.0], power_w=1.5),
        make_receiver_grid(origin=[3.0, -1.0, -0.5], x_axis=[0.0, 1.0, 0.0], y_axis=[0.0, 0.0, 1.0],
                           shape=(2, 3), spacing=(1.0, 0.5)),
    ])


def thin_wall_scene() -> Scene:
    glass = PhysicalMaterial(layers=(MaterialLayer(0.006, 6.27, 0.2287), MaterialLayer(0.006, 6.27, 0.2287)),
                             eps_r=6.27, sigma_e=0.2287, thickness_m=0.006)
    w = make_mesh_structure(vertices=torch.tensor([[2.0, -4.0, -4.0], [2.0, 4.0, -4.0], [2.0, -4.0, 4.0], [2.0, 4.0, 4.0]]),
                            faces=torch.tensor([[0, 1, 2], [1, 3, 2]]), material=glass, surface_id=1)
    w2 = make_mesh_structure(vertices=torch.tensor([[4.0, -4.0, -4.0], [4.0, 4.0, -4.0], [4.0, -4.0, 4.0], [4.0, 4.0, 4.0]]),
                             faces=torch.tensor([[0, 1, 2], [1, 3, 2]]), material=PhysicalMaterial(eps_r=4.0, sigma_e=0.02, thickness_m=0.1), surface_id=2)
    return Scene(structures=[w, w2], endpoints=[
        make_transmitter([0.0, 0.3, 0.2]),
        make_receiver([6.0, -0.5, 0.4]), make_receiver([3.0, 1.0, -0.3]), make_receiver([5.5, 2.0, 1.0]),
    ])


def small_city(n_boxes: int = 4, seed: int = 7, grid=(8, 8), spacing=6.0, tx_height=12.0,
               polarization=None) -> tuple[Scene, float]:
    layout = city_layout(n_boxes, seed, lot_size=30.0, footprint=(8.0, 20.0), height=(6.0, 25.0))
    rng = np.random.default_rng(seed + 1000)
    tx = street_point(layout, rng, tx_height)
    structures = city_scene(layout)
    rows, cols = grid
    origin = (-(rows - 1) / 2.0 * spacing, -(cols - 1) / 2.0 * spacing, 1.5)
    g = make_receiver_grid(origin=origin, x_axis=(1.0, 0.0, 0.0), y_axis=(0.0, 1.0, 0.0), shape=grid,
                           spacing=(spacing, spacing))
    return Scene(structures=structures, endpoints=[make_transmitter(tx, polarization=polarization), g]), 28.0e9
