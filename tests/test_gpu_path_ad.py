"""First-order AD of per-path coefficients on the GPU: the path solver's
``a`` and the deterministic path table's ``coefficient`` (reference
``tests/ad/test_solver_material_frequency_ad.py``: the same loss,
Re(sum a) + 0.5 Im(sum a), on an open wall, a layered thin sheet and free
space; here against central finite differences of the solve with
``ad_mode="none"``).

Checked: material eps_r / sigma_e, transmitter position and frequency
gradients (reverse mode) for both solvers, forward mode against the same
differences, and the primal values unchanged by ``ad_mode``.
"""

from __future__ import annotations

import pytest
import torch

from witwin_channel_b200 import Config as DetConfig
from witwin_channel_b200 import solve as det_solve
from witwin_channel_b200.path import Config as PathConfig
from witwin_channel_b200.path import solve as path_solve
from witwin_channel_b200.scene import (
    MaterialLayer,
    PhysicalMaterial,
    Scene,
    make_mesh_structure,
    make_receiver,
    make_transmitter,
)

pytestmark = pytest.mark.gpu
FREQ = 3.0e9


def _wall_scene(eps, sigma, tx):
    wall = make_mesh_structure(
        vertices=torch.tensor([[2.5, -3.0, -1.0], [2.5, 3.0, -1.0], [2.5, -3.0, 2.0], [2.5, 3.0, 2.0]]),
        faces=torch.tensor([[0, 1, 2], [1, 3, 2]]), material=PhysicalMaterial(eps_r=eps, sigma_e=sigma),
        surface_id=1)
    return Scene(structures=[wall], endpoints=[make_transmitter(tx), make_receiver(torch.tensor([0.0, 1.0, 0.5]))])


def _sheet_scene(eps):
    material = PhysicalMaterial(layers=(MaterialLayer(0.06, eps, 0.02), MaterialLayer(0.09, 2.5, 0.01)),
                                eps_r=eps, sigma_e=0.02, thickness_m=0.06)
    sheet = make_mesh_structure(
        vertices=torch.tensor([[3.0, -4.0, -4.0], [3.0, 4.0, -4.0], [3.0, -4.0, 4.0], [3.0, 4.0, 4.0]]),
        faces=torch.tensor([[0, 1, 2], [1, 3, 2]]), material=material, surface_id=1)
    return Scene(structures=[sheet], endpoints=[make_transmitter([0.0, 0.0, 0.0]),
                                                make_receiver([6.0, 0.4, 0.2])])


def _coefficients(scene, solver, components, ad_mode, freq=FREQ):
    if solver == "path":
        return path_solve(scene, PathConfig(max_depth=1, components=components, ad_mode=ad_mode),
                          reference_frequency_hz=freq).a
    res = det_solve(scene, DetConfig(max_depth=1, components=components, export_paths=True, ad_mode=ad_mode),
                    reference_frequency_hz=freq)
    return res.paths.coefficient


def _loss(a):
    return a.real.sum() + 0.5 * a.imag.sum()


@pytest.mark.parametrize("solver", ["path", "deterministic"])
def test_reflection_material_and_position_gradients_match_differences(solver):
    eps = torch.tensor(4.0, requires_grad=True)
    sigma = torch.tensor(0.02, requires_grad=True)
    tx = torch.tensor([0.0, -1.0, 0.5], requires_grad=True)
    a = _coefficients(_wall_scene(eps, sigma, tx), solver, {"reflection"}, "vjp")
    assert a.requires_grad
    _loss(a).backward()

    def loss_at(e=4.0, s=0.02, t=(0.0, -1.0, 0.5)):
        with torch.no_grad():
            return float(_loss(_coefficients(_wall_scene(torch.tensor(e), torch.tensor(s), torch.tensor(t)), solver,
                                             {"reflection"}, "none").to(torch.complex128)))

    fd_eps = (loss_at(e=4.0 + 1e-3) - loss_at(e=4.0 - 1e-3)) / 2e-3
    fd_sig = (loss_at(s=0.02 + 1e-3) - loss_at(s=0.02 - 1e-3)) / 2e-3
    assert abs(float(eps.grad) - fd_eps) <= 2e-3 * abs(fd_eps) + 1e-9, (float(eps.grad), fd_eps)
    assert abs(float(sigma.grad) - fd_sig) <= 2e-3 * abs(fd_sig) + 1e-9, (float(sigma.grad), fd_sig)
    base = [0.0, -1.0, 0.5]
    for k in range(3):
        p, m = list(base), list(base)
        p[k] += 1e-3
        m[k] -= 1e-3
        fd = (loss_at(t=p) - loss_at(t=m)) / 2e-3
        assert abs(float(tx.grad[k]) - fd) <= 3e-3 * float(tx.grad.abs().max()) + 1e-9, (k, float(tx.grad[k]), fd)


@pytest.mark.parametrize("solver", ["path", "deterministic"])
def test_transmission_layer_and_frequency_gradients(solver):
    eps = torch.tensor(4.0, requires_grad=True)
    freq = torch.tensor(FREQ, dtype=torch.float64, requires_grad=True)
    a = _coefficients(_sheet_scene(eps), solver, {"transmission"}, "vjp", freq=freq)
    _loss(a).backward()

    def loss_at(e=4.0, f=FREQ):
        with torch.no_grad():
            return float(_loss(_coefficients(_sheet_scene(torch.tensor(e)), solver, {"transmission"}, "none",
                                             freq=f).to(torch.complex128)))

    fd = (loss_at(e=4.0 + 1e-3) - loss_at(e=4.0 - 1e-3)) / 2e-3
    assert abs(float(eps.grad) - fd) <= 2e-3 * abs(fd) + 1e-9, (float(eps.grad), fd)
    fd_f = (loss_at(f=FREQ + 2e4) - loss_at(f=FREQ - 2e4)) / 4e4
    assert abs(float(freq.grad) - fd_f) <= 5e-3 * abs(fd_f) + 1e-15, (float(freq.grad), fd_f)


def test_forward_mode_and_primal_contract():
    import torch.autograd.forward_ad as fwAD

    tx0 = torch.tensor([0.0, -1.0, 0.5])
    u = torch.tensor([0.3, -0.2, 0.5])
    plain = _coefficients(_wall_scene(4.0, 0.02, tx0), "path", {"los", "reflection"}, "none")
    with fwAD.dual_level():
        tx = fwAD.make_dual(tx0.clone(), u)
        a = _coefficients(_wall_scene(4.0, 0.02, tx), "path", {"los", "reflection"}, "jvp")
        primal, tangent = fwAD.unpack_dual(a)
    assert torch.equal(primal, plain)
    h = 1e-3
    ap = _coefficients(_wall_scene(4.0, 0.02, tx0 + h * u), "path", {"los", "reflection"}, "none")
    am = _coefficients(_wall_scene(4.0, 0.02, tx0 - h * u), "path", {"los", "reflection"}, "none")
    fd = (ap.to(torch.complex128) - am.to(torch.complex128)) / (2 * h)
    torch.testing.assert_close(tangent.to(torch.complex128), fd, rtol=0, atol=float(3e-3 * fd.abs().max()))
