"""Batched solves (several scenes x transmitters x frequencies per launch
sequence) against one solve per (scene, transmitter, frequency)."""

from __future__ import annotations

import pytest
import torch

from tests import scenes as sc
from witwin_channel_b200 import Config, solve
from witwin_channel_b200.batch import single_transmitter_scene, solve_batch
from witwin_channel_b200.scene import Scene, make_transmitter

pytestmark = pytest.mark.gpu
FREQS = (3.5e9, 28.0e9)


def _two_tx_city(seed):
    scene, _ = sc.small_city(n_boxes=4, seed=seed, grid=(12, 10))
    txs = scene.transmitters
    extra = make_transmitter([float(txs[0].position[0]) + 3.0, float(txs[0].position[1]) - 2.0, 8.0])
    return Scene(structures=scene.structures, endpoints=[txs[0], extra] + list(scene.receivers))


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_batch_matches_single_solves(precision):
    scenes = [_two_tx_city(3), _two_tx_city(4)]
    cfg = Config(components={"los", "reflection", "diffraction"}, max_depth=2)
    out = solve_batch(scenes, cfg, FREQS, precision=precision)
    for scene, res in zip(scenes, out):
        assert tuple(res["path_gain"].shape[:2]) == (len(FREQS), 2)
        for t in range(2):
            sub = single_transmitter_scene(scene, t)
            for fi, f in enumerate(FREQS):
                ref = solve(sub, cfg, reference_frequency_hz=f, precision=precision).path_gain[0].double().cpu()
                got = res["path_gain"][fi, t].double().cpu()
                # 1e-3 dB on every cell above 1e-5 of the map's maximum (interference nulls aside)
                assert torch.all((got - ref).abs() <= 2.3e-4 * ref + 1e-5 * float(ref.max()))


def test_batch_vjp_matches_single_frequency_vjps():
    scene = _two_tx_city(5)
    eps = torch.tensor(5.24, dtype=torch.float64, requires_grad=True)
    shared = type(scene.structures[1].material)(eps_r=eps, sigma_e=0.2, thickness_m=0.3)
    for st in scene.structures[1:]:
        st.material = shared
    cfg = Config(components={"los", "reflection", "diffraction"}, max_depth=2, ad_mode="vjp")
    freqs = torch.tensor(FREQS, dtype=torch.float64, requires_grad=True)
    (batch,) = solve_batch([scene], cfg, freqs)
    w = torch.rand(batch["path_gain"].shape, generator=torch.Generator().manual_seed(0), dtype=torch.float64).cuda()
    scale = batch["path_gain"].detach().max()
    (w * batch["path_gain"] / scale).sum().backward()
    g_eps, g_f = float(eps.grad), freqs.grad.clone()
    eps.grad = None
    total_eps = 0.0
    for fi, f in enumerate(FREQS):
        ft = torch.tensor(f, dtype=torch.float64, requires_grad=True)
        res = solve(scene, cfg, reference_frequency_hz=ft)
        (w[fi] * res.path_gain / scale).sum().backward()
        total_eps += float(eps.grad)
        eps.grad = None
        # same records, same FP64 adjoint; the cotangents pass through FP32 outputs
        assert abs(float(ft.grad) - float(g_f[fi])) <= 1e-6 * max(abs(float(ft.grad)), 1e-30) + 1e-30
    assert abs(g_eps - total_eps) <= 1e-6 * abs(total_eps)


def test_captured_batch_graph_replays_the_eager_batch():
    """A ``BatchGraph`` (the batched forward captured once in a CUDA graph)
    reproduces the eager batched forward bit for bit on every replay, with a
    fixed stream pool and with the pool size picked by timing."""
    from witwin_channel_b200.batch import BatchGraph

    scenes = [_two_tx_city(6), _two_tx_city(7), _two_tx_city(8)]
    cfg = Config(components={"los", "reflection", "diffraction"}, max_depth=2)
    eager = solve_batch(scenes, cfg, FREQS)
    graph = BatchGraph(scenes, cfg, FREQS, streams=2)
    for _ in range(2):
        out = graph.replay()
        graph.check()
        for a, b in zip(out, eager):
            assert torch.equal(a["path_gain"], b["path_gain"])
            assert torch.equal(a["field"], b["field"])
    tuned = BatchGraph(scenes, cfg, FREQS, streams="auto", tuning_replays=2)
    assert set(tuned.tuning) == set(BatchGraph.STREAM_CANDIDATES)
    assert tuned.streams == min(tuned.tuning, key=tuned.tuning.get)
    for a, b in zip(tuned.replay(), eager):
        assert torch.equal(a["path_gain"], b["path_gain"])
    with pytest.raises(ValueError):
        BatchGraph(scenes, Config(components={"los"}, ad_mode="vjp"), FREQS)


def test_all_frequency_linearisation_equals_per_frequency_fields():
    """``wcb_rows_jvp`` with ``freq_index=-1`` (every frequency in one pass,
    diffraction geometry shared) gives each frequency's FP64 record fields."""
    from witwin_channel_b200 import autograd as ad

    scene = _two_tx_city(9)
    cfg = Config(components={"los", "reflection", "diffraction"}, max_depth=2, ad_mode="vjp")
    freqs = torch.tensor((3.5e9, 6.0e9, 28.0e9, 39.0e9), dtype=torch.float64, requires_grad=True)
    v = ad.vjp_forward(scene, cfg, freqs)
    assert v["count"] > 0
    state = v["power_total"].grad_fn.state  # the autograd node keeps the frozen records
    both = ad.rows_field64_all(state)
    assert tuple(both.shape) == (4, v["count"], 2)
    for fi in range(4):
        one, _ = ad.rows_jvp(state, fi, None)
        torch.testing.assert_close(both[fi], one, rtol=1e-12, atol=1e-30)
