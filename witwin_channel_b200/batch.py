"""Batched radiomaps: several scenes, each solved for all its transmitters and
all frequencies in one launch sequence.

A scene's transmitters and frequencies share one geometry pass (visibility,
image chains, edge prefilter): the per-cell kernels test each candidate path
once and evaluate its field at up to four frequencies.  Scenes are issued on
a small pool of CUDA streams without host synchronisation between them, so
small scenes overlap, and their device status words are checked once at the
end.  With ``ad_mode="vjp"`` each scene's records are frozen once and the
fields, accumulation and adjoint run per frequency (``autograd.vjp_forward``).
"""

from __future__ import annotations

from typing import Any

import torch

from . import _native, engine
from .compiler import compile_scene
from .deterministic import Config, _endpoints, _layout, _validate


def _layout_nf(values: torch.Tensor, rx: dict) -> torch.Tensor:
    return torch.stack([_layout(values[f], rx) for f in range(values.shape[0])])


def solve_batch(scenes: list, config: Config, frequencies_hz, *, precision: str = "mixed",
                streams: int = 4) -> list[dict]:
    """Radiomaps of every scene at every frequency: per scene ``path_gain``
    (NF, T, ...) in the single-scene layout (grids as (T, shape[1], shape[0]))
    and ``field`` when ``config.return_field``.  With ``config.ad_mode ==
    "vjp"`` the outputs are differentiable in each scene's values."""
    freqs = [float(f) for f in (frequencies_hz.detach().cpu() if isinstance(frequencies_hz, torch.Tensor)
                                else frequencies_hz)]
    if not 1 <= len(freqs) <= 4:
        raise ValueError("solve_batch takes 1 to 4 frequencies per call")
    for scene in scenes:
        _validate(scene, config)
    if config.ad_mode == "vjp":
        from .autograd import vjp_forward

        out = []
        for scene in scenes:
            v = vjp_forward(scene, config, frequencies_hz)
            rx = v["ep"].rx
            item = {"path_gain": _layout_nf(v["power_total"], rx)}
            if config.return_field:
                item["field"] = _layout_nf(torch.complex(v["field_total_real"], v["field_total_imag"]), rx)
            out.append(item)
        return out
    device = torch.device("cuda", torch.cuda.current_device())
    prec = _native.PRECISION_FP64 if precision == "fp64" else _native.PRECISION_MIXED
    bits = engine.component_bits(config.components)
    pool = [torch.cuda.Stream(device=device) for _ in range(max(1, streams))]
    current = torch.cuda.current_stream(device)
    pending = []
    for i, scene in enumerate(scenes):
        compiled = compile_scene(scene, device)
        ep = _endpoints(scene, device)
        mats = compiled.material_tables(freqs, device)
        cells = engine.alloc_cells(len(freqs), ep.num_tx, ep.num_rx, device, fp64=(prec == _native.PRECISION_FP64))
        s = pool[i % len(pool)]
        s.wait_stream(current)
        with torch.cuda.stream(s):
            # a workspace per scene: concurrent solves must not share scratch
            res = engine.run_solve(compiled, ep, mats, freqs, components=bits, max_depth=config.max_depth,
                                   coherent=config.coherent, precision=prec, cells=cells, check_status=False,
                                   workspace=engine.Workspace())
        # every tensor the stream reads stays referenced until the streams are joined
        pending.append((ep, cells, res["status"], s, (res, mats, compiled)))
    out = []
    for ep, cells, status, s, _alive in pending:
        current.wait_stream(s)
        engine.check_device_status(status)
        rx = ep.rx
        item = {"path_gain": _layout_nf(cells.path_gain, rx)}
        if config.return_field:
            item["field"] = _layout_nf(cells.field, rx)
        out.append(item)
    return out


def single_transmitter_scene(scene: Any, t: int):
    """A copy of ``scene`` with only its transmitter ``t`` (the unbatched form)."""
    from .scene import Scene

    txs = scene.transmitters
    return Scene(structures=scene.structures, endpoints=[txs[t]] + list(scene.receivers),
                 metadata=dict(getattr(scene, "metadata", {})))
