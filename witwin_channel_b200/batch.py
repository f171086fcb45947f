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


class BatchGraph:
    """The batched radiomap forward of a fixed set of scenes, transmitters,
    receivers, materials and frequencies, captured once in a CUDA graph and
    replayed as one graph launch per step.

    Everything a step reads is prepared before the capture and stays resident:
    the compiled scenes, the endpoint and material tables, one workspace and
    one set of cell outputs per scene.  The capture records every scene's
    ``wcb_solve`` on a pool of ``streams`` CUDA streams (and the solve's own
    side stream), so a replay runs them with the same overlap as the eager
    form and no host work or synchronisation between launches.  A change of
    any input value (a moved vertex, a new material value, another frequency)
    needs a new ``BatchGraph``.  ``streams`` may be ``"auto"``: each candidate
    pool size is captured and timed over a few replays, and the fastest graph
    is kept (``tuning`` records the times).

    ``replay()`` returns the per-scene outputs of :func:`solve_batch`;
    ``check()`` reads the scenes' device status words (one synchronisation)."""

    STREAM_CANDIDATES = (1, 2, 4, 8)

    def __init__(self, scenes: list, config: Config, frequencies_hz, *, precision: str = "mixed",
                 streams: int | str = 4, tuning_replays: int = 3) -> None:
        freqs = [float(f) for f in (frequencies_hz.detach().cpu() if isinstance(frequencies_hz, torch.Tensor)
                                    else frequencies_hz)]
        if not 1 <= len(freqs) <= 4:
            raise ValueError("BatchGraph takes 1 to 4 frequencies")
        if config.ad_mode != "none":
            raise ValueError("BatchGraph captures the forward only (ad_mode='none')")
        for scene in scenes:
            _validate(scene, config)
        self.device = torch.device("cuda", torch.cuda.current_device())
        self.config = config
        self.frequencies = freqs
        self._prec = _native.PRECISION_FP64 if precision == "fp64" else _native.PRECISION_MIXED
        self._bits = engine.component_bits(config.components)
        self._items = []
        for scene in scenes:
            compiled = compile_scene(scene, self.device)
            ep = _endpoints(scene, self.device)
            mats = compiled.material_tables(freqs, self.device)
            cells = engine.alloc_cells(len(freqs), ep.num_tx, ep.num_rx, self.device,
                                       fp64=(self._prec == _native.PRECISION_FP64))
            self._items.append({"compiled": compiled, "ep": ep, "mats": mats, "cells": cells,
                                "workspace": engine.Workspace()})
        candidates = self.STREAM_CANDIDATES if streams == "auto" else (int(streams),)
        self.tuning: dict[int, float] = {}
        best = None
        for count in candidates:
            graph, alive = self._capture(count)
            if len(candidates) > 1:
                self.tuning[count] = self._time(graph, tuning_replays)
            if best is None or (len(candidates) > 1 and self.tuning[count] < self.tuning[best[0]]):
                best = (count, graph, alive)
        self.streams, self.graph, self._alive = best

    def _launch(self, pool: list, keep: list) -> None:
        current = torch.cuda.current_stream(self.device)
        pool = pool[:max(1, min(len(pool), len(self._items)))]  # only streams that take work join a capture
        for i, item in enumerate(self._items):
            s = pool[i % len(pool)]
            s.wait_stream(current)
            with torch.cuda.stream(s):
                res = engine.run_solve(item["compiled"], item["ep"], item["mats"], self.frequencies,
                                       components=self._bits, max_depth=self.config.max_depth,
                                       coherent=self.config.coherent, precision=self._prec, cells=item["cells"],
                                       check_status=False, workspace=item["workspace"])
            keep.append(res)
        for s in pool:
            current.wait_stream(s)

    def _capture(self, count: int):
        pool = [torch.cuda.Stream(device=self.device) for _ in range(max(1, count))]
        # an eager run first: sizes the workspaces and loads every kernel
        warm: list = []
        self._launch(pool, warm)
        torch.cuda.synchronize(self.device)
        for res in warm:
            engine.check_device_status(res["status"])
        graph = torch.cuda.CUDAGraph()
        keep: list = []
        with torch.cuda.graph(graph):
            self._launch(pool, keep)
        return graph, (pool, keep)

    def _time(self, graph, replays: int) -> float:
        graph.replay()
        torch.cuda.synchronize(self.device)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(max(1, replays)):
            graph.replay()
        e1.record()
        torch.cuda.synchronize(self.device)
        return e0.elapsed_time(e1) / max(1, replays)

    def replay(self) -> list[dict]:
        self.graph.replay()
        out = []
        for item in self._items:
            rx = item["ep"].rx
            res = {"path_gain": _layout_nf(item["cells"].path_gain, rx)}
            if self.config.return_field:
                res["field"] = _layout_nf(item["cells"].field, rx)
            out.append(res)
        return out

    def check(self) -> None:
        for res in self._alive[1]:
            engine.check_device_status(res["status"])
