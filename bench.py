"""Benchmark: deterministic radiomap on the 64-box urban canyon.

Workload (one "step"): one full radiomap solve of a seeded 64-box urban canyon
(8x8 lots of 50 m, 770 triangles), one transmitter at 25 m on a street,
256x256 receiver grid at 1.5 m with 1.5 m spacing, 28 GHz, line of sight +
specular reflection to depth 3 + first-order UTD diffraction, coherent
accumulation.  Data are synthetic (seeded); no dataset is read.

* ``value``: rays per second (segment visibility/penetration queries plus the
  discovery bounces) over the whole job, inputs resident in HBM, the L2
  flushed (256 MiB write) before every timed step, device time from CUDA
  events, max over ranks.
* ``e2e``: the same metric through the public ``solve()`` call with host
  inputs and the radiomap copied back to host every step.
* ``roofline``: the fused main kernel's algorithmic bytes (64*ceil(log2 F)+48
  per ray, 84 per output cell) over its event-timed duration, against the
  measured HBM copy bandwidth.
* ``cpu_baseline``: the FP64 NumPy oracle on a bounded sample of receiver
  cells with its per-transmitter discovery amortised over the full grid.

Multi-GPU: one process per GPU; every rank solves its own transmitter
position (weak scaling, no data-path collective); the step time is the max
over ranks.
"""

from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "radiomap rays/s (urban canyon, 64 boxes, 256x256 grid, 28 GHz, depth 3 + UTD)"
UNIT = "rays/s"
HBM_FALLBACK = 6650.0
PROFILE_SUMMARY = ROOT / "profiles" / "urban_canyon_kernels.md"


def _peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return json.loads(p.read_text())
        except Exception:
            pass
    return {}


def _traffic_per_launch(kernel: str) -> float | None:
    """DRAM bytes per launch of `kernel` from the committed ncu summary
    (a line ``traffic_bytes_per_launch[<kernel>]: <bytes>``)."""
    if not PROFILE_SUMMARY.exists():
        return None
    key = f"traffic_bytes_per_launch[{kernel}]:"
    for line in PROFILE_SUMMARY.read_text().splitlines():
        if line.strip().startswith(key):
            try:
                return float(line.split(":", 1)[1].strip())
            except ValueError:
                return None
    return None


class ClockSampler:
    """nvidia-smi clocks/throttle sampling during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.samples: list[list[str]] = []
        self._stop = threading.Event()
        self._thread: threading.Thread | None = None

    def _run(self) -> None:
        while not self._stop.is_set():
            try:
                out = subprocess.run(
                    ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits"],
                    capture_output=True, text=True, timeout=5)
                if out.returncode == 0 and out.stdout.strip():
                    self.samples.append([x.strip() for x in out.stdout.strip().split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._thread = threading.Thread(target=self._run, daemon=True)
        self._thread.start()
        return self

    def __exit__(self, *exc):
        self._stop.set()
        if self._thread:
            self._thread.join(timeout=10)

    def summary(self) -> dict:
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm = sorted(float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit())
        mx = max((float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()), default=None)
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if len(s) > 3 + i and s[3 + i] == "Active"})
        return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": mx, "reasons": reasons,
                "samples": len(self.samples)}


def _bytes_per_ray(faces: int) -> int:
    return 64 * int(math.ceil(math.log2(max(faces, 2)))) + 48


B_CELL = 84


def run_native(args) -> None:
    import torch
    import torch.distributed as dist

    from witwin_channel_b200 import Config, _native, engine, solve
    from witwin_channel_b200.compiler import compile_scene
    from witwin_channel_b200.deterministic import _endpoints
    from witwin_channel_b200.workloads import urban_canyon_scene

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    scene, freq = urban_canyon_scene(seed=1)
    if rank > 0:
        # weak scaling: each rank solves its own transmitter on the same city
        import numpy as np

        from witwin_channel_b200.scene import make_transmitter
        from witwin_channel_b200.workloads import city_layout, street_point

        layout = city_layout(64, 1)
        tx = street_point(layout, np.random.default_rng(5000 + rank), 25.0)
        scene.endpoints[0] = make_transmitter(tx)
    cfg = Config(components={"los", "reflection", "diffraction"}, max_depth=3)
    compiled = compile_scene(scene, device)
    ep = _endpoints(scene, device)
    mats = compiled.material_tables([freq], device)
    bits = engine.component_bits(cfg.components)
    cells = engine.alloc_cells(1, ep.num_tx, ep.num_rx, device)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=device)
    faces = compiled.native.num_faces

    def step():
        engine.run_solve(compiled, ep, mats, [freq], components=bits, max_depth=cfg.max_depth, coherent=True, cells=cells)

    _native.profile_enable(True)
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    launches0 = _native.launch_count()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    rays = 0
    main_rays = 0
    main_ms = 0.0
    main_launches = 0
    kernel_ms: dict[str, float] = {}
    kernel_rays: dict[str, int] = {}
    last_prof: dict = {}
    sampler = ClockSampler(local)
    t_wall0 = time.perf_counter()
    with sampler:
        torch.cuda.synchronize()
        for i in range(args.steps):
            flush.fill_(i & 0xFF)  # L2 flush, outside the timed interval
            starts[i].record()
            step()
            ends[i].record()
            prof = _native.profile_read()
            rays += prof["rays"] + prof["prep_rays"]
            main_rays += prof["rays"]
            main_ms += prof["main_ms"]
            main_launches += prof["main_launches"]
            for k, v in prof["kernel_ms"].items():
                kernel_ms[k] = kernel_ms.get(k, 0.0) + v
            for k, v in prof["kernel_rays"].items():
                kernel_rays[k] = kernel_rays.get(k, 0) + v
            last_prof = prof
        torch.cuda.synchronize()
    t_wall = time.perf_counter() - t_wall0
    launches = _native.launch_count() - launches0
    step_ms = sum(s.elapsed_time(e) for s, e in zip(starts, ends))
    if world > 1:
        t = torch.tensor([step_ms, float(rays)], dtype=torch.float64, device=device)
        tmax = t.clone()
        dist.all_reduce(tmax[:1], op=dist.ReduceOp.MAX)
        dist.all_reduce(t[1:], op=dist.ReduceOp.SUM)
        step_ms_all, rays_all = float(tmax[0]), float(t[1])
    else:
        step_ms_all, rays_all = step_ms, float(rays)
    value = rays_all / (step_ms_all / 1000.0)
    # e2e through the public API: host inputs, radiomap back to host
    e2e_steps = max(1, args.steps)
    _native.profile_enable(False)
    cfg_api = Config(components={"los", "reflection", "diffraction"}, max_depth=3, return_field=False)
    for _ in range(2):
        solve(scene, cfg_api, reference_frequency_hz=freq).path_gain.cpu()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    h2d = 0
    d2h = 0
    e0.record()
    for _ in range(e2e_steps):
        res = solve(scene, cfg_api, reference_frequency_hz=freq)
        host = res.path_gain.cpu()
        d2h += host.numel() * host.element_size()
        h2d += ep.tx_pos.numel() * 4 + ep.tx_power.numel() * 4 + ep.tx_pol.numel() * 4 + 4 * 5 * mats.eps_r.numel()
    e1.record()
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1)
    if world > 1:
        t = torch.tensor([e2e_ms], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t[0])
    e2e_value = rays_all / args.steps * e2e_steps / (e2e_ms / 1000.0)
    if rank == 0:
        peaks = _peaks()
        hbm = float(peaks.get("hbm_gbs", HBM_FALLBACK))
        cells_n = ep.num_tx * ep.num_rx
        # dominant per-cell kernel: its rays and the slot bytes it writes per cell
        dominant = max(("k_reflect", "k_diffract", "k_los_trans"), key=lambda k: kernel_ms.get(k, 0.0))
        cell_bytes = {"k_reflect": 12, "k_diffract": 16, "k_los_trans": 12}[dominant]
        bytes_per_launch = kernel_rays.get(dominant, 0) / args.steps * _bytes_per_ray(faces) + cells_n * cell_bytes
        launch_ms = kernel_ms.get(dominant, 0.0) / args.steps
        achieved = bytes_per_launch / (launch_ms / 1000.0) / 1e9 if launch_ms > 0 else 0.0
        traffic = _traffic_per_launch(dominant)
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            cpu = cpu_baseline(scene, freq, cfg, budget_s=args.cpu_budget, cores=1)
        line = {
            "metric": METRIC,
            "value": value,
            "unit": UNIT,
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": step_ms_all / args.steps,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "fp32+fp64",
            "data": "synthetic (seeded 64-box canyon)",
            "config": {
                "workload": "urban canyon: 64 boxes on 8x8 lots of 50 m (770 triangles), 1 Tx at 25 m, "
                            "256x256 grid at 1.5 m spacing, 28 GHz, LoS + reflection depth 3 + UTD order 1",
                "triangles": faces,
                "grid": [256, 256],
                "frequency_hz": freq,
                "max_depth": 3,
                "rays_per_step": rays / args.steps,
                "per_cell_kernel_rays_per_step": main_rays / args.steps,
                "kernel_ms_per_step": {k: v / args.steps for k, v in kernel_ms.items()},
                "kernel_rays_per_step": {k: v / args.steps for k, v in kernel_rays.items()},
                "reflection_candidates_per_depth": last_prof.get("chains"),
                "diffraction_edges_after_prefilter": last_prof.get("edges"),
                "cells_per_step": cells_n,
                "l2": "flushed (256 MiB write) before every timed step",
                "parallelism": f"replicas x{world} (one transmitter per rank)",
            },
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d // e2e_steps,
                    "d2h_bytes_per_step": d2h // e2e_steps, "ms_per_step": e2e_ms / e2e_steps},
            "roofline": {
                "bound": "hbm",
                "kernel": dominant,
                "achieved": achieved,
                "peak": hbm,
                "unit": "GB/s",
                "frac": achieved / hbm,
                "peak_source": "measured" if "hbm_gbs" in peaks else "fallback",
                "traffic": traffic,
                "algorithmic_bytes_per_launch": bytes_per_launch,
                "launch_ms": launch_ms,
            },
            "cpu_baseline": cpu,
            "gpu_launches": launches,
            "clocks": sampler.summary(),
            "wall_s": t_wall,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


# --------------------------------------------------------------------------
# CPU side (oracle): used for the cpu_baseline field and the reference arm
# --------------------------------------------------------------------------
def _cpu_worker(payload):
    import numpy as np

    from oracle import geom
    from oracle import solve as osolve

    arrays, rx_idx, kw, discovered = payload
    sub = dict(arrays)
    sub["rx_pos"] = arrays["rx_pos"][rx_idx]
    sub["rx_pol"] = arrays["rx_pol"][rx_idx]
    geom.RAY_COUNTER[0] = 0
    t0 = time.perf_counter()
    osolve.solve(sub, discovered=discovered, **kw)
    return time.perf_counter() - t0, geom.RAY_COUNTER[0], len(rx_idx)


def cpu_baseline(scene, freq, cfg, *, budget_s: float = 15.0, cores: int = 1, sample_cells: int | None = None) -> dict:
    """Oracle rays/s on a bounded sample of receiver cells.

    The per-transmitter discovery (262,144 Fibonacci rays x depth) runs once
    and its cost is amortised over the full grid; the per-cell work runs on
    ``sample_cells`` cells spread over the grid, on ``cores`` processes."""
    import multiprocessing as mp

    import numpy as np

    from oracle import geom
    from oracle import solve as osolve

    arrays = osolve.scene_arrays(scene, freq)
    R = arrays["rx_pos"].shape[0]
    kw = dict(components=set(cfg.components), max_depth=cfg.max_depth, coherent=cfg.coherent, frequency=freq)
    geom.RAY_COUNTER[0] = 0
    t0 = time.perf_counter()
    discovered = osolve.discover(arrays, max_depth=cfg.max_depth)
    t_disc = time.perf_counter() - t0
    disc_rays = geom.RAY_COUNTER[0]
    n = sample_cells or max(cores * 2, 8)
    rng = np.random.default_rng(0)
    cells = np.sort(rng.choice(R, size=min(n, R), replace=False))
    chunks = [c for c in np.array_split(cells, max(cores, 1)) if len(c)]
    t1 = time.perf_counter()
    if cores > 1:
        ctx = mp.get_context("spawn")
        with ctx.Pool(cores) as pool:
            res = pool.map(_cpu_worker, [(arrays, c, kw, discovered) for c in chunks])
    else:
        res = [_cpu_worker((arrays, c, kw, discovered)) for c in chunks]
    t_cells = time.perf_counter() - t1
    rays_cells = sum(r[1] for r in res)
    ncell = sum(r[2] for r in res)
    # full-grid extrapolation: per-cell rate on the sample + discovery once
    rate_cells = rays_cells / t_cells
    full_rays = disc_rays + rays_cells / ncell * R
    full_time = t_disc + t_cells / ncell * R
    return {
        "value": full_rays / full_time,
        "unit": UNIT,
        "cores": cores,
        "kind": "port",
        "sample": f"FP64 NumPy oracle, {ncell} of {R} cells (random, seed 0) on {cores} process(es); "
                  f"discovery of {disc_rays} ray bounces once ({t_disc:.1f} s) amortised over the grid; "
                  f"per-cell rate {rate_cells:.3g} rays/s",
        "seconds": t_disc + t_cells,
    }


def run_reference(args) -> None:
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from witwin_channel_b200 import Config
    from witwin_channel_b200.workloads import urban_canyon_scene

    scene, freq = urban_canyon_scene(seed=1)
    cfg = Config(components={"los", "reflection", "diffraction"}, max_depth=3)
    cores = os.cpu_count() or 1
    samples = []
    t_all = time.perf_counter()
    for i in range(args.warmup + args.steps):
        r = cpu_baseline(scene, freq, cfg, budget_s=args.cpu_budget, cores=cores, sample_cells=cores * 2)
        if i >= args.warmup:
            samples.append(r)
    value = sorted(s["value"] for s in samples)[len(samples) // 2]
    line = {
        "impl": "reference",
        "metric": METRIC,
        "value": value,
        "unit": UNIT,
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": (time.perf_counter() - t_all) * 1000.0 / max(args.steps + args.warmup, 1),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "fp64",
        "data": "synthetic (seeded 64-box canyon)",
        "config": {"workload": "urban canyon: 64 boxes, 256x256 grid, 28 GHz, LoS + reflection depth 3 + UTD order 1",
                   "implementation": "FP64 NumPy oracle of the reference algorithm on host cores "
                                     "(the reference's CUDA build needs the absent RayD/OptiX sources)"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port", "sample": samples[-1]["sample"]},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="native", choices=["native", "reference"])
    ap.add_argument("--cpu-budget", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "native":
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_native(args)


if __name__ == "__main__":
    main()
