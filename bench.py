"""Benchmark: batched deterministic radiomaps, forward + VJP.

Workload (one "step"): eight seeded scenes of 16..256 boxes (grids 64^2 to
512^2 at 4..1 m spacing), each with 4 transmitters at 5-40 m on streets and 4
frequencies {3.5, 6, 28, 39} GHz, line of sight + specular reflection to depth
3 + first-order UTD diffraction, coherent accumulation.  A step is the
differentiable batched forward of every (scene, transmitter, frequency) job
(``solve_batch`` with ``ad_mode="vjp"``: the radiomaps, mixed precision
record search) and the VJP of the summed radiomaps with respect to each
scene's concrete eps_r and sigma_e and every transmitter position.  Data are
synthetic (seeded); no dataset is read.

* ``value``: rays per second (segment visibility/penetration queries plus the
  discovery bounces of every solve in the step) over the whole job, the L2
  flushed (256 MiB write) before every timed step, device time from CUDA
  events, max over ranks.
* ``e2e``: the same steps with every radiomap and gradient copied back to
  host memory, timed by the host clock.
* ``roofline``: the step's dominant kernel by serialised time (the
  reverse-mode diffraction VJP) against the instruction-issue bound: its
  warp instructions per record (ncu) x records per launch over its live
  event-timed duration, against 148 SMs x 4 schedulers x the sampled SM clock.
* ``fp64_plain``: the same jobs in the plain FP64 single-transmitter form
  (one FP64 differentiable forward and its VJP per scene, transmitter and
  frequency).
* ``cpu_baseline``: the FP64 NumPy oracle on a bounded sample of the workload.
* side legs: the urban canyon radiomap (``canyon``), the canyon gradient step
  (``vjp``), the large city with transmission and CFR (``large``) and the
  propagation consumer (``consumer``).

Multi-GPU: one process per GPU; the 32 (scene, transmitter) jobs are
partitioned across ranks by a longest-processing-time assignment (cost: grid
cells x boxes), each rank runs its jobs' forward and VJP, and the per-scene
material gradients are summed across ranks with one all-reduce per step (the
only collective); strong scaling, step time the max over ranks.
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

METRIC = ("radiomap rays/s and VJP step time (batched forward + VJP: 8 scenes of 16..256 boxes, 4 Tx x 4 "
          "frequencies each, depth 3 + UTD)")
UNIT = "rays/s"
HBM_FALLBACK = 6650.0
CANYON_PROFILE = ROOT / "profiles" / "urban_canyon_kernels.md"
BATCHED_PROFILE = ROOT / "profiles" / "batched_vjp_kernels.md"
WORKLOAD = ("urban canyon: 64 boxes on 8x8 lots of 50 m (770 triangles), 1 Tx at 25 m, 256x256 grid at 1.5 m "
            "spacing, 28 GHz, LoS + reflection depth 3 + UTD order 1")
BATCHED_WORKLOAD = ("batched: 8 seeded scenes (16, 32, 48, 64, 96, 128, 192, 256 boxes), grids 64^2..512^2 at 4..1 m, "
                    "4 Tx at 5-40 m x {3.5, 6, 28, 39} GHz per scene, LoS + reflection depth 3 + UTD order 1; step = "
                    "the differentiable batched forward (every job's radiomap, mixed precision) and the VJP of the "
                    "summed radiomaps w.r.t. each scene's concrete eps_r, sigma_e and Tx positions")


def _peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return json.loads(p.read_text())
        except Exception:
            pass
    return {}


def _profile_figure(path: Path, key: str) -> float | None:
    """A figure from a committed ncu summary: the number on the line
    ``<key>: <number>`` (e.g. ``traffic_bytes_per_launch[k_reflect]: 1742080``)."""
    if not path.exists():
        return None
    for line in path.read_text().splitlines():
        if line.strip().startswith(key + ":"):
            try:
                return float(line.split(":", 1)[1].strip().split()[0])
            except (ValueError, IndexError):
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
        self._proc: subprocess.Popen | None = None
        self._thread: threading.Thread | None = None

    def _read(self) -> None:
        assert self._proc is not None and self._proc.stdout is not None
        for line in self._proc.stdout:
            parts = [x.strip() for x in line.strip().split(",")]
            if len(parts) >= 7:
                self.samples.append(parts)

    def __enter__(self):
        # one nvidia-smi process sampling every 50 ms, started before and stopped after the timed region
        try:
            self._proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "50"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._thread = threading.Thread(target=self._read, daemon=True)
            self._thread.start()
            time.sleep(0.1)
        except Exception:
            self._proc = None
        return self

    def __exit__(self, *exc):
        if self._proc is not None:
            time.sleep(0.06)
            self._proc.terminate()
            try:
                self._proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self._proc.kill()
        if self._thread:
            self._thread.join(timeout=5)

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


def _batched_jobs(world: int, rank: int) -> list[tuple[int, int]]:
    """This rank's (scene, transmitter) jobs: a longest-processing-time
    assignment of the 32 jobs by cost (grid cells x boxes), ties to the lower
    rank, so every rank computes the same partition."""
    from witwin_channel_b200.workloads import BATCH_BOXES, BATCH_GRID

    jobs = sorted(((BATCH_GRID[s] ** 2 * BATCH_BOXES[s], s, t) for s in range(len(BATCH_BOXES)) for t in range(4)),
                  key=lambda x: (-x[0], x[1], x[2]))
    load = [0] * world
    mine = []
    for cost, s, t in jobs:
        r = min(range(world), key=lambda i: (load[i], i))
        load[r] += cost
        if r == rank:
            mine.append((s, t))
    return sorted(mine)


def _batched_setup(jobs: list[tuple[int, int]]):
    """The workload's scenes restricted to ``jobs`` with their differentiable
    values: one concrete material per scene with eps_r / sigma_e leaves (made
    for all eight scenes, so every rank holds the same material leaves) and
    the jobs' transmitter positions as leaves."""
    import torch

    from witwin_channel_b200.scene import PhysicalMaterial, Scene
    from witwin_channel_b200.workloads import batched_scenes

    full = batched_scenes()
    materials, scenes, tx_leaves = [], [], []
    for s, sc in enumerate(full):
        eps = torch.tensor(5.24, dtype=torch.float64, requires_grad=True)
        sig = torch.tensor(0.5, dtype=torch.float64, requires_grad=True)
        materials += [eps, sig]
        mat = PhysicalMaterial(eps_r=eps, sigma_e=sig, thickness_m=0.3, name="concrete")
        for st in sc.structures[1:]:
            st.material = mat
        for a in sc.transmitters:
            a.position = a.position.detach().clone().requires_grad_(True)
        picked = [sc.transmitters[t] for (ss, t) in jobs if ss == s]
        if not picked:
            continue
        tx_leaves += [a.position for a in picked]
        scenes.append(Scene(structures=sc.structures, endpoints=picked + list(sc.receivers),
                            metadata=dict(getattr(sc, "metadata", {}) or {})))
    return full, scenes, materials, tx_leaves


def run_leg(args) -> None:
    """One side leg alone (``--only-leg``), its dict printed as one JSON line:
    the small workloads the committed ncu summaries are captured on."""
    import torch

    torch.cuda.set_device(0)
    device = torch.device("cuda", 0)
    if args.only_leg == "canyon":
        leg = _canyon_run(args, device)
    elif args.only_leg == "consumer":
        leg = _consumer_run(device)
    elif args.only_leg == "large":
        leg = _large_run(device)
    else:
        leg = _vjp_run(device)
    print(json.dumps({"leg": args.only_leg, **leg}), flush=True)


def run_native(args) -> None:
    import torch
    import torch.distributed as dist

    from witwin_channel_b200 import Config, _native
    from witwin_channel_b200.batch import solve_batch
    from witwin_channel_b200.sharding import allreduce_gradients
    from witwin_channel_b200.workloads import BATCH_FREQS

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    jobs = _batched_jobs(world, rank)
    full, scenes, materials, tx_leaves = _batched_setup(jobs)
    leaves = materials + tx_leaves
    comps = {"los", "reflection", "diffraction"}
    cfg_ad = Config(components=comps, max_depth=3, ad_mode="vjp", return_field=False)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=device)

    def step(host_out: list | None = None):
        # the differentiable batched forward (every job's radiomap) and its VJP
        for t in leaves:
            t.grad = None
        res = solve_batch(scenes, cfg_ad, BATCH_FREQS) if scenes else []
        if res:
            loss = sum(r["path_gain"].double().sum() for r in res) * 1e6
            loss.backward()
        if world > 1:
            allreduce_gradients(materials)  # the scenes' material gradients over the ranks' jobs
        if host_out is not None:
            for r in res:
                host_out.append(r["path_gain"].detach().cpu())
            for t in leaves:
                if t.grad is not None:
                    host_out.append(t.grad.detach().cpu())
        return res

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    # rays traced per step and the live duration of the reverse-mode
    # diffraction VJP kernel, from one profiled (untimed) step
    _native.profile_enable(True)
    step()
    torch.cuda.synchronize()
    prof = _native.profile_read()
    _native.profile_enable(False)
    rays_per_step = float(prof["acc_rays"])
    vjp_ms, vjp_records, vjp_launches = (prof["acc_vjp_diffraction_ms"], prof["acc_vjp_diffraction_records"],
                                         prof["acc_vjp_diffraction_launches"])
    if world > 1:
        dist.barrier()
    launches0 = _native.launch_count()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    sampler = ClockSampler(local)
    t_wall0 = time.perf_counter()
    with sampler:
        torch.cuda.synchronize()
        for i in range(args.steps):
            flush.fill_(i & 0xFF)  # L2 flush, outside the timed interval
            starts[i].record()
            step()
            ends[i].record()
        torch.cuda.synchronize()
    t_wall = time.perf_counter() - t_wall0
    launches = _native.launch_count() - launches0
    per_step = [a.elapsed_time(b) for a, b in zip(starts, ends)]
    step_ms = sum(per_step)
    # e2e: the same steps with every radiomap and gradient copied to host memory, host clock
    e2e_steps = max(1, min(args.steps, 5))
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    t0 = time.perf_counter()
    d2h = 0
    for _ in range(e2e_steps):
        out: list = []
        step(out)
        d2h += sum(x.numel() * x.element_size() for x in out)
    torch.cuda.synchronize()
    e2e_ms = (time.perf_counter() - t0) * 1e3
    # inputs a step copies host -> device: transmitter positions and the material scalars
    h2d = sum(3 * 4 for _ in tx_leaves) + 16 * len(scenes) + 4 * 4
    if world > 1:
        t = torch.tensor([step_ms, e2e_ms], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        step_ms_all, e2e_ms_all = float(t[0]), float(t[1])
        r = torch.tensor([rays_per_step], dtype=torch.float64, device=device)
        dist.all_reduce(r, op=dist.ReduceOp.SUM)
        rays_all = float(r[0])
    else:
        step_ms_all, e2e_ms_all, rays_all = step_ms, e2e_ms, rays_per_step
    value = rays_all * args.steps / (step_ms_all / 1000.0)
    e2e_value = rays_all * e2e_steps / (e2e_ms_all / 1000.0)
    single = world == 1
    plain = None if (args.no_batched or not single) else _batched_plain(full, device)
    forward_graph = None if (args.no_batched or not single) else _batched_forward_graph(full, device)
    canyon = None if (args.no_canyon or not single) else _canyon_run(args, device)
    vjp = None if (args.no_vjp or not single) else _vjp_run(device)
    large = None if (args.no_large or not single) else _large_run(device)
    consumer_leg = None if (args.no_consumer or not single) else _consumer_run(device)
    if rank == 0:
        clocks = sampler.summary()
        # issue-bound roofline of the dominant kernel (the reverse-mode diffraction VJP)
        inst_per_record = _profile_figure(BATCHED_PROFILE, "warp_instructions_per_record[k_vjp_diffraction]")
        dram_per_record = _profile_figure(BATCHED_PROFILE, "dram_bytes_per_record[k_vjp_diffraction]")
        l2_per_record = _profile_figure(BATCHED_PROFILE, "l2_bytes_per_record[k_vjp_diffraction]")
        sm_mhz = clocks.get("sm_mhz") or 1965.0
        launch_ms = vjp_ms / max(vjp_launches, 1)
        records_per_launch = vjp_records / max(vjp_launches, 1)
        peak_issue = 148 * 4 * sm_mhz * 1e6  # warp instructions per second: 4 schedulers x 148 SMs
        achieved = (inst_per_record * records_per_launch / (launch_ms / 1000.0)) if (inst_per_record and launch_ms) \
            else None
        roofline = {
            "bound": "issue",
            "kernel": "k_vjp_diffraction",
            "achieved": achieved,
            "peak": peak_issue,
            "unit": "warp instructions/s",
            "frac": achieved / peak_issue if achieved else None,
            "traffic": dram_per_record * records_per_launch if dram_per_record else None,
            "l2_bytes_per_launch": l2_per_record * records_per_launch if l2_per_record else None,
            "launch_ms": launch_ms,
            "records_per_launch": records_per_launch,
            "per_record_figures": "warp instructions, DRAM and L2 bytes per record from the committed ncu summary "
                                  "profiles/batched_vjp_kernels.md",
            "hbm_peak_gbs": float(_peaks().get("hbm_gbs", HBM_FALLBACK)),
        }
        cpu = None if args.no_cpu_baseline or not single else batched_cpu_baseline(full, cores=1)
        line = {
            "metric": METRIC,
            "value": value,
            "unit": UNIT,
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": step_ms_all / args.steps,
            "higher_is_better": True,
            "scaling": "strong",
            "vs_baseline": None,
            "dtype": "fp32+fp64",
            "data": "synthetic (seeded scenes)",
            "config": {
                "workload": BATCHED_WORKLOAD,
                "scenes": len(full),
                "jobs_this_rank": len(jobs),
                "frequencies_hz": list(BATCH_FREQS),
                "max_depth": 3,
                "rays_per_step": rays_all,
                "per_step_ms": [round(x, 3) for x in per_step],
                "l2": "flushed (256 MiB write) before every timed step",
                "parallelism": (f"{world} ranks: the 32 (scene, Tx) jobs partitioned (longest processing time first), "
                                "material gradients summed by one all-reduce per step") if world > 1 else "single GPU",
            },
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h // e2e_steps, "ms_per_step": e2e_ms_all / e2e_steps},
            "roofline": roofline,
            "cpu_baseline": cpu,
            "fp64_plain": None if plain is None else dict(
                plain, speedup=plain["ms_per_step"] / (step_ms_all / args.steps),
                batched_ms_per_step=step_ms_all / args.steps),
            "forward_graph": forward_graph,
            "canyon": canyon,
            "vjp": vjp,
            "large": large,
            "consumer": consumer_leg,
            "gpu_launches": launches,
            "clocks": clocks,
            "wall_s": t_wall,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def _canyon_run(args, device, steps: int = 50) -> dict:
    """The urban canyon radiomap (64 boxes, 256x256 grid, 28 GHz, depth 3 +
    UTD): per-step device time with inputs resident and the L2 flushed, the
    same metric end to end through ``solve()``, the kernels' bound and the
    plain FP64 comparison."""
    import torch

    from witwin_channel_b200 import Config, _native, engine, solve
    from witwin_channel_b200.compiler import compile_scene
    from witwin_channel_b200.deterministic import _endpoints
    from witwin_channel_b200.workloads import urban_canyon_scene

    scene, freq = urban_canyon_scene(seed=1)
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
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    rays = 0
    main_rays = 0
    kernel_ms: dict[str, float] = {}
    kernel_rays: dict[str, int] = {}
    last_prof: dict = {}
    torch.cuda.synchronize()
    for i in range(steps):
        flush.fill_(i & 0xFF)  # L2 flush, outside the timed interval
        starts[i].record()
        step()
        ends[i].record()
        prof = _native.profile_read()
        rays += prof["rays"] + prof["prep_rays"]
        main_rays += prof["rays"]
        for k, v in prof["kernel_ms"].items():
            kernel_ms[k] = kernel_ms.get(k, 0.0) + v
        for k, v in prof["kernel_rays"].items():
            kernel_rays[k] = kernel_rays.get(k, 0) + v
        last_prof = prof
    torch.cuda.synchronize()
    _native.profile_enable(False)
    step_ms = sum(s_.elapsed_time(e_) for s_, e_ in zip(starts, ends))
    value = rays / (step_ms / 1000.0)
    # e2e through the public API: host inputs, radiomap back to host
    cfg_api = Config(components={"los", "reflection", "diffraction"}, max_depth=3, return_field=False)
    for _ in range(2):
        solve(scene, cfg_api, reference_frequency_hz=freq).path_gain.cpu()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    h2d = d2h = 0
    e0.record()
    for _ in range(steps):
        res = solve(scene, cfg_api, reference_frequency_hz=freq)
        host = res.path_gain.cpu()
        d2h += host.numel() * host.element_size()
        h2d += ep.tx_pos.numel() * 4 + ep.tx_power.numel() * 4 + ep.tx_pol.numel() * 4 + 4 * 5 * mats.eps_r.numel()
    e1.record()
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1)
    e2e_value = rays / (e2e_ms / 1000.0)
    # dominant per-cell kernel: its rays and the bytes it writes per cell (slot
    # values; for diffraction one visibility bit per kept edge)
    peaks = _peaks()
    hbm = float(peaks.get("hbm_gbs", HBM_FALLBACK))
    cells_n = ep.num_tx * ep.num_rx
    edges_kept = float(last_prof.get("edges") or 0)
    kinds = ("k_reflect", "k_diffract_vis", "k_diffract_utd", "k_los_trans")
    dominant = max(kinds, key=lambda k: kernel_ms.get(k, 0.0))
    cell_bytes = {"k_reflect": 12, "k_diffract_vis": edges_kept / 8, "k_diffract_utd": 16 + edges_kept / 8,
                  "k_los_trans": 12}[dominant]
    rays_of = {"k_reflect": "k_reflect", "k_diffract_vis": "k_diffract", "k_los_trans": "k_los_trans"}
    dom_rays = kernel_rays.get(rays_of.get(dominant, ""), 0)
    bytes_per_launch = dom_rays / steps * _bytes_per_ray(faces) + cells_n * cell_bytes
    launch_ms = kernel_ms.get(dominant, 0.0) / steps
    achieved = bytes_per_launch / (launch_ms / 1000.0) / 1e9 if launch_ms > 0 else 0.0
    fp64 = _fp64_plain(compiled, ep, mats, freq, bits, cfg, device, step_ms / steps)
    cpu = None if args.no_cpu_baseline else cpu_baseline(scene, freq, cfg, cores=1)
    return {
        "workload": WORKLOAD,
        "value": value,
        "unit": UNIT,
        "ms_per_step": step_ms / steps,
        "steps": steps,
        "triangles": faces,
        "rays_per_step": rays / steps,
        "per_cell_kernel_rays_per_step": main_rays / steps,
        "kernel_ms_per_step": {k: v / steps for k, v in kernel_ms.items()},
        "kernel_rays_per_step": {k: v / steps for k, v in kernel_rays.items()},
        "reflection_candidates_per_depth": last_prof.get("chains"),
        "diffraction_edges_after_prefilter": last_prof.get("edges"),
        "cells_per_step": cells_n,
        "l2": "flushed (256 MiB write) before every timed step",
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d // steps,
                "d2h_bytes_per_step": d2h // steps, "ms_per_step": e2e_ms / steps},
        "roofline": {
            "bound": "issue",
            "kernel": dominant,
            "issue_active": _profile_figure(CANYON_PROFILE, f"issue_active[{dominant}]"),
            "hbm_model": {"achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                          "algorithmic_bytes_per_launch": bytes_per_launch, "launch_ms": launch_ms,
                          "peak_source": "measured" if "hbm_gbs" in peaks else "fallback"},
            "traffic": _profile_figure(CANYON_PROFILE, f"traffic_bytes_per_launch[{dominant}]"),
            "l2_bytes_per_launch": _profile_figure(CANYON_PROFILE, f"l2_bytes_per_launch[{dominant}]"),
        },
        "cpu_baseline": cpu,
        "fp64_plain": fp64,
    }


def _fp64_plain(compiled, ep, mats, freq, bits, cfg, device, mixed_ms: float, steps: int = 11) -> dict:
    """The same solve with every stage in FP64 (the plain form the mixed path is compared with)."""
    import torch

    from witwin_channel_b200 import engine

    cells = engine.alloc_cells(1, ep.num_tx, ep.num_rx, device, fp64=True)

    def step():
        engine.run_solve(compiled, ep, mats, [freq], components=bits, max_depth=cfg.max_depth, coherent=True,
                         precision=1, cells=cells)

    for _ in range(3):
        step()
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    for a, b in ev:
        a.record()
        step()
        b.record()
    torch.cuda.synchronize()
    per = sorted(a.elapsed_time(b) for a, b in ev)
    ms = per[len(per) // 2]
    # median: FP64 solves here show occasional GPU-side stalls of 10-20 ms
    # that the mixed form's steps do not
    return {"ms_per_step": ms, "mean_ms_per_step": sum(per) / len(per), "statistic": "median of per-step events",
            "mixed_ms_per_step": mixed_ms, "mixed_speedup": ms / mixed_ms if mixed_ms else None, "steps": steps}


def _vjp_run(device, steps: int = 7) -> dict:
    """The gradient workload: forward + VJP of the log10 path-gain MSE on the
    urban canyon w.r.t. concrete (eps_r, sigma_e), frequency, Tx position and
    the vertices of 8 seeded boxes (the target map comes from eps_r x1.10 and
    the boxes displaced by N(0, 0.5 m))."""
    import torch

    from witwin_channel_b200 import Config, _native, solve
    from witwin_channel_b200.workloads import gradient_run, log_mse

    g = gradient_run(seed=1)
    cfg = Config(components=g["components"], max_depth=g["max_depth"], ad_mode="vjp")
    leaves = [g["leaves"]["eps_r"], g["leaves"]["sigma_e"], g["leaves"]["tx"], g["frequency"]] + g["leaves"]["vertices"]

    def step():
        for t in leaves:
            t.grad = None
        res = solve(g["scene"], cfg, reference_frequency_hz=g["frequency"])
        loss = log_mse(res.path_gain, g["target"])
        loss.backward()
        return loss, res

    step()
    step()
    torch.cuda.synchronize()
    # per step: the device-timeline span (events) and the host wall time to the
    # step's end (both include the host-side gaps between launches); medians
    step_ms, wall_ms = [], []
    for _ in range(steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0 = time.perf_counter()
        e0.record()
        loss, res = step()
        e1.record()
        torch.cuda.synchronize()
        wall_ms.append((time.perf_counter() - t0) * 1e3)
        step_ms.append(e0.elapsed_time(e1))
    _native.profile_enable(True)
    step()
    torch.cuda.synchronize()
    prof = _native.profile_read()
    _native.profile_enable(False)
    vg = torch.cat([v.grad.reshape(-1) for v in g["leaves"]["vertices"]])
    return {
        "workload": "urban canyon 64 boxes, 256x256 grid, 28 GHz, LoS + reflection depth 3 + UTD; loss = MSE of "
                    "log10 path gain vs a target from eps_r x1.10 and 8 boxes displaced N(0, 0.5 m); gradients for "
                    "concrete eps_r and sigma_e, frequency, Tx position and the 8 boxes' 64 vertices",
        "ms_per_step": float(sorted(step_ms)[len(step_ms) // 2]),
        "host_wall_ms_per_step": float(sorted(wall_ms)[len(wall_ms) // 2]),
        "diffraction_records_per_step": prof["acc_vjp_diffraction_records"],
        "diffraction_vjp_kernel_ms": prof["acc_vjp_diffraction_ms"],
        "steps_ms": [round(x, 3) for x in step_ms],
        "steps": steps,
        "paths": int(res.metadata["counts"]["path_count"]),
        "loss": float(loss),
        "grad": {"eps_r": float(g["leaves"]["eps_r"].grad), "sigma_e": float(g["leaves"]["sigma_e"].grad),
                 "frequency": float(g["frequency"].grad), "tx": [float(x) for x in g["leaves"]["tx"].grad],
                 "vertices_norm": float(vg.norm())},
    }


def _consumer_run(device, steps: int = 3) -> dict:
    """The canyon as a propagation-consumer request: its transmitter and the
    256 x 256 grid points as explicit endpoint batches, LoS + reflection depth
    3 + UTD, scalar transport through ``propagation.consumer.evaluate``; beside
    it the deterministic solve exporting the same rows as a path table.  Times
    are CUDA events around whole calls (host work between launches included)."""
    import torch

    from witwin_channel_b200.workloads import urban_canyon_scene

    scene, freq = urban_canyon_scene(seed=1)

    from witwin_channel_b200 import Config, solve
    from witwin_channel_b200.compiler import compile_scene
    from witwin_channel_b200.propagation import consumer

    try:
        tx = scene.transmitters[0]
        grid = scene.receivers[0]
        pts = grid.points().to(device).contiguous()
        R = int(pts.shape[0])
        sources = consumer.EndpointBatch(
            stable_ids=torch.zeros(1, dtype=torch.int64, device=device),
            positions_m=tx.position.detach().float().reshape(1, 3).to(device).contiguous(),
            polarizations=tx.polarization.detach().float().reshape(1, 3).to(device).contiguous(),
            powers_w=torch.tensor([float(tx.power_w)], dtype=torch.float32, device=device))
        sinks = consumer.EndpointBatch(
            stable_ids=torch.arange(R, dtype=torch.int64, device=device), positions_m=pts,
            polarizations=grid.polarization.detach().float().reshape(1, 3).expand(R, 3).to(device).contiguous())
        comps = frozenset({"los", "reflection", "diffraction"})
        request = consumer.PropagationRequest(sources=sources, sinks=sinks, reference_frequency_hz=freq,
                                              components=comps, max_depth=3, response="scalar_transport",
                                              topology_mode="discover", ad_mode="none")
        compiled = compile_scene(scene, device)
        cfg = Config(components=set(comps), max_depth=3, export_paths=True, return_field=False)

        def timed(fn):
            out = fn()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(steps):
                out = fn()
            e1.record()
            torch.cuda.synchronize()
            return out, e0.elapsed_time(e1) / steps

        ev, ev_ms = timed(lambda: consumer.evaluate(compiled, request))
        table, det_ms = timed(lambda: solve(scene, cfg, reference_frequency_hz=freq).paths)
        # fixed-topology replay of the LoS + reflection rows: at the discovery
        # endpoints, over 8 slots of sinks moved 0..0.35 m (one replay for the
        # block), and over 4 frequency columns; rediscovery beside it
        lr = frozenset({"los", "reflection"})
        req_lr = consumer.PropagationRequest(sources=sources, sinks=sinks, reference_frequency_hz=freq,
                                             components=lr, max_depth=3, response="scalar_transport",
                                             topology_mode="discover", ad_mode="none")
        found, rediscover_ms = timed(lambda: consumer.evaluate(compiled, req_lr))
        prepared = consumer.prepare_fixed_topology(found.paths.topology)

        def replay_request(src, snk, topology, slots=1, offsets=None):
            return consumer.FixedTopologyRequest(sources=src, sinks=snk, reference_frequency_hz=freq,
                                                 topology=topology, response="scalar_transport", ad_mode="none",
                                                 slot_count=slots, frequency_offsets_hz=offsets)

        replay, replay_ms = timed(lambda: consumer.reevaluate(compiled, replay_request(sources, sinks, prepared)))
        T = 8
        shift = torch.linspace(0.0, 0.35, T, device=device).view(T, 1, 1) * torch.tensor([1.0, 0.6, 0.0],
                                                                                        device=device)
        stacked_sinks = consumer.EndpointBatch(
            stable_ids=sinks.stable_ids.repeat(T), positions_m=(pts.unsqueeze(0) + shift).reshape(-1, 3).contiguous(),
            polarizations=sinks.polarizations.repeat(T, 1).contiguous())
        stacked_sources = consumer.EndpointBatch(
            stable_ids=sources.stable_ids.repeat(T), positions_m=sources.positions_m.repeat(T, 1).contiguous(),
            polarizations=sources.polarizations.repeat(T, 1).contiguous(), powers_w=sources.powers_w.repeat(T))
        replicated = consumer.replicate_over_slots(prepared, T, source_count=1, sink_count=R)
        slotted, slots_ms = timed(lambda: consumer.reevaluate(
            compiled, replay_request(stacked_sources, stacked_sinks, replicated, slots=T)))
        offsets = (0.0, 1.0e8, 2.0e8, 3.0e8)
        _wide, wide_ms = timed(lambda: consumer.reevaluate(
            compiled, replay_request(sources, sinks, prepared, offsets=offsets)))
        K = prepared.row_count
        return {
            "workload": "urban canyon as explicit batches: 1 source x 65,536 sinks, LoS + reflection depth 3 + UTD, "
                        "scalar transport",
            "evaluate_ms": ev_ms,
            "deterministic_export_ms": det_ms,
            "paths": ev.paths.path_count,
            "candidates": ev.diagnostics.candidate_count,
            "same_row_count_as_table": ev.paths.path_count == int(table.tx_id.shape[0]),
            "replay": {
                "workload": "the LoS + reflection (depth 3) rows of the canyon request, frozen and replayed",
                "rows": K,
                "rediscover_ms": rediscover_ms,
                "replay_ms": replay_ms,
                "replay_rows_per_s": K / (replay_ms * 1e-3),
                "replay_all_valid": bool(replay.row_valid.all()),
                "slots": T,
                "slot_block_ms": slots_ms,
                "slot_rows_per_s": T * K / (slots_ms * 1e-3),
                "slot_valid_fraction": float(slotted.row_valid.float().mean()),
                "wideband_columns": len(offsets) + 1,
                "wideband_ms": wide_ms,
            },
        }
    except Exception as exc:  # reported in the leg; the headline line stands
        return {"error": f"{type(exc).__name__}: {exc}"}


def _large_run(device, steps: int = 2) -> dict:
    """The large-city workload: 2048 boxes with subdivided roofs (~112k
    triangles), 25% with an interior two-layer glass sheet, 1 Tx, 1024^2 grid,
    28 GHz, LoS + reflection depth 5 + UTD + transmission, paths exported and
    converted to a CFR over 1024 subcarriers spanning 400 MHz."""
    import numpy as np
    import torch

    from witwin_channel_b200 import Config, _native, solve
    from witwin_channel_b200.channel import cfr
    from witwin_channel_b200.workloads import large_city_scene

    from witwin_channel_b200.compiler import compile_scene

    scene, freq = large_city_scene()
    cfg = Config(components={"los", "reflection", "diffraction", "transmission"}, max_depth=5, export_paths=True,
                 return_field=False)
    # scene compile (host binned-SAH BVH, groups, edges; uploads) and, after a
    # rigid move of one box, the in-place device refit of the same scene
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    compiled = compile_scene(scene, device)
    torch.cuda.synchronize()
    build_ms = (time.perf_counter() - t0) * 1e3
    freqs = (np.arange(1024) - 512) * 390.625e3
    R = int(scene.receivers[0].shape[0]) * int(scene.receivers[0].shape[1])
    _native.profile_enable(True)
    res = solve(scene, cfg, reference_frequency_hz=freq)
    torch.cuda.synchronize()
    e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    e[0].record()
    for _ in range(steps):
        res = solve(scene, cfg, reference_frequency_hz=freq)
    e[1].record()
    prof = _native.profile_read()
    h = cfr(res.paths, freqs, num_tx=1, num_rx=R)
    torch.cuda.synchronize()
    c0, c1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    c0.record()
    for _ in range(steps):
        del h  # the next call reuses this spectrum's cached block instead of allocating another 8.6 GB
        h = cfr(res.paths, freqs, num_tx=1, num_rx=R)
    c1.record()
    torch.cuda.synchronize()
    rays = prof["rays"] + prof["prep_rays"]
    cfr_ms = c0.elapsed_time(c1) / steps
    st = scene.structures[1]
    st.geometry.vertices = st.vertices.detach() + torch.tensor([0.25, -0.125, 0.0])
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    refitted = compile_scene(scene, device)
    torch.cuda.synchronize()
    refit_ms = (time.perf_counter() - t0) * 1e3
    # the device LBVH rebuild of the refitted scene, and one solve on it
    try:
        t0 = time.perf_counter()
        lbvh_depth = refitted.native.rebuild_bvh()
        lbvh_ms = (time.perf_counter() - t0) * 1e3
        res_l = solve(scene, cfg, reference_frequency_hz=freq)
        torch.cuda.synchronize()
        e[2].record()
        res_l = solve(scene, cfg, reference_frequency_hz=freq)
        e3 = torch.cuda.Event(enable_timing=True)
        e3.record()
        torch.cuda.synchronize()
        lbvh_solve_ms = e[2].elapsed_time(e3)
        lbvh_paths = int(res_l.metadata["counts"]["path_count"])
        del res_l
    except Exception as exc:  # reported in the leg; the rest of the leg stands
        lbvh_depth, lbvh_ms, lbvh_solve_ms, lbvh_paths = f"{type(exc).__name__}: {exc}", None, None, None
    out = {
        "workload": "2048 boxes (46x46 lots, roofs split 4x4 on even / 5x5 on odd boxes, ~134k triangles, 25% with "
                    "a 2-layer glass sheet), "
                    "1 Tx, 1024x1024 grid at 1 m, 28 GHz, LoS + reflection depth 5 + UTD + transmission; CFR "
                    "over 1024 subcarriers (390.625 kHz spacing)",
        "triangles": int(sum(int(st.faces.shape[0]) for st in scene.structures)),
        "build_ms": build_ms,
        "refit_ms": refit_ms,
        "refit_in_place": refitted is compiled,
        "lbvh_rebuild_ms": lbvh_ms,
        "lbvh_depth": lbvh_depth,
        "lbvh_solve_ms": lbvh_solve_ms,
        "lbvh_paths": lbvh_paths,
        "solve_ms": e[0].elapsed_time(e[1]) / steps,
        "kernel_ms": prof["kernel_ms"],
        "rays": rays,
        "rays_per_s_kernels": rays / ((prof["main_ms"] + prof["prep_ms"]) / 1000.0),
        "paths": int(res.metadata["counts"]["path_count"]),
        "cfr_ms": cfr_ms,
        "cfr_bytes": int(h.numel() * 8),
        "cfr_write_gbs": h.numel() * 8 / (cfr_ms / 1000.0) / 1e9,
    }
    del h, res
    torch.cuda.empty_cache()
    return out


def _batched_forward_graph(full, device, reps: int = 5) -> dict:
    """The headline workload's batched forward (radiomaps only) issued eagerly
    (``solve_batch``) and as a captured CUDA graph (``BatchGraph``, stream pool
    size picked by timing); best of ``reps`` each, inputs resident."""
    import torch

    from witwin_channel_b200 import Config
    from witwin_channel_b200.batch import BatchGraph, solve_batch
    from witwin_channel_b200.workloads import BATCH_FREQS

    try:
        cfg = Config(components={"los", "reflection", "diffraction"}, max_depth=3, return_field=False)

        def best(fn):
            fn()
            torch.cuda.synchronize()
            t = float("inf")
            for _ in range(reps):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                fn()
                e1.record()
                torch.cuda.synchronize()
                t = min(t, e0.elapsed_time(e1))
            return t

        eager_ms = best(lambda: solve_batch(full, cfg, BATCH_FREQS))
        graph = BatchGraph(full, cfg, BATCH_FREQS, streams="auto")
        graph_ms = best(graph.replay)
        graph.check()
        same = all(torch.equal(a["path_gain"], b["path_gain"])
                   for a, b in zip(graph.replay(), solve_batch(full, cfg, BATCH_FREQS)))
        return {"eager_ms": eager_ms, "graph_ms": graph_ms, "streams": graph.streams,
                "tuning_ms": graph.tuning, "graph_equals_eager": same,
                "statistic": f"best of {reps} after one untimed run"}
    except Exception as exc:  # reported in the leg; the headline line stands
        return {"error": f"{type(exc).__name__}: {exc}"}


def _batched_plain(full, device, reps: int = 2) -> dict:
    """The plain FP64 single-transmitter form of the headline step: per
    (scene, transmitter, frequency) one FP64 differentiable forward (record
    search and values in FP64) and its VJP of the same loss; best of ``reps``
    after one untimed run."""
    import torch

    from witwin_channel_b200 import Config, solve
    from witwin_channel_b200.batch import single_transmitter_scene
    from witwin_channel_b200.workloads import BATCH_FREQS

    comps = {"los", "reflection", "diffraction"}
    cfg_ad = Config(components=comps, max_depth=3, ad_mode="vjp", return_field=False)
    subs = [[single_transmitter_scene(sc, t) for t in range(len(sc.transmitters))] for sc in full]

    def plain():
        for per_scene in subs:
            for sub in per_scene:
                for f in BATCH_FREQS:
                    res = solve(sub, cfg_ad, reference_frequency_hz=f, precision="fp64")
                    (res.path_gain.double().sum() * 1e6).backward()

    plain()
    torch.cuda.synchronize()
    best = float("inf")
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        plain()
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    return {"ms_per_step": best, "jobs": sum(len(x) for x in subs) * len(BATCH_FREQS),
            "form": "one FP64 differentiable forward and its VJP per (scene, Tx, frequency)",
            "statistic": f"best of {reps} after one untimed run"}


# --------------------------------------------------------------------------
# CPU side (oracle): used for the cpu_baseline field and the reference arm
# --------------------------------------------------------------------------
_ORACLE: dict = {}


def _oracle_init(arrays, kw, face_group_id, discovered, edge_visible):
    _ORACLE.update(arrays=arrays, kw=kw, face_group_id=face_group_id, discovered=discovered,
                   edge_visible=edge_visible)


def _oracle_trace(task):
    """Discovery bounces for one transmitter along a subset of the Fibonacci directions."""
    from oracle import geom
    from oracle import solve as osolve

    tx, index = task
    dirs = geom.fibonacci_directions(osolve.DISCOVERY_RAYS)[index]
    geom.RAY_COUNTER[0] = 0
    t0 = time.perf_counter()
    chains = osolve.discover_directions(_ORACLE["arrays"], _ORACLE["face_group_id"], tx, dirs,
                                        max_depth=_ORACLE["kw"]["max_depth"])
    return chains, time.perf_counter() - t0, geom.RAY_COUNTER[0]


def _oracle_cells(cells):
    """The per-cell oracle (LoS, reflection candidates, UTD) on a few receiver cells."""
    from oracle import geom
    from oracle import solve as osolve

    arrays = _ORACLE["arrays"]
    sub = dict(arrays)
    sub["rx_pos"] = arrays["rx_pos"][cells]
    sub["rx_pol"] = arrays["rx_pol"][cells]
    geom.RAY_COUNTER[0] = 0
    t0 = time.perf_counter()
    osolve.solve(sub, discovered=_ORACLE["discovered"], edge_visible=_ORACLE["edge_visible"], **_ORACLE["kw"])
    return time.perf_counter() - t0, geom.RAY_COUNTER[0], len(cells)


class OracleBaseline:
    """The FP64 NumPy oracle timed on the host cores on a bounded sample of the workload.

    Set-up (untimed): the full per-transmitter chain discovery (262,144
    Fibonacci rays x depth), spread over every host core, so the sampled
    cells see the same reflection candidates as the full solve.  A timed
    sample: a strided subset of the discovery rays plus a few receiver cells,
    on ``cores`` processes; the rate is extrapolated to the full grid
    (all discovery rays once, every cell)."""

    def __init__(self, scene, freq, cfg):
        import multiprocessing as mp

        import numpy as np

        from oracle import solve as osolve

        self.np = np
        self.arrays = osolve.scene_arrays(scene, freq)
        self.kw = dict(components=set(cfg.components), max_depth=cfg.max_depth, coherent=cfg.coherent,
                       frequency=freq)
        self.R = self.arrays["rx_pos"].shape[0]
        self.T = self.arrays["tx_pos"].shape[0]
        self.face_group_id = osolve.discovery_groups(self.arrays, max_depth=cfg.max_depth)
        self.ctx = mp.get_context("spawn")
        self.host_cores = os.cpu_count() or 1
        t0 = time.perf_counter()
        self.discovered = None
        if self.face_group_id is not None:
            n = osolve.DISCOVERY_RAYS
            parts = [np.arange(i, n, self.host_cores * 4) for i in range(self.host_cores * 4)]
            with self.ctx.Pool(self.host_cores, initializer=_oracle_init,
                               initargs=(self.arrays, self.kw, self.face_group_id, None, None)) as pool:
                self.discovered = []
                for t in range(self.T):
                    res = pool.map(_oracle_trace, [(t, p) for p in parts])
                    chains = np.full((n, cfg.max_depth), -1, dtype=np.int64)
                    for p, r in zip(parts, res):
                        chains[p] = r[0]
                    self.discovered.append(chains)
        self.setup_s = time.perf_counter() - t0
        self.edge_visible = None
        self.edge_rays = 0
        self.edge_s = 0.0
        if "diffraction" in self.kw["components"]:
            from oracle import geom

            geom.RAY_COUNTER[0] = 0
            t1 = time.perf_counter()
            self.edge_visible = osolve.tx_edge_masks(self.arrays, freq)
            self.edge_s = time.perf_counter() - t1
            self.edge_rays = geom.RAY_COUNTER[0]
        self.pools: dict[int, object] = {}

    def _pool(self, cores):
        if cores not in self.pools:
            self.pools[cores] = self.ctx.Pool(cores, initializer=_oracle_init,
                                              initargs=(self.arrays, self.kw, self.face_group_id, self.discovered,
                                                        self.edge_visible))
        return self.pools[cores]

    def close(self):
        for p in self.pools.values():
            p.close()
            p.join()
        self.pools.clear()

    def sample(self, cores: int, *, disc_rays_per_core: int = 2048, cells_per_core: int = 8, seed: int = 0) -> dict:
        np = self.np
        from oracle import solve as osolve

        rng = np.random.default_rng(seed)
        pool = self._pool(cores)
        n = osolve.DISCOVERY_RAYS
        t_start = time.perf_counter()
        disc_time = disc_rays = disc_dirs = 0
        if self.face_group_id is not None:
            take = min(n, disc_rays_per_core * cores)
            picked = np.sort(rng.choice(n, size=take, replace=False))
            tasks = [(int(rng.integers(self.T)), c) for c in np.array_split(picked, cores) if len(c)]
            t0 = time.perf_counter()
            res = pool.map(_oracle_trace, tasks)
            disc_time = time.perf_counter() - t0
            disc_rays = sum(r[2] for r in res)
            disc_dirs = take
        cells = np.sort(rng.choice(self.R, size=min(self.R, cells_per_core * cores), replace=False))
        t0 = time.perf_counter()
        res = pool.map(_oracle_cells, [c for c in np.array_split(cells, cores) if len(c)])
        cell_time = time.perf_counter() - t0
        cell_rays = sum(r[1] for r in res)
        ncell = sum(r[2] for r in res)
        # per-transmitter edge prefilter (timed once, single process) + per-cell work
        full_rays = self.edge_rays + cell_rays / ncell * self.R * self.T
        full_time = self.edge_s + cell_time / ncell * self.R * self.T
        if disc_dirs:
            full_rays += disc_rays / disc_dirs * n * self.T
            full_time += disc_time / disc_dirs * n * self.T
        return {
            "value": full_rays / full_time,
            "unit": UNIT,
            "cores": cores,
            "kind": "port",
            "sample": f"FP64 NumPy oracle on {cores} process(es): {disc_dirs} of {n} discovery rays x depth "
                      f"({disc_rays} bounces, {disc_time:.1f} s) and {ncell} of {self.R} receiver cells "
                      f"({cell_rays} segment queries, {cell_time:.1f} s) plus the Tx edge prefilter "
                      f"({self.edge_rays} segments, {self.edge_s:.1f} s, 1 process), extrapolated to the full grid; "
                      f"chain set from a full untimed discovery ({self.setup_s:.1f} s on {self.host_cores} cores)",
            "seconds": time.perf_counter() - t_start,
        }


BATCHED_SAMPLE = (1, 0, 28.0e9)  # scene 1 (32 boxes, 96^2 grid), its first transmitter, 28 GHz


def _batched_sample_scene(full=None):
    from witwin_channel_b200 import Config
    from witwin_channel_b200.batch import single_transmitter_scene
    from witwin_channel_b200.workloads import batched_scenes

    full = full if full is not None else batched_scenes()
    s, t, f = BATCHED_SAMPLE
    return single_transmitter_scene(full[s], t), f, Config(components={"los", "reflection", "diffraction"},
                                                           max_depth=3)


def batched_cpu_baseline(full, *, cores: int = 1) -> dict:
    """The oracle on a bounded sample of the batched workload: one of its
    (scene, transmitter, frequency) jobs, a discovery-ray subset and a few
    receiver cells, extrapolated to that job's full grid."""
    scene, freq, cfg = _batched_sample_scene(full)
    out = cpu_baseline(scene, freq, cfg, cores=cores)
    s, t, f = BATCHED_SAMPLE
    out["sample"] = f"job (scene {s}, Tx {t}, {f / 1e9:g} GHz) of the batched workload: " + out["sample"]
    return out


def cpu_baseline(scene, freq, cfg, *, cores: int = 1) -> dict:
    base = OracleBaseline(scene, freq, cfg)
    try:
        return base.sample(cores, disc_rays_per_core=4096, cells_per_core=8)
    finally:
        base.close()


def run_reference(args) -> None:
    """The oracle port of the reference's CPU algorithm on all host cores (the
    reference's own CUDA build needs sources it does not ship).  Rank 0 only."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    scene, freq, cfg = _batched_sample_scene()
    base = OracleBaseline(scene, freq, cfg)
    cores = base.host_cores
    samples = []
    times = []
    try:
        for i in range(args.warmup + args.steps):
            t0 = time.perf_counter()
            r = base.sample(cores, seed=i)
            if i >= args.warmup:
                samples.append(r)
                times.append(time.perf_counter() - t0)
    finally:
        base.close()
    value = sorted(s["value"] for s in samples)[len(samples) // 2]
    line = {
        "impl": "reference",
        "metric": METRIC,
        "value": value,
        "unit": UNIT,
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": 1000.0 * sum(times) / max(len(times), 1),
        "higher_is_better": True,
        "scaling": "strong",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (seeded scenes)",
        "config": {"workload": BATCHED_WORKLOAD,
                   "implementation": "FP64 NumPy oracle (a port of the reference algorithm) on host cores; "
                                     "the reference's CUDA build needs external ray-tracing sources it does not ship",
                   "step": "one bounded sample of one (scene, Tx, frequency) job of the workload (scene %d, Tx %d, "
                           "%g GHz: discovery-ray subset + receiver-cell subset) extrapolated to that job's grid"
                           % (BATCHED_SAMPLE[0], BATCHED_SAMPLE[1], BATCHED_SAMPLE[2] / 1e9)},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": samples[-1]["sample"]},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="native", choices=["native", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-vjp", action="store_true")
    ap.add_argument("--no-batched", action="store_true")
    ap.add_argument("--no-large", action="store_true")
    ap.add_argument("--no-consumer", action="store_true")
    ap.add_argument("--no-canyon", action="store_true")
    ap.add_argument("--only-leg", choices=["canyon", "vjp", "consumer", "large"], default=None,
                    help="run one side leg alone (profiling runs); no headline line")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "native":
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    elif args.only_leg:
        run_leg(args)
    else:
        run_native(args)


if __name__ == "__main__":
    main()
