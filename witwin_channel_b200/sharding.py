"""Multi-GPU sharding of the radiomap solve: one process per GPU, no exchange.

The units of the deterministic solve (transmitter, frequency, receiver tile)
are independent: each rank owns a disjoint slice of them, solves it with no
collective on the data path, and the per-rank outputs are joined by
concatenation.  The only collectives are the step-time reduction (max over
ranks) and, when a caller wants the whole map on every rank, one all-gather
of the outputs at the end.  Works with any ``torch.distributed`` backend
(NCCL on GPUs, gloo on CPU tensors).
"""

from __future__ import annotations

import torch
import torch.distributed as dist


def shard_range(count: int, rank: int, world: int) -> tuple[int, int]:
    """Balanced contiguous ``[start, stop)`` slice of ``count`` units for ``rank``."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank must lie in [0, world)")
    if count < 0:
        raise ValueError("count must be non-negative")
    base, extra = divmod(count, world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def reduce_step_time(step_ms: float, units: float, device: torch.device | None = None,
                     group=None) -> tuple[float, float]:
    """Job step time (max over ranks) and the units all ranks processed (sum)."""
    if not (dist.is_available() and dist.is_initialized()):
        return float(step_ms), float(units)
    t = torch.tensor([float(step_ms)], dtype=torch.float64, device=device)
    u = torch.tensor([float(units)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    dist.all_reduce(u, op=dist.ReduceOp.SUM, group=group)
    return float(t[0]), float(u[0])


def gather_concat(local: torch.Tensor, group=None) -> torch.Tensor:
    """Concatenate every rank's ``local`` along dim 0 in rank order.  Ranks may
    hold different leading sizes (uneven shards); trailing dims must agree."""
    if not (dist.is_available() and dist.is_initialized()):
        return local
    world = dist.get_world_size(group)
    n = torch.tensor([local.shape[0]], dtype=torch.int64, device=local.device)
    sizes = [torch.zeros_like(n) for _ in range(world)]
    dist.all_gather(sizes, n, group=group)
    sizes = [int(s.item()) for s in sizes]
    cap = max(sizes) if sizes else 0
    padded = local.new_zeros((cap,) + tuple(local.shape[1:]))
    padded[: local.shape[0]] = local
    parts = [torch.empty_like(padded) for _ in range(world)]
    dist.all_gather(parts, padded.contiguous(), group=group)
    return torch.cat([p[:s] for p, s in zip(parts, sizes)], dim=0)
