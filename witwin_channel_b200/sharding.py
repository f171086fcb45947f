"""Multi-GPU sharding of the radiomap solve: one process per GPU, no exchange.

The units of the deterministic solve (transmitter, frequency, receiver tile)
are independent: each rank owns a disjoint slice of them, solves it with no
collective on the data path, and the per-rank outputs are joined by
concatenation.  The only collectives are the step-time reduction (max over
ranks) and, when a caller wants the whole map on every rank, one all-gather
of the outputs at the end.  A gradient step over a sharded job (a loss that
is a sum over the ranks' cells) needs one exchange: the sum of the ranks'
dense gradients, one all-reduce of one FP64 buffer.  Works with any
``torch.distributed`` backend (NCCL on GPUs, gloo on CPU tensors).
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


def shard_grid(grid, rank: int, world: int):
    """Rows ``[start, stop)`` of receiver grid ``grid`` (``shard_range`` over
    its first axis) as a grid of their own: same axes, spacing and
    polarisation, origin moved to row ``start`` (its points equal the full
    grid's rows up to the FP32 rounding of the moved origin).  Returns
    ``(sub_grid, (start, stop))``."""
    from .scene import make_receiver_grid

    start, stop = shard_range(int(grid.shape[0]), rank, world)
    origin = grid.origin.detach().double() + grid.x_axis.detach().double() * (start * float(grid.spacing[0]))
    sub = make_receiver_grid(origin=origin.float(), x_axis=grid.x_axis, y_axis=grid.y_axis,
                             shape=(stop - start, int(grid.shape[1])), spacing=grid.spacing,
                             polarization=grid.polarization)
    return sub, (start, stop)


def allreduce_gradients(tensors, group=None) -> None:
    """Sum the ``.grad`` of every tensor in ``tensors`` over the ranks, in
    place: the dense gradients (vertices, materials, frequency, transmitter
    positions...) are packed in list order into one FP64 buffer, reduced by
    one ``all_reduce(SUM)`` and unpacked; a missing gradient counts as zero.
    Every rank must pass the same tensors in the same order.  With NCCL the
    buffer lives on the current CUDA device."""
    if not (dist.is_available() and dist.is_initialized()):
        return
    if not tensors:
        return
    grads = [t.grad if t.grad is not None else torch.zeros_like(t) for t in tensors]
    backend = dist.get_backend(group)
    device = torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" else torch.device("cpu")
    flat = torch.cat([g.detach().reshape(-1).to(device=device, dtype=torch.float64) for g in grads])
    dist.all_reduce(flat, op=dist.ReduceOp.SUM, group=group)
    offset = 0
    for t, g in zip(tensors, grads):
        n = g.numel()
        t.grad = flat[offset:offset + n].reshape(t.shape).to(device=t.device, dtype=t.dtype)
        offset += n
