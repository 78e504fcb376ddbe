"""One process per GPU, independent work per rank ("replicas").

The single-level step has no exchange step on this path (the reference's
halo exchange and dt all-reduce exist only because it splits one level over
MPI ranks; here a level lives on one GPU). Multi-GPU runs therefore shard
independent work: ensemble members / boxes are dealt out to ranks, each rank
advances its share with no data-path collective, and only the timing and the
reported totals are combined (max of the device times, sum of the work).
"""
from __future__ import annotations

import datetime
import os
from typing import Sequence, TypeVar

T = TypeVar("T")


def world() -> tuple[int, int, int]:
    """(world_size, rank, local_rank) from the torchrun environment."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend: str = "nccl", timeout_s: float = 120.0) -> tuple[int, int, int]:
    """Join the process group when WORLD_SIZE > 1 (short timeout: a rank that
    never arrives ends the others' next collective with an error)."""
    ws, rank, local = world()
    if ws > 1:
        import torch.distributed as dist
        if not dist.is_initialized():
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return ws, rank, local


def shard(items: Sequence[T], rank: int, world_size: int) -> list[T]:
    """Rank `rank`'s share of `items`: a contiguous block, sizes differing by at most one."""
    n = len(items)
    base, extra = divmod(n, world_size)
    lo = rank * base + min(rank, extra)
    hi = lo + base + (1 if rank < extra else 0)
    return list(items[lo:hi])


def shard_by_cells(sizes: Sequence[int], world_size: int) -> list[list[int]]:
    """Deal item indices to ranks so that the cell counts balance (largest
    first onto the least-loaded rank; deterministic)."""
    order = sorted(range(len(sizes)), key=lambda k: (-sizes[k], k))
    load = [0] * world_size
    out: list[list[int]] = [[] for _ in range(world_size)]
    for k in order:
        r = min(range(world_size), key=lambda q: (load[q], q))
        out[r].append(k)
        load[r] += sizes[k]
    return [sorted(o) for o in out]


def _reduce(v: float, op: str, device) -> float:
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(v)
    t = torch.tensor([float(v)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return float(t.item())


def max_over_ranks(v: float, device="cpu") -> float:
    return _reduce(v, "max", device)


def sum_over_ranks(v: float, device="cpu") -> float:
    return _reduce(v, "sum", device)


def barrier():
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.barrier()


def finish():
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        dist.barrier()
        dist.destroy_process_group()
