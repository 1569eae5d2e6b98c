"""One process per GPU: how ranks split the work and combine their results.

Paths, pixels, frames and views are independent, so rendering shards with no
collective on the data path: each rank renders its own frames (own sample
streams) or its own share of the views.  The two exchanges are
  * timing: the job's time is the slowest rank's, its vertex count the sum;
  * differentiable rendering: the brick-sample and albedo gradients of each
    rank's views are summed over the ranks (one all-reduce each), as the
    gradient of a loss summed over all views.
Every function works with any torch.distributed backend (NCCL for CUDA tensors,
gloo for CPU tensors) and does nothing when the job has one rank.
"""
from __future__ import annotations


def world() -> tuple[int, int]:
    """(rank, world size) of the initialised process group, else (0, 1)."""
    import torch.distributed as dist

    if dist.is_available() and dist.is_initialized():
        return dist.get_rank(), dist.get_world_size()
    return 0, 1


def frame_seed(base: int, rank: int) -> int:
    """Seed of a rank's frame: distinct per rank, so ranks draw independent paths."""
    return int(base) + int(rank)


def my_views(views: list, rank: int, size: int) -> list:
    """This rank's share of the views (round robin: view i goes to rank i mod size)."""
    return list(views[rank::size])


def slowest_and_total(seconds: float, vertices: float, device="cpu") -> tuple[float, float]:
    """(max over ranks of seconds, sum over ranks of vertices)."""
    import torch
    import torch.distributed as dist

    rank, size = world()
    if size == 1:
        return float(seconds), float(vertices)
    t = torch.tensor([float(seconds)], dtype=torch.float64, device=device)
    v = torch.tensor([float(vertices)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.all_reduce(v, op=dist.ReduceOp.SUM)
    return float(t.item()), float(v.item())


def slowest(seconds: float, device="cpu") -> float:
    """Max over ranks of seconds."""
    import torch
    import torch.distributed as dist

    rank, size = world()
    if size == 1:
        return float(seconds)
    t = torch.tensor([float(seconds)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_gradients(*tensors) -> None:
    """Sums each gradient tensor over the ranks in place (the brick-sample and
    albedo gradients of views rendered on different ranks); None entries are
    skipped."""
    import torch.distributed as dist

    rank, size = world()
    if size == 1:
        return
    for t in tensors:
        if t is not None:
            dist.all_reduce(t, op=dist.ReduceOp.SUM)
