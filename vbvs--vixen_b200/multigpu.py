"""Multi-GPU layout of the ray-casting path: replicas only.

Rays are independent and scenes read-only, so N GPUs run N replicas: every
rank holds its own copy of the scene and casts its own rays; nothing crosses
between GPUs in the data path.  Two ways to give ranks their rays:
  - weak scaling (the benchmark): rank r renders its own camera, seeded by
    `rank_seed(base, r)`, so per-GPU work stays fixed as N grows;
  - strong scaling: the rays of one frame are split into contiguous,
    near-equal ranges (`ray_range`), and the hit records concatenate back in
    rank order.
The only collective of the casts is the timing reduction: the max over ranks
of each rank's device-measured time (`max_over_ranks`).  The adjoint has one
real exchange when a step's views are split across ranks (`view_range`): each
rank accumulates the gradient of its views into its own copy of the attribute
gradient pool, and one sum all-reduce (`allreduce_sum_`, NCCL over NVLink on
GPUs) leaves the gradient of all views on every rank.
"""
from __future__ import annotations


def rank_seed(base: int, rank: int) -> int:
    """Seed of rank `rank`'s camera (rank 0 keeps the base seed)."""
    return base + 7919 * rank


def ray_range(n: int, rank: int, world: int) -> tuple[int, int]:
    """Contiguous [begin, end) share of n rays for `rank` of `world`; sizes differ by at most one."""
    if world < 1 or not (0 <= rank < world):
        raise ValueError("rank must be in [0, world)")
    q, r = divmod(n, world)
    begin = rank * q + min(rank, r)
    return begin, begin + q + (1 if rank < r else 0)


def max_over_ranks(values, group=None):
    """Elementwise max over ranks of a list of floats (identity without a process group)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return [float(v) for v in values]
    dev = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return [float(v) for v in t.cpu()]


def aggregate_throughput(units_per_rank: int, world: int, max_time_s: float) -> float:
    """Whole-job throughput: the units all ranks processed over the slowest rank's time."""
    return units_per_rank * world / max_time_s


def view_range(views: int, rank: int, world: int) -> tuple[int, int]:
    """Contiguous [begin, end) share of a step's views for `rank` of `world`."""
    return ray_range(views, rank, world)


def allreduce_sum_(tensor, group=None):
    """Sum `tensor` over ranks in place (identity without a process group); returns it."""
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        dist.all_reduce(tensor, op=dist.ReduceOp.SUM, group=group)
    return tensor
