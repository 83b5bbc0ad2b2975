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
gradient pool, and the ranks sum those pools.  A step's pixels touch only a
small part of the pool (at most one voxel or DXT1 block per pixel), so
`sparse_allreduce_` exchanges the touched entries alone: every rank gathers
the (index, value) pairs of every rank and adds them in rank order, which
moves a few tens of MB where the dense sum (`allreduce_sum_`) moves the whole
pool, and leaves every rank with bit-identical sums.
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


def touched_entries(records, kind: int):
    """Gradient-pool entries a step's hit records can write: for VX_DIFF_VOXEL_RGB (kind 0) the
    3 channels of every hit voxel (brick * 512 + voxel), for VX_DIFF_DXT1_ENDPOINTS (kind 1) the
    6 endpoint channels of every hit block (brick * 32 + voxel / 16); sorted, unique.
    records: (n, 4) int32 tensor of vx_hit records (any device)."""
    import torch
    r = records.reshape(-1, 4)
    flags = (r[:, 3] >> 16) & 0xFF
    hit = (flags & 1).bool()
    brick = r[:, 1][hit].to(torch.int64) & 0xFFFFFFFF
    voxel = r[:, 3][hit].to(torch.int64) & 0xFFFF
    key = brick * 512 + voxel if kind == 0 else brick * 32 + (voxel >> 4)
    per = 3 if kind == 0 else 6
    key = torch.unique(key)
    return (key[:, None] * per + torch.arange(per, device=key.device)[None, :]).reshape(-1)


def sparse_allreduce_(grad, entries, group=None):
    """Sum a gradient pool over ranks when each rank's pool is zero outside its `entries` (sorted
    unique int64 indices): all-gather every rank's (index, value) pairs, then every rank adds the
    values of all ranks in rank order (a dense [ranks, touched] table summed along ranks, so the
    result is the same bits on every rank).  Identity without a process group; returns grad."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return grad
    world = dist.get_world_size(group)
    vals = grad[entries]
    count = torch.tensor([entries.numel()], dtype=torch.int64, device=grad.device)
    counts = [torch.zeros_like(count) for _ in range(world)]
    dist.all_gather(counts, count, group=group)
    m = int(max(int(c.item()) for c in counts))
    pad_i = torch.full((m,), -1, dtype=torch.int64, device=grad.device)
    pad_v = torch.zeros((m,), dtype=grad.dtype, device=grad.device)
    pad_i[:entries.numel()] = entries
    pad_v[:entries.numel()] = vals
    all_i = [torch.empty_like(pad_i) for _ in range(world)]
    all_v = [torch.empty_like(pad_v) for _ in range(world)]
    dist.all_gather(all_i, pad_i, group=group)
    dist.all_gather(all_v, pad_v, group=group)
    idx = torch.cat([a[:int(c.item())] for a, c in zip(all_i, counts)])
    uniq, inv = torch.unique(idx, return_inverse=True)
    table = torch.zeros((world, uniq.numel()), dtype=grad.dtype, device=grad.device)
    off = 0
    for r, (v, c) in enumerate(zip(all_v, counts)):
        n = int(c.item())
        table[r, inv[off:off + n]] = v[:n]
        off += n
    total = table[0].clone()
    for r in range(1, world):  # fixed rank order: the same bits on every rank
        total += table[r]
    grad[uniq] = total
    return grad
