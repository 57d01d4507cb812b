"""Replica sharding across ranks (one process per GPU).  The reconstruction path has no
exchange step: independent scans, bootstrap replicates and dynamic frames are split
across ranks, and only the timing (max over ranks) and final statistics are reduced."""
from __future__ import annotations


def replicate_range(nrep: int, rank: int, world: int) -> tuple[int, int]:
    """(first, count) of the replicates rank `rank` owns out of `nrep` (contiguous blocks,
    the first `nrep % world` ranks take one extra)."""
    if world <= 0 or not (0 <= rank < world):
        raise ValueError('bad rank/world')
    base, extra = divmod(nrep, world)
    first = rank * base + min(rank, extra)
    return first, base + (1 if rank < extra else 0)


def max_over_ranks(value: float, device=None) -> float:
    """Maximum of a scalar over all ranks of the default process group (identity if the
    group is not initialised).  Works with NCCL (CUDA device) and gloo (CPU)."""
    import torch
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(t):
    """In-place sum of a tensor over ranks (final mean/std accumulators of replicates)."""
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(t)
    return t


def mean_std_over_ranks(local, group=None):
    """Voxel-wise mean and standard deviation (ddof 1) of the images of all ranks: `local`
    [n_local, ...] holds this rank's replicates (n_local may differ between ranks, and may
    be 0).  Two all-reduces in float64 -- the sum, then the sum of squared deviations from
    the global mean (the centred form, which keeps its precision when the spread is small
    against the mean).  Returns (mean, std) as float32 tensors on `local`'s device; with
    no process group, the statistics of `local` itself."""
    import torch
    import torch.distributed as dist
    x = local.double()
    dist_on = dist.is_available() and dist.is_initialized() and dist.get_world_size(group) > 1
    n = torch.tensor([float(x.shape[0])], dtype=torch.float64, device=x.device)
    s1 = x.sum(0)
    if dist_on:
        dist.all_reduce(n, group=group)
        dist.all_reduce(s1, group=group)
    ntot = float(n.item())
    if ntot < 1:
        raise ValueError('no replicates on any rank')
    mean = s1 / ntot
    s2 = ((x - mean) ** 2).sum(0)
    if dist_on:
        dist.all_reduce(s2, group=group)
    std = (s2 / (ntot - 1)).sqrt() if ntot > 1 else torch.zeros_like(mean)
    return mean.float(), std.float()
