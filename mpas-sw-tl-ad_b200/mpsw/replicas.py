"""Replica parallelism over GPUs: one process per GPU, each with the whole mesh and its own
trajectory, sharing out independent members (perturbations or cost-function gradients).

Members never interact, so the data path has no collective: a rank integrates its members
alone, and the only communication is at the end (the slowest rank's time, and gathering the
members' results where one rank needs all of them).  The reference is serial and has no
parallel decomposition; this module is new.  Works with any torch.distributed backend (NCCL on
GPUs, gloo on CPU for tests); without an initialised process group it is the identity.
"""
from __future__ import annotations

import torch


def _dist():
    import torch.distributed as dist
    return dist if dist.is_available() and dist.is_initialized() else None


def rank_world() -> tuple[int, int]:
    d = _dist()
    return (d.get_rank(), d.get_world_size()) if d else (0, 1)


def shard(total: int, rank: int, world: int) -> tuple[int, int]:
    """Members [start, start + count) of `total` that `rank` of `world` integrates: contiguous
    blocks, sizes differing by at most one, lower ranks taking the extra members."""
    if total < 0 or world < 1 or not 0 <= rank < world:
        raise ValueError('bad shard request: total=%d rank=%d world=%d' % (total, rank, world))
    base, extra = divmod(total, world)
    start = rank * base + min(rank, extra)
    return start, base + (1 if rank < extra else 0)


def member_seed(base: int, rank: int) -> int:
    """Seed of a rank's synthetic members, distinct across ranks."""
    return base + 1000 * rank


def max_over_ranks(value: float, device=None) -> float:
    """The largest `value` over all ranks (the job's time is its slowest rank's time)."""
    d = _dist()
    if d is None:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    d.all_reduce(t, op=d.ReduceOp.MAX)
    return float(t.item())


def gather_members(local: torch.Tensor, total: int) -> torch.Tensor:
    """All ranks' members side by side: `local` is this rank's [n, count] block of the shard
    layout of `total` members; every rank gets the [n, total] array."""
    d = _dist()
    if d is None:
        if local.shape[1] != total:
            raise ValueError('single process holds %d of %d members' % (local.shape[1], total))
        return local
    rank, world = d.get_rank(), d.get_world_size()
    start, count = shard(total, rank, world)
    if local.shape[1] != count:
        raise ValueError('rank %d holds %d members, its shard has %d' % (rank, local.shape[1], count))
    width = shard(total, 0, world)[1]  # the largest shard
    pad = torch.zeros(local.shape[0], width, dtype=local.dtype, device=local.device)
    pad[:, :count] = local
    parts = [torch.empty_like(pad) for _ in range(world)]
    d.all_gather(parts, pad.contiguous())
    return torch.cat([parts[r][:, :shard(total, r, world)[1]] for r in range(world)], dim=1)
