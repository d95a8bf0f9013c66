"""Replicas over GPUs: arenas are independent, so N GPUs run N independent batches and exchange nothing on the data
path.  The only cross-rank steps are the host-side ones here: every rank adopts rank 0's tuned configuration, timings
are taken as the max over ranks, and (for a fixed total) the arena range of each rank is a run of whole AoSoA-32
blocks.  Works with any torch.distributed backend (nccl on GPUs, gloo on CPUs)."""
from __future__ import annotations

LANES = 32


def shard(total: int, rank: int, world: int) -> tuple[int, int]:
    """[first, first + count) of `total` arenas for `rank`: whole blocks of 32 arenas, the remainder on the last ranks."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} of {world}")
    blocks = (total + LANES - 1) // LANES
    base, extra = divmod(blocks, world)
    b0 = rank * base + max(0, rank - (world - extra))
    nb = base + (1 if rank >= world - extra else 0)
    first = b0 * LANES
    return first, max(0, min(total, (b0 + nb) * LANES) - first)


def broadcast_config(config: dict, dist=None, device=None) -> dict:
    """Rank 0's configuration on every rank."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return config
    obj = [config]
    dist.broadcast_object_list(obj, src=0, device=device)
    return obj[0]


def max_over_ranks(value: float, dist=None, device=None) -> float:
    """The max of `value` over ranks (timings: the job is as slow as its slowest replica)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return value
    import torch

    t = torch.tensor([float(value)], dtype=torch.float32, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
