"""Sharding one ff_sieve job over several GPUs (one process per GPU).

The odd sums of a job are independent, so a job splits into contiguous shards, one per
rank, with no exchange while the sums are searched: each rank sieves the map its own shard
needs and searches it. The only collective is the gather of the packed records to rank 0,
which then emits ff_seg's text in the reference's order from the whole record array
(ffb_emit). The per-sum search cost grows about linearly with the sum (the cumulative cost of
sums up to s grows as s^2), so shard boundaries are placed at equal shares of s^2.
"""
import math


def odd_sums(lo, hi):
    return (hi - lo) // 2 + 1 if hi >= lo else 0


def shard_bounds(lo, hi, world, rank):
    """Contiguous shard [a, b] (odd sums) of the odd sums lo..hi for `rank` of `world`,
    balanced by search cost. Shards are disjoint, ascending with the rank, cover lo..hi, and
    may be empty (a > b) when there are fewer sums than ranks."""
    if world == 1:
        return lo, hi

    def cut(q):  # smallest odd sum at or above the point where the cost share reaches q
        s = int(math.sqrt(lo * lo + q * (hi * hi - lo * lo)))
        s = max(lo, min(hi + 2, s))
        return s if s & 1 else s + 1
    a = lo if rank == 0 else cut(rank / world)
    b = hi if rank == world - 1 else cut((rank + 1) / world) - 2
    return a, b


def gather_records(dist, local, lo, hi, world, rank):
    """All ranks' packed records (a 1-D int64 tensor of the rank's shard) to rank 0 as one
    tensor over lo..hi (None on the other ranks). Every rank takes the same collective
    steps: one all_gather of equal-length padded buffers."""
    import torch
    sizes = [odd_sums(*shard_bounds(lo, hi, world, r)) for r in range(world)]
    width = max(max(sizes), 1)
    buf = torch.zeros(width, dtype=torch.int64, device=local.device)
    n = sizes[rank]
    if n:
        buf[:n] = local[:n]
    parts = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(parts, buf)
    if rank != 0:
        return None
    return torch.cat([p[:sizes[r]] for r, p in enumerate(parts)])
