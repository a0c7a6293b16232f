"""Sharding one ff_sieve job over several GPUs (one process per GPU).

The prime map is split into equal byte slabs, one per rank (the reference likewise hands
the map's slabs to its devices, source/pull_scheduler.cpp:149-202): each rank sieves its
slab into its place in a full-size map buffer and an all-gather over NVLink fills in the
other ranks' slabs, so every rank holds the whole map after sieving 1/N of it. The odd sums
are independent, so they split into contiguous shards, one per rank, searched with no
exchange; the packed records are gathered to rank 0, which emits ff_seg's text in the
reference's order from the whole record array (ffb_emit). The per-sum search cost grows
about linearly with the sum (the cumulative cost of sums up to s grows as s^2), so shard
boundaries are placed at equal shares of s^2.
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


def map_slab(mpv, world, rank):
    """Rank's slab of the prime map for values 0..mpv: (seg_lo, seg_hi, slab_bytes). Every
    slab is slab_bytes long (a multiple of 256 bytes, so each starts 16-byte aligned at a
    value that is a multiple of 4096) and rank r's starts at byte r * slab_bytes of a buffer
    of world * slab_bytes bytes; the values [seg_lo, seg_hi) are sieved into it (seg_hi <=
    seg_lo for a rank past the end of the map: nothing to sieve)."""
    map_bytes = (mpv + 1 + 15) >> 4
    slab = -(-map_bytes // world)
    slab = -(-slab // 256) * 256
    lo = min(rank * slab * 16, mpv + 1)
    hi = min((rank + 1) * slab * 16, mpv + 1)
    return lo, hi, slab


def gather_map(dist, full, slab_bytes):
    """In-place all-gather of the ranks' map slabs: `full` (uint8, world * slab_bytes) holds
    this rank's slab at its place; afterwards it holds every rank's."""
    world = dist.get_world_size()
    rank = dist.get_rank()
    mine = full[rank * slab_bytes:(rank + 1) * slab_bytes]
    dist.all_gather_into_tensor(full[:world * slab_bytes], mine)


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
