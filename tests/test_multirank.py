"""The multi-GPU path on CPU: the sums of one job sharded over 2 and 3 ranks (gloo, one
process per rank), each rank's records computed for its shard alone, gathered to rank 0 with
the same collective the GPU run uses, and the text emitted from the gathered records with
ffb_emit. The oracle stands in for the device search here (no GPU on this path); the text
must equal ff_seg's."""
import datetime
import hashlib
import os
import re
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "ff-gpu_b200")
ORACLE = os.path.join(ROOT, "oracle")
NORM = re.compile(rb"(Prime|Freudenthal) time: [0-9]+")


def norm(b):
    return NORM.sub(rb"\1 time: N", b)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, args, out_path):
    for p in (PKG, ORACLE):
        if p not in sys.path:
            sys.path.insert(0, p)
    import numpy as np
    import torch
    import torch.distributed as dist
    import ffb200 as ffb
    import ffo
    from shard import gather_records, odd_sums, shard_bounds
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    try:
        g, _ = ffb.geometry(*args)
        sched = ffb.schedule(g.sumStart, g.sumLimit, g.maxPrimeMapValue)
        firsts = [f | 1 for f, l in sched if (f | 1) <= l]
        lasts = [l - (0 if l & 1 else 1) for f, l in sched if (f | 1) <= l]
        lo, hi = min(firsts), max(lasts)
        a, b = shard_bounds(lo, hi, world, rank)
        local = torch.zeros(max(odd_sums(a, b), 1), dtype=torch.int64)
        if a <= b:
            with ffo.Context(b, map_bound=(1 << 32) - 1) as c:
                rec, _ = c.eval_range(a, b)
                out = np.zeros(rec.size, dtype=np.uint64)
                for i in np.nonzero(rec)[0]:
                    low, high = int(rec[i]) >> 32, int(rec[i]) & 0xFFFFFFFF
                    v = (low | (c.is_prime(low) << 31)) << 32 | high | (c.is_prime(high) << 31)
                    out[i] = v
            local[:out.size] = torch.from_numpy(out.view(np.int64))
        full = gather_records(dist, local, lo, hi, world, rank)
        if rank == 0:
            assert full.numel() == odd_sums(lo, hi)
            with open(out_path, "wb") as f:
                f.write(ffb.emit(args, full.numpy(), lo))
    finally:
        dist.destroy_process_group()


def _run(world, args, tmp_path):
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    port = _free_port()
    out = str(tmp_path / f"out_{world}.txt")
    procs = [ctx.Process(target=_worker, args=(r, world, port, args, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
    codes = [p.exitcode for p in procs]
    for p in procs:
        if p.is_alive():
            p.kill()
    assert codes == [0] * world, codes
    with open(out, "rb") as f:
        return f.read()


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_job_equals_ff_seg(world, tmp_path, golden, ffb):
    text = _run(world, (5, 65536), tmp_path)
    assert norm(text) == norm(golden["leg65536"])


def test_sharded_odd_range(tmp_path, oracle, ffb):
    args = (1000001, 1002500)
    text = _run(2, args, tmp_path)
    assert norm(text) == norm(oracle.run(*args, map_bound=(1 << 32) - 1))


def _slab_worker(rank, world, port, mpv, out_path):
    for p in (PKG, ORACLE):
        if p not in sys.path:
            sys.path.insert(0, p)
    import math
    import numpy as np
    import torch
    import torch.distributed as dist
    import ffo
    from shard import gather_map, map_slab
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    try:
        lo, hi, slab = map_slab(mpv, world, rank)
        full = torch.full((world * slab,), 0xA5, dtype=torch.uint8)
        if hi > lo:
            # the rank's slab as the device's slab sieve writes it (the reference slab
            # contract, source/sieve_slab_kernel.h:40-107, with the map's list)
            primes = ffo.odd_primes(math.isqrt(mpv))
            part = ffo.slab_relative(lo, hi, primes)[:(hi - lo + 15) >> 4]
            full[rank * slab:rank * slab + part.size] = torch.from_numpy(part)
        gather_map(dist, full, slab)
        if rank == 0:
            np.save(out_path, full.numpy())
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,mpv", [(2, 10_000_015), (3, 10_000_015), (3, 4_015)])
def test_map_slabs_all_gathered(world, mpv, tmp_path, oracle):
    """Each rank sieves its slab of the map (map_slab) and the in-place all-gather
    (gather_map) leaves the byte-exact map of values 0..mpv on every rank; slabs past the end
    of a small map stay empty."""
    import multiprocessing as mp
    import numpy as np
    sys.path.insert(0, PKG)
    from shard import map_slab
    ctx = mp.get_context("spawn")
    port = _free_port()
    out = str(tmp_path / "map.npy")
    procs = [ctx.Process(target=_slab_worker, args=(r, world, port, mpv, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
    codes = [p.exitcode for p in procs]
    for p in procs:
        if p.is_alive():
            p.kill()
    assert codes == [0] * world, codes
    got = np.load(out)
    want = oracle.build_map(mpv)
    nbytes = (mpv + 1 + 15) >> 4
    assert np.array_equal(got[:nbytes], want[:nbytes])
    bounds = [map_slab(mpv, world, r) for r in range(world)]
    assert bounds[0][0] == 0 and max(b[1] for b in bounds) == mpv + 1
    assert all(b[0] % 4096 == 0 for b in bounds if b[1] > b[0])


def test_shard_bounds_partition():
    sys.path.insert(0, PKG)
    from shard import odd_sums, shard_bounds
    for lo, hi in ((5, 2097151), (5, 65535), (1000001, 1002499), (5, 9), (7, 7)):
        for world in (1, 2, 3, 4, 8):
            parts = [shard_bounds(lo, hi, world, r) for r in range(world)]
            covered = [s for a, b in parts for s in range(a, b + 1, 2)]
            assert covered == list(range(lo, hi + 1, 2)), (lo, hi, world)
            assert all(a & 1 for a, b in parts)
            if world > 1 and hi - lo > 10000:
                cost = [b * b - a * a for a, b in parts]
                assert max(cost) / min(cost) < 1.01, (lo, hi, world, cost)
    assert sum(odd_sums(*shard_bounds(5, 2097151, 8, r)) for r in range(8)) == 1048574


def test_emit_rejects_records_that_do_not_cover(ffb):
    import numpy as np
    with pytest.raises(ValueError):
        ffb.emit((5, 2627), np.zeros(10, dtype=np.uint64), 5)
