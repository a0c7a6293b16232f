"""GPU sieve through the C ABI against the oracle's restatement of SegmentFill.

Ranges follow the reference's own sieve unit test (test/source/slab_cmp.cpp:232-265), plus
unaligned/odd segment starts, the full-map engine, and the sieve-sweep sizes with their
exact prime counts."""
import ctypes
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

u8p = ctypes.POINTER(ctypes.c_uint8)
u32p = ctypes.POINTER(ctypes.c_uint32)

SLAB_CMP = [(0, 65536), (0, 524288), (0, 1048576), (500000, 524288), (100000, 300000),
            (0, 256), (524288, 1048576), (524272, 524400), (1200, 2000), (0, 2000000)]
EXTRA = [(1, 5000), (7, 100003), (3, 17), (0, 1), (0, 17), (999999, 1000001), (123457, 9876543),
         (2 ** 33 - 12345, 2 ** 33 + 3000000)]


def small_primes(hi, with_two):
    """test/source/slab_cmp.cpp:62-91: primes up to isqrt(segHi), 2 included."""
    import ffo
    p = ffo.odd_primes(max(math.isqrt(hi), 2)).astype(np.uint32)
    return np.concatenate([[2], p]).astype(np.uint32) if with_two else p


def slab_run(ffb, lo, hi, primes, fn="SieveSlabRun_sm_120"):
    out = np.zeros((hi + 15) >> 4, dtype=np.uint8)
    rc = getattr(ffb.load(), fn)(0, primes.ctypes.data_as(u32p), len(primes), lo, hi,
                                 out.ctypes.data_as(u8p))
    assert rc == 0
    return out


@pytest.mark.parametrize("lo,hi", SLAB_CMP + EXTRA)
@pytest.mark.parametrize("with_two", [True, False])
def test_slab_matches_segment_fill(ffb, oracle, lo, hi, with_two):
    primes = small_primes(hi, with_two)
    got = slab_run(ffb, lo, hi, primes)
    want = oracle.slab_relative(lo, hi, primes)
    assert np.array_equal(got, want), np.nonzero(got != want)[0][:8]


def test_slab_sparse_and_unsorted_lists(ffb, oracle):
    # lists that are not the standard prime prefix take the literal path
    for primes in ([3, 7, 13], [5, 3], [2, 2, 9], [1], [0, 3], [17, 19, 23, 1009]):
        pr = np.array(primes, dtype=np.uint32)
        assert np.array_equal(slab_run(ffb, 1000, 120000, pr), oracle.slab_relative(1000, 120000, pr))


@pytest.mark.parametrize("mpv", [15, 31, 1023, 268435471, 2 ** 24 + 15, 123456789])
def test_engine_full_map(ffb, oracle, mpv):
    primes = oracle.odd_primes(math.isqrt(mpv))
    out = np.zeros((mpv + 1 + 15) >> 4, dtype=np.uint8)
    rc = ffb.load().SieveSlabEngineRun_sm_100a(0, primes.ctypes.data_as(u32p), len(primes), mpv,
                                               out.ctypes.data_as(u8p))
    assert rc == 0
    assert np.array_equal(out, oracle.build_map(mpv))


POP = None


def prime_count_below(d_map, n):
    """Primes < n (n a multiple of 16) from a device map: popcount of its first n/16 bytes,
    plus one for 2."""
    import torch
    global POP
    if POP is None:
        POP = torch.tensor([bin(i).count("1") for i in range(256)], dtype=torch.int64, device="cuda")
    return int(POP[d_map[: n // 16].long()].sum().item()) + 1


@pytest.mark.parametrize("logn,pi", [(24, 1077871), (28, 14630843), (32, 203280221)])
def test_sieve_sweep_prime_counts(ffb, oracle, logn, pi):
    import torch
    n = 1 << logn
    d = torch.empty(((n + 1 + 15) >> 4) + 16, dtype=torch.uint8, device="cuda")
    assert ffb.load().ffb_sieve_map_async(0, n, d.data_ptr(), None) == 0
    torch.cuda.synchronize()
    assert prime_count_below(d, n) == pi
    if logn <= 28:
        assert np.array_equal(d[: (n + 16) >> 4].cpu().numpy(), oracle.build_map(n))
    else:  # windows of the 2^32 map against the literal fill
        rnd = np.random.default_rng(1)
        host = d.cpu().numpy()
        primes = oracle.odd_primes(1 << 16)
        for start in rnd.integers(0, n >> 4, 8):
            lo = int(start) << 4
            hi = min(lo + (1 << 20), n + 1)
            want = oracle.slab_relative(lo, hi, primes)[: (hi - lo + 15) >> 4]
            got = host[lo >> 4: (hi + 15) >> 4]
            assert np.array_equal(got[: len(want) - 1], want[:-1])


@pytest.mark.parametrize("tile_kb", [64, 96, 128, 160, 192, 216])
def test_sieve_tile_sizes_give_the_same_map(ffb, oracle, tile_kb):
    """The C3 sweep's tile sizes (ffb_sieve_map_tiled_async): every tile gives the map of the
    literal fill (2^28) and the exact prime count."""
    import torch
    n = 1 << 28
    d = torch.empty(((n + 1 + 15) >> 4) + 16, dtype=torch.uint8, device="cuda")
    assert ffb.load().ffb_sieve_map_tiled_async(0, n, d.data_ptr(), tile_kb * 1024, None) == 0
    torch.cuda.synchronize()
    assert prime_count_below(d, n) == 14630843
    assert np.array_equal(d[: (n + 16) >> 4].cpu().numpy(), oracle.build_map(n))


def test_sieve_tile_size_limits(ffb):
    lib = ffb.load()
    assert lib.ffb_sieve_map_tiled_async(0, 1 << 20, None, 217 * 1024, None) == -1
    assert lib.ffb_sieve_map_tiled_async(0, 1 << 20, None, 1000, None) == -1


def test_pool_ops_and_semantics(ffb, oracle):
    """slabCompute(primeSlab=0) clears bits INTO whatever the slab holds, like the reference."""
    lib = ffb.load()
    pool = lib.SievePoolGet_sm_100a(0)
    assert pool
    import torch
    primes = oracle.odd_primes(1000)
    lo, hi = 2 ** 20, 2 ** 20 + 500000
    nbytes = (hi - lo + 15) >> 4
    rnd = np.random.default_rng(3)
    init = rnd.integers(0, 256, nbytes, dtype=np.uint8)
    d = torch.from_numpy(init.copy()).cuda()

    class Ops(ctypes.Structure):
        _fields_ = [(n, ctypes.c_void_p) for n in (
            "alloc", "memset", "free", "copyH2D", "copyD2H", "slabCompute", "createStream",
            "destroyStream", "createEvent", "destroyEvent", "recordEvent", "waitEvent", "syncEvent",
            "elapsedEvents", "allocPinned", "freePinned", "copyH2DAsync", "copyD2HAsync",
            "slabComputeAsync")]
    ops = Ops.from_address(pool)
    slab = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_int, u32p, ctypes.c_uint32, ctypes.c_uint64,
                            ctypes.c_uint64, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_int)(ops.slabCompute)
    assert slab(0, primes.ctypes.data_as(u32p), len(primes), lo, hi, d.data_ptr(), nbytes, 0) == 0
    want = init & oracle.slab_relative(lo, hi, primes)[:nbytes]
    assert np.array_equal(d.cpu().numpy(), want)
    # primed: memset 0xff first -> the plain slab
    assert slab(0, primes.ctypes.data_as(u32p), len(primes), lo, hi, d.data_ptr(), nbytes, 1) == 0
    assert np.array_equal(d.cpu().numpy(), oracle.slab_relative(lo, hi, primes)[:nbytes])
    # alloc/free/event round trip
    alloc = ctypes.CFUNCTYPE(ctypes.c_void_p, ctypes.c_int, ctypes.c_uint64)(ops.alloc)
    free = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_int, ctypes.c_void_p)(ops.free)
    p = alloc(0, 1 << 20)
    assert p and free(0, p) == 0


@pytest.mark.parametrize("world", [2, 3, 8])
def test_map_range_slabs_assemble_the_map(ffb, oracle, world):
    """ffb_sieve_map_range_async on each rank's slab (shard.map_slab), written at its place in
    one buffer, gives the whole map: what a sharded job all-gathers."""
    import torch
    from shard import map_slab
    mpv = (1 << 28) + 12345 * 16 + 15
    slab = map_slab(mpv, world, 0)[2]
    d = torch.full((world * slab + 256,), 0xA5, dtype=torch.uint8, device="cuda")
    lib = ffb.load()
    for r in range(world):
        lo, hi, _ = map_slab(mpv, world, r)
        if hi > lo:
            assert lib.ffb_sieve_map_range_async(0, lo, hi, d.data_ptr() + (lo >> 4), None) == 0
    torch.cuda.synchronize()
    n = (mpv + 1 + 15) >> 4
    assert np.array_equal(d[:n].cpu().numpy(), oracle.build_map(mpv)[:n])
    assert lib.ffb_sieve_map_range_async(0, 100, 1000, d.data_ptr(), None) == -1   # unaligned
    assert ffb.take_errors(0) == 0
