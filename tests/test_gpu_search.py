"""GPU search through the C ABI: byte parity with the reference's goldens (every leg up to
2^21 by SHA-256), with the reference binary on short and quirk ranges, and per-sum parity
with the oracle under the m4_kernel_unit setup (map only up to sumLimit, so Miller-Rabin
answers most of the probes)."""
import ctypes
import hashlib
import math
import os
import re
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
NORM = re.compile(rb"(Prime|Freudenthal) time: [0-9]+")


def norm(b):
    return NORM.sub(rb"\1 time: N", b)


def sha(b):
    return hashlib.sha256(b).hexdigest()


def test_leg_65536_byte_exact(ffb, golden):
    assert norm(ffb.run(5, 65536)) == golden["leg65536"]
    assert ffb.take_errors() == 0


def test_small_ranges_match_reference_binary(ffb, golden):
    ctx = ffb.load().ffb_context_create(0)
    try:
        bad = [c["args"] for c in golden["small"] if sha(norm(ffb.run(*c["args"], ctx=ctx))) != c["sha256"]]
    finally:
        ffb.load().ffb_context_destroy(ctx)
    assert not bad, bad


@pytest.mark.parametrize("leg", [131072, 262144, 524288, 1048576, 2097152])
def test_leg_sha256(ffb, golden, leg):
    out = norm(ffb.run(5, leg))
    assert out.count(b") sum =") == golden["legs"][str(leg)]["solutions"]
    assert sha(out) == golden["legs"][str(leg)]["sha256"]


def test_cli_leg_65536(ffb, golden):
    exe = os.path.join(ROOT, "ff-gpu_b200", "bin", "ff_sieve")
    r = subprocess.run([exe, "5", "65536"], capture_output=True, check=True)
    assert norm(r.stdout) == golden["leg65536"]


def _m4_map(limit):
    """test/source/m4_kernel_unit.cpp:436-446: a map of (sumLimit>>4)+1 bytes sieved up to
    sumLimit, with maxPrimeMapValue = sumLimit."""
    import ffo
    m = np.full((limit >> 4) + 1, 0xFF, dtype=np.uint8)
    m[0] ^= 0x80
    primes = ffo.odd_primes(math.isqrt(limit))
    ffo.load().ffo_segment_fill(0, limit + 1, primes.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)),
                                len(primes), m.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)))
    return m


@pytest.mark.parametrize("start,limit", [(5, 65535), (40001, 46131), (250001, 262143)])
def test_search_kernel_run_records(ffb, oracle, start, limit):
    import torch
    lib = ffb.load()
    hmap = _m4_map(limit)
    dmap = torch.from_numpy(hmap).cuda()
    n = (limit - start) // 2 + 1
    rec = torch.zeros(n * 32, dtype=torch.uint8, device="cuda")
    cnt = torch.zeros(1, dtype=torch.int32, device="cuda")
    assert lib.SearchKernelGetLaunchFn_sm_120(0)
    rc = lib.GpuSearchLaunch(0, b"nvidia", dmap.data_ptr(), limit, start, limit, rec.data_ptr(),
                             cnt.data_ptr())
    assert rc == 0
    torch.cuda.synchronize()
    r = rec.cpu().numpy().view(np.uint8).reshape(n, 32)
    sums = r[:, 0:4].copy().view(np.uint32)[:, 0]
    lows = r[:, 8:16].copy().view(np.uint64)[:, 0]
    highs = r[:, 16:24].copy().view(np.uint64)[:, 0]
    with oracle.Context(limit, map_bound=limit) as ctx:
        want, _ = ctx.eval_range(start, limit)
    wl, wh = want >> np.uint64(32), want & np.uint64(0xFFFFFFFF)
    solved = want != 0
    idx = np.arange(n)
    assert np.array_equal(sums != 0, solved), idx[(sums != 0) != solved][:8]
    assert np.array_equal(sums[solved], (start + 2 * idx[solved]).astype(np.uint32))
    assert np.array_equal(lows[solved], wl[solved]) and np.array_equal(highs[solved], wh[solved])
    assert int(cnt.item()) == int(solved.sum())
    assert lib.GpuSearchLaunch(0, b"amd", dmap.data_ptr(), limit, start, limit, rec.data_ptr(),
                               cnt.data_ptr()) == -1
    assert ffb.take_errors() == 0


def test_output_independent_of_map_bound_on_gpu(ffb, oracle):
    """Finding: IsPrime is exact with Miller-Rabin above the map, so any map bound gives the
    same records (here a 2^20-value map against the full map of the 2^18 leg)."""
    import torch
    lib = ffb.load()
    g, _ = ffb.geometry(5, 262144)
    full = torch.empty(((g.maxPrimeMapValue + 1 + 15) >> 4) + 16, dtype=torch.uint8, device="cuda")
    assert lib.ffb_sieve_map_async(0, g.maxPrimeMapValue, full.data_ptr(), None) == 0
    lo, hi = 200001, 262143
    n = (hi - lo) // 2 + 1
    a = torch.empty(n, dtype=torch.int64, device="cuda")
    b = torch.empty(n, dtype=torch.int64, device="cuda")
    assert lib.ffb_search_async(0, full.data_ptr(), g.maxPrimeMapValue, lo, hi, a.data_ptr(), None) == 0
    assert lib.ffb_search_async(0, full.data_ptr(), (1 << 20) - 1, lo, hi, b.data_ptr(), None) == 0
    torch.cuda.synchronize()
    assert torch.equal(a, b)
    assert int((a != 0).sum()) > 0
    assert ffb.take_errors() == 0


@pytest.mark.parametrize("args,budget", [((5, 262144), 64 << 20), ((5, 65536), 1 << 20)])
def test_run_with_a_capped_map(ffb, golden, args, budget):
    """ffb_run under a map budget far below the job's map (the path a job whose map exceeds
    device memory takes): the largest map under the cap, Miller-Rabin above it, and the
    text still ff_seg's."""
    lib = ffb.load()
    ctx = lib.ffb_context_create(0)
    try:
        assert lib.ffb_context_set_map_budget(ctx, budget) == 0
        text = ffb.run(*args, ctx=ctx)
    finally:
        lib.ffb_context_destroy(ctx)
    leg = golden["legs"][str(args[1])]
    assert hashlib.sha256(norm(text)).hexdigest() == leg["sha256"]
    assert ffb.take_errors() == 0


def test_every_launch_shape_gives_the_same_records(ffb, oracle):
    """ffb_search_shape_async over every shape the batch's autotuner times (warps per block,
    warps per sum, sums per chunk): the records of a range near 2^19 all equal the ordinary
    launch's, which equal the oracle's on the same sums; shapes outside the offered set and
    several warps per sum over a map that does not cover every probe are refused."""
    import torch
    lib = ffb.load()
    lo, hi = 450001, 524287
    mpv = lib.ffb_probe_bound(hi)
    d_map = torch.empty(((mpv + 1 + 15) >> 4) + 256, dtype=torch.uint8, device="cuda")
    assert lib.ffb_sieve_map_async(0, mpv, d_map.data_ptr(), None) == 0
    n = (hi - lo) // 2 + 1
    want = torch.empty(n, dtype=torch.int64, device="cuda")
    assert lib.ffb_search_async(0, d_map.data_ptr(), mpv, lo, hi, want.data_ptr(), None) == 0
    torch.cuda.synchronize()
    shapes = [(w, c, 1) for w in (4, 8, 16) for c in (16, 32, 64)] + \
             [(w, 32 * g, g) for w in (4, 8, 16) for g in (2, 4)]
    for w, c, g in shapes:
        got = torch.full((n,), -1, dtype=torch.int64, device="cuda")
        assert lib.ffb_search_shape_async(0, d_map.data_ptr(), mpv, lo, hi, got.data_ptr(), w, c, g,
                                          None) == 0
        torch.cuda.synchronize()
        assert torch.equal(got, want), (w, c, g)
    assert ffb.take_errors(0) == 0
    # the oracle on the first 2000 sums (low<<32|high; the device adds the two prime flags)
    with oracle.Context(hi + 2, map_bound=(1 << 32) - 1) as c:
        rec, _ = c.eval_range(lo, lo + 3998)
    w = want[:2000].cpu().numpy().view(np.uint64) & np.uint64(0x7FFFFFFF7FFFFFFF)
    assert np.array_equal(w, rec)
    p = d_map.data_ptr()
    assert lib.ffb_search_shape_async(0, p, mpv, lo, hi, want.data_ptr(), 8, 48, 1, None) == -1
    assert lib.ffb_search_shape_async(0, p, mpv, lo, hi, want.data_ptr(), 8, 32, 2, None) == -1
    assert lib.ffb_search_shape_async(0, p, 1 << 20, lo, hi, want.data_ptr(), 8, 64, 2, None) == -1
    assert lib.ffb_search_shape_async(0, p, mpv, lo, hi, want.data_ptr(), 12, 32, 1, None) == -1
    # below the probes (the Miller-Rabin variant) only one warp per sum and 32 sums a chunk
    assert lib.ffb_search_shape_async(0, p, 1 << 20, lo, hi, want.data_ptr(), 8, 64, 1, None) == -1


def test_ranges_above_2_21_match_reference_binary(ffb):
    """ffb_run on the short ranges above 2^21 that the reference binary ran
    (tests/golden/above_2_21.json)."""
    import json
    with open(os.path.join(ROOT, "tests", "golden", "above_2_21.json")) as f:
        cases = json.load(f)
    for c in cases:
        assert sha(norm(ffb.run(*c["args"]))) == c["sha256"], c["args"]
