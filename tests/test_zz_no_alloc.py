"""ffb_search_noalloc: the search for callers that cannot call cudaMalloc (a host whose
device memory belongs to its own pool or framework allocator, or a latency-critical caller
for which an allocation or free may synchronise the device). Its scratch is an array
compiled into the library, so the tests check that
  * it gives exactly the records of the ordinary entry point, ffb_search_async, on two calls
    in a row (the array keeps the previous call's contents);
  * called first in a fresh process (no other entry point of the library has run, so none
    of its allocated per-device state exists), it gives the oracle's records, and a second
    call leaves the device's free memory unchanged;
  * out-of-range requests, and a missing error word, are refused.

This file is named to be collected last, so a run that stops at the first failure has
already run every other test; it also passes on its own in a fresh process."""
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _map(ffb, limit, hi):
    import torch
    lib = ffb.load()
    mpv = max(ffb.geometry(5, limit)[0].maxPrimeMapValue, lib.ffb_probe_bound(hi))
    d_map = torch.empty(((mpv + 1 + 15) >> 4) + 64, dtype=torch.uint8, device="cuda")
    assert lib.ffb_sieve_map_async(0, mpv, d_map.data_ptr(), None) == 0
    return d_map, mpv


@pytest.mark.parametrize("bound_kind", ["full", "small"])
def test_noalloc_matches_search_async_twice(ffb, bound_kind):
    import torch
    lib = ffb.load()
    lo, hi = 200001, 262143
    d_map, mpv = _map(ffb, 262144, hi)
    # "small": most probes above the bound go to Miller-Rabin (integer work: exact match)
    bound = mpv if bound_kind == "full" else (1 << 20) - 1
    n = (hi - lo) // 2 + 1
    want = torch.empty(n, dtype=torch.int64, device="cuda")
    assert lib.ffb_search_async(0, d_map.data_ptr(), bound, lo, hi, want.data_ptr(), None) == 0
    torch.cuda.synchronize()
    assert ffb.take_errors(0) == 0
    assert int((want != 0).sum()) > 0
    err = torch.full((1,), 7, dtype=torch.int32, device="cuda")
    for _ in range(2):
        got = torch.full((n,), -1, dtype=torch.int64, device="cuda")  # must be overwritten
        rc = lib.ffb_search_noalloc(0, d_map.data_ptr(), bound, lo, hi, got.data_ptr(),
                                    err.data_ptr(), None)
        assert rc == 0
        torch.cuda.synchronize()
        assert torch.equal(got, want)
        assert int(err.item()) == 0


# Runs in a fresh interpreter: the map is sieved on the CPU by the oracle and copied in by
# torch (the caller's own memory), so ffb_search_noalloc is the first and only entry point
# of the library that runs on the device.
_FIRST_CALL = r"""
import sys
import numpy as np
import torch
sys.path[:0] = [sys.argv[1] + "/ff-gpu_b200", sys.argv[1] + "/oracle"]
import ffb200, ffo
lo, hi, mpv = 100001, 131071, (1 << 30) - 1
h_map = ffo.build_map(mpv)
with ffo.Context(hi + 2, map_bound=mpv) as c:
    want, _ = c.eval_range(lo, hi)
lib = ffb200.load()
torch.cuda.init()
d_map = torch.from_numpy(h_map).cuda()
n = (hi - lo) // 2 + 1
err = torch.full((1,), 7, dtype=torch.int32, device="cuda")
free = []
for i in range(2):
    got = torch.full((n,), -1, dtype=torch.int64, device="cuda")
    torch.cuda.synchronize()
    free.append(torch.cuda.mem_get_info()[0])
    assert lib.ffb_search_noalloc(0, d_map.data_ptr(), mpv, lo, hi, got.data_ptr(),
                                  err.data_ptr(), None) == 0
    torch.cuda.synchronize()
    free.append(torch.cuda.mem_get_info()[0])
    g = got.cpu().numpy().view(np.uint64)
    # the oracle packs low<<32|high; the device record adds the two primality flags
    assert np.array_equal(g & np.uint64(0x7FFFFFFF7FFFFFFF), want), f"call {i}: records differ"
    assert int(err.item()) == 0
    assert (g != 0).sum() > 0
assert free[2] == free[3], f"the second call changed free device memory: {free}"
print("first-call: ok")
"""


def test_noalloc_first_call_in_fresh_process():
    r = subprocess.run([sys.executable, "-c", _FIRST_CALL, ROOT], capture_output=True,
                       text=True, timeout=600)
    assert r.returncode == 0 and "first-call: ok" in r.stdout, r.stdout + r.stderr


def test_noalloc_rejects_out_of_range(ffb):
    import torch
    lib = ffb.load()
    buf = torch.zeros(64, dtype=torch.int64, device="cuda")
    p = buf.data_ptr()
    assert lib.ffb_search_noalloc(0, p, 1000, 4, 101, p, p, None) == -1          # even first sum
    assert lib.ffb_search_noalloc(0, p, 1000, 101, 99, p, p, None) == -1         # empty range
    assert lib.ffb_search_noalloc(0, p, 1000, 5, (1 << 25) + 3, p, p, None) == -1  # beyond 2^25
    assert lib.ffb_search_noalloc(0, None, 1000, 5, 101, p, p, None) == -1       # no map
    assert lib.ffb_search_noalloc(0, p, 1000, 5, 101, p, None, None) == -1       # no error word
    assert lib.ffb_search_noalloc(99, p, 1000, 5, 101, p, p, None) == -1         # no device
