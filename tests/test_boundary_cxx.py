"""The C++ half of the boundary, called from C++ (tests/cxx/boundary_check.cpp) the way the
reference's own harnesses call it:

* GpuPrime::IsPrime / operator[] / AskMillerRabin (source/gpu_prime.cpp:8-71) over a host map,
  on values below, at and above the map bound (Miller-Rabin there), against the oracle;
* PrintOutputTags (source/m4/gpu_search_emission.cpp:34-50) against the reference's tag rule;
* GpuSearchLaunch + GpuSearchEmit (gpu_search_emission.cpp:84-96, the m4_order harness's
  sequence) on the 5..65536 leg, against the solution lines of the reference golden.
"""
import math
import os
import random
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "ff-gpu_b200")
BIN = os.path.join(PKG, "bin", "boundary_check")


@pytest.fixture(scope="module")
def binary():
    subprocess.run(["make", "-s", "-C", PKG, "check"], check=True)
    return BIN


@pytest.fixture(scope="module")
def small_map(oracle, tmp_path_factory):
    mpv = (1 << 24) - 1
    m = oracle.build_map(mpv)
    path = tmp_path_factory.mktemp("map") / "map.bin"
    m.tofile(path)
    return str(path), mpv


def _values(mpv):
    rnd = random.Random(7)
    vals = list(range(0, 200)) + [mpv - 2, mpv - 1, mpv, mpv + 1, mpv + 2, mpv + 4]
    vals += [rnd.randrange(3, mpv) for _ in range(3000)]
    vals += [rnd.randrange(mpv, 1 << 47) | 1 for _ in range(3000)]
    # strong pseudoprimes and the reference's Miller-Rabin thresholds
    vals += [2047, 1373653, 25326001, 3215031751, 3215031753, 2152302898747, 2152302898749,
             3474749660383, 3474749660385, 341550071728321 - 2, (1 << 47) - 1, (1 << 48) - 59]
    # primes above the map (every base runs)
    vals += [p for p in (1000000007, 998244353, 4294967291, 281474976710597) if p > mpv]
    return vals


def test_gpu_prime_matches_oracle(binary, small_map, oracle):
    path, mpv = small_map
    vals = _values(mpv)
    r = subprocess.run([binary, "isprime", path, str(mpv)], input="\n".join(map(str, vals)),
                       capture_output=True, text=True, check=True)
    lines = r.stdout.split("\n")
    assert len([ln for ln in lines if ln]) == len(vals)
    with oracle.Context(5000, map_bound=mpv) as c:
        for v, ln in zip(vals, lines):
            n, isp, op, mr = ln.split()
            assert int(n) == v
            want = c.is_prime(v)
            assert int(isp) == want and int(op) == want, v
            if v % 2 == 1 and v > 2:
                assert int(mr) == oracle.miller_rabin(v), v


def _tag(is_prime, term, last):
    """PrintOutputTags' rule (source/m4/gpu_search_emission.cpp:34-50)."""
    if is_prime:
        return " (prime)" + (", " if last else "")
    if term & -term == term:
        n = round(math.log2(term))
        s = f" (2^{n})"
        if last:
            s += "," + " " * max(1, 3 - math.floor(math.log10(n + 0.001)))
        return s
    return ",         " if last else ""


def test_print_output_tags(binary, small_map, oracle):
    path, mpv = small_map
    terms = [1, 2, 3, 4, 5, 6, 7, 8, 9, 15, 16, 17, 1024, 1025, 65536, 1 << 20, (1 << 20) + 7,
             1 << 23, 16777213, 33554432, 1 << 40, 1000003]
    r = subprocess.run([binary, "tags", path, str(mpv)], input="\n".join(map(str, terms)),
                       capture_output=True, text=True, check=True)
    got = r.stdout.split("\n")
    with oracle.Context(5000, map_bound=mpv) as c:
        for t, ln in zip(terms, got):
            p = c.is_prime(t)
            assert ln == f"{t}|{_tag(p, t, True)}|{_tag(p, t, False)}|", t


@pytest.mark.gpu
def test_gpu_search_emit_leg_65536(binary, golden):
    r = subprocess.run([binary, "emit", "65536"], capture_output=True, check=True)
    want = b"".join(ln + b"\n" for ln in golden["leg65536"].split(b"\n") if b") sum =" in ln)
    assert r.stdout == want
    assert b"2357 solutions" in r.stderr
