"""The CPU restatement (oracle/) pinned against the reference's goldens and against the
reference binary's outputs committed under tests/golden/."""
import hashlib
import random

import numpy as np
import pytest


def sha(b):
    return hashlib.sha256(b).hexdigest()


def test_leg_65536_byte_exact(oracle, golden):
    out = oracle.run(5, 65536)
    assert out == golden["leg65536"]
    assert out.count(b") sum =") == golden["legs"]["65536"]["solutions"]


@pytest.mark.parametrize("leg", [131072, 262144])
def test_leg_sha256(oracle, golden, leg):
    out = oracle.run(5, leg)
    assert sha(out) == golden["legs"][str(leg)]["sha256"]
    assert out.count(b") sum =") == golden["legs"][str(leg)]["solutions"]


def test_small_ranges_match_reference_binary(oracle, golden):
    # a map up to 2^20 keeps each case fast; the map bound does not change the output
    # (test_output_independent_of_map_bound)
    bad = [c["args"] for c in golden["small"]
           if sha(oracle.run(*c["args"], map_bound=1 << 20, threads=2)) != c["sha256"]]
    assert not bad, f"oracle differs from ff_seg on {bad}"


@pytest.mark.parametrize("bound", [65536, 1000, 16])
def test_output_independent_of_map_bound(oracle, golden, bound):
    # Miller-Rabin is exact over the domain, so the map is only a cache
    assert oracle.run(5, 65536, map_bound=bound) == golden["leg65536"]


def test_geometry_kats(oracle):
    # test/source/budget_selftest.cpp:45-57
    g, _ = oracle.geometry(5, 2097152)
    assert g.max_prime_map_value == 274877906959
    assert (g.max_prime_map_value + 1 + 15) >> 4 == 17179869185
    g, _ = oracle.geometry(5, 1048576)
    assert (g.max_prime_map_value + 1 + 15) >> 4 == 4294967297
    g, hdr = oracle.geometry(5, 65536)
    assert (g.max_prime_map_value + 1 + 15) >> 4 == 16777217
    assert hdr == (b"maxPrimeMapValue 268435471 numPrimesRequested 3538 totalBytes 16791369\n"
                   b"maxPrimeMapValue 268435471 numPrimesRequested 3538 sqrtLimit 16384\n")
    assert oracle.parse_args(6, 100) == (7, 100)
    assert oracle.parse_args() == (5, 2627)
    assert oracle.parse_args(99, 98) == (99, 99)


def test_renormalised_header(oracle):
    # above sumLimit ~4.83M the reference caps the map at PRIMEMEM (segmentedSieve.C:148-176)
    g, hdr = oracle.geometry(5, 6000000)
    assert g.renormalised == 1
    assert hdr.count(b"\n") == 3
    assert g.max_prime_map_value == ((85 << 30) - 4 * g.num_primes_requested << 4) - 1


def _py_mr(n):
    """Deterministic Miller-Rabin for n < 3.3e24 (first 12 prime bases)."""
    if n < 2:
        return False
    for p in (2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37):
        if n % p == 0:
            return n == p
    d, s = n - 1, 0
    while d % 2 == 0:
        d //= 2
        s += 1
    for a in (2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37):
        x = pow(a, d, n)
        if x in (1, n - 1):
            continue
        for _ in range(s - 1):
            x = x * x % n
            if x == n - 1:
                break
        else:
            return False
    return True


def test_miller_rabin_against_exact(oracle):
    rnd = random.Random(7)
    cases = [3215031751, 2152302898747, 3474749660383, 341550071728321 - 2,
             1000000000039, 999999999989, 2 ** 47 - 115, 25326001, 3825123056546413051 % (2 ** 48) | 1]
    cases += [rnd.randrange(17, 2 ** 48) | 1 for _ in range(3000)]
    for n in cases:
        assert oracle.miller_rabin(n) == _py_mr(n), n


def _segment_fill_py(lo, hi, primes, nbytes):
    m = np.full(nbytes, 0xFF, dtype=np.uint8)
    if lo == 0:
        m[0] ^= 0x80
    for p in primes:
        p = int(p)
        if p * p >= hi:
            continue
        first = max(p * p, -(-lo // p) * p)
        if first % 2 == 0:
            first += p
        i = np.arange(first, hi, 2 * p, dtype=np.int64)
        np.bitwise_and.at(m, (i - lo) >> 4, ~(0x80 >> ((((i - lo) >> 1) & 7))).astype(np.uint8))
    return m


# test/source/slab_cmp.cpp:232-265
SLAB_CMP = [(0, 65536), (0, 524288), (0, 1048576), (500000, 524288), (100000, 300000),
            (0, 256), (524288, 1048576), (524272, 524400), (1200, 2000), (0, 2000000)]


@pytest.mark.parametrize("lo,hi", SLAB_CMP[:9] + [(1201, 3000), (7, 500)])
def test_slab_relative_matches_literal_fill(oracle, lo, hi):
    primes = np.concatenate([[2], oracle.odd_primes(int(hi ** 0.5) + 1)]).astype(np.uint32)
    got = oracle.slab_relative(lo, hi, primes)
    want = _segment_fill_py(lo, hi, primes, (hi + 15) >> 4)
    assert np.array_equal(got, want)


def test_ranges_above_2_21_match_reference_binary(oracle):
    """Short ranges with limits from 2.2M to 3.2M (the served configuration's limits reach
    2^22, beyond the reference's legs), against the reference binary's output
    (tests/golden/above_2_21.json): the oracle with a 2^30 map and Miller-Rabin above it."""
    import json
    import os
    with open(os.path.join(os.path.dirname(__file__), "golden", "above_2_21.json")) as f:
        cases = json.load(f)
    assert len(cases) >= 5 and min(c["args"][1] for c in cases) > 1 << 21
    for c in cases:
        out = oracle.run(*c["args"], map_bound=(1 << 30) - 1)
        assert sha(out) == c["sha256"], c["args"]
