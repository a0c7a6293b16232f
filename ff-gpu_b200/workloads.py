"""Seeded synthetic workloads of the batched and served modes.

Both use numpy's PCG64 generator with the stated seed:

* batched (seed 0): 256 ranges, start ~ U{5..2^21}, length = floor(2^U[8,18]),
  limit = start + length - 1 (every range has at least 128 odd sums);
* served (seed 1): 10,000 requests, limit ~ U{69..2^22}, length = floor(2^U[6,20]),
  start = max(5, limit - length + 1), Poisson arrivals (exponential gaps) at a given rate.

Each range is an `ff_sieve <start> <limit>` request; its output is what ff_seg prints for it.
"""
import numpy as np


def batched_ranges(seed=0, n=256):
    rng = np.random.Generator(np.random.PCG64(seed))
    starts = rng.integers(5, 2 ** 21, size=n, endpoint=True)
    lengths = np.floor(2.0 ** rng.uniform(8, 18, size=n)).astype(np.int64)
    return [(int(s), int(s + l - 1)) for s, l in zip(starts, lengths)]


def served_requests(seed=1, n=10000, rate=100.0):
    """[(arrival_seconds, start, limit)] sorted by arrival."""
    rng = np.random.Generator(np.random.PCG64(seed))
    limits = rng.integers(69, 2 ** 22, size=n, endpoint=True)
    lengths = np.floor(2.0 ** rng.uniform(6, 20, size=n)).astype(np.int64)
    starts = np.maximum(5, limits - lengths + 1)
    gaps = rng.exponential(1.0 / rate, size=n)
    arrivals = np.cumsum(gaps)
    return [(float(t), int(s), int(l)) for t, s, l in zip(arrivals, starts, limits)]
