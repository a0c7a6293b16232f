"""Algorithmic work of the reference search on the 2^21 job (odd sums 5 .. 2^21-1), counted
by the instrumented CPU restatement (oracle/, test infrastructure), for the integer roofline
that bench.py reports for the search kernel.

The oracle runs the reference algorithm (reference/segmentedSieve.C:408-639, 800-823) and
counts per sum: IsPrime calls, (evenTerm, oddTerm) splits handed to DoesPeterKnow,
AllButOne... calls, the trial-division steps inside them and the divisor pairs they test.
The counts are taken on 64 windows of 512 consecutive odd sums spread evenly over the job
(midpoint rule; the per-sum work is a smooth function of the sum) and scaled to the job.
IsPrime calls are counted whether the oracle's map or its Miller-Rabin answered them: on
the device the map covers every probe of the job, so each is one map lookup.

Writes tests/golden/search_work.json. Run from the repository root (a few minutes):
    python tests/golden/make_search_work.py
"""
import json
import os
import sys
import time

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

LO, HI = 5, (1 << 21) - 1
WINDOWS, WIDTH = 64, 512


def main():
    import ffo
    total = (HI - LO) // 2 + 1
    keys = ("map_probes", "mr_calls", "splits", "abop_calls", "trial_steps", "divisors")
    acc = {k: 0 for k in keys}
    sampled = 0
    t0 = time.time()
    with ffo.Context(HI + 2, map_bound=(1 << 33) - 1, threads=8) as c:
        for i in range(WINDOWS):
            centre = LO + (2 * i + 1) * (HI - LO) // (2 * WINDOWS)
            lo = max(LO, (centre - WIDTH) | 1)
            hi = lo + 2 * (WIDTH - 1)
            _, k = c.eval_range(lo, hi, threads=8)
            for key in keys:
                acc[key] += k[key]
            sampled += k["sums"]
    scale = total / sampled
    per_job = {"isprime_calls": round((acc["map_probes"] + acc["mr_calls"]) * scale)}
    for key in ("splits", "abop_calls", "trial_steps", "divisors"):
        per_job[key] = round(acc[key] * scale)
    doc = {"workload": f"odd sums {LO}..{HI} ({total} sums), the 2^21 job",
           "sample": f"{WINDOWS} windows of {WIDTH} consecutive odd sums at evenly spaced "
                     f"centres ({sampled} sums), scaled by {scale:.3f}",
           "generator": "tests/golden/make_search_work.py (instrumented CPU restatement, oracle/)",
           "per_job": per_job}
    with open(os.path.join(ROOT, "tests", "golden", "search_work.json"), "w") as f:
        json.dump(doc, f, indent=1)
    print(json.dumps(doc, indent=1), f"\n{time.time() - t0:.0f} s")


if __name__ == "__main__":
    main()
