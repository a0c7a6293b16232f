"""Oracle fixtures for the batched and served workloads: ff_seg's text for every range.

For the batched configuration (256 ranges, seed 0) and the first requests of the served
stream (seed 1) this evaluates the union of all their sums ONCE with the CPU restatement
(oracle/, test infrastructure) and emits each range's stdout from those records with
ffo_emit (header, the 62-way schedule's lines, timing lines normalised to N), writing:

  batched_seed0.json   per range: args, sha256 of the normalised stdout, solution count,
                       byte length
  served_seed1.json    the same for the first --served requests (default 300) in arrival
                       order

The oracle's map covers values up to --map-bound (default 2^39 - 1, 34 GB of RAM: every
probe of sums up to 2.57M); probes above it are answered by the deterministic Miller-Rabin,
which is exact there, so the texts do not depend on the bound. Run from the repository
root (about an hour on 8 cores):
    python tests/golden/make_workload_golden.py [--served 300] [--threads 8]
"""
import argparse
import hashlib
import json
import os
import sys
import time

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "ff-gpu_b200"))
OUT = os.path.join(ROOT, "tests", "golden")


def schedule_span(ffo, a, b):
    """(first, last) odd sums evaluated for `ff_seg a b`, or None when there are none."""
    g, _ = ffo.geometry(*ffo.parse_args(a, b))
    lo, hi = None, None
    for f, l in ffo.schedule(g.sum_start, g.sum_limit, g.max_prime_map_value):
        f |= 1
        l -= 1 - (l & 1)
        if f > l:
            continue
        lo = f if lo is None else min(lo, f)
        hi = l if hi is None else max(hi, l)
    return None if lo is None else (lo, hi)


def merged(spans):
    out = []
    for f, l in sorted(s for s in spans if s):
        if out and f <= out[-1][1] + 2:
            out[-1][1] = max(out[-1][1], l)
        else:
            out.append([f, l])
    return out


def fixtures(ffo, ctx, arg_lists, threads, label):
    spans = [schedule_span(ffo, a, b) for a, b in arg_lists]
    groups = merged(spans)
    recs = []
    t0 = time.time()
    for f, l in groups:
        r, _ = ctx.eval_range(f, l, threads=threads)
        recs.append((f, l, r))
        print(f"{label}: evaluated {f}..{l} ({(l - f) // 2 + 1} sums) at {time.time() - t0:.0f} s",
              file=sys.stderr, flush=True)
    rows = []
    for (a, b), sp in zip(arg_lists, spans):
        if sp is None:
            f, l, r = 1, 1, None
        else:
            f, l, r = next(g for g in recs if g[0] <= sp[0] and sp[1] <= g[1])
        if r is None:
            text = ffo.run(a, b, map_bound=1 << 20)
        else:
            text = ctx.emit([a, b], r, f)
        rows.append({"args": [a, b], "sha256": hashlib.sha256(text).hexdigest(),
                     "solutions": text.count(b") sum ="), "bytes": len(text)})
    return rows, groups


def main():
    import ffo
    import workloads
    ap = argparse.ArgumentParser()
    ap.add_argument("--served", type=int, default=300)
    ap.add_argument("--threads", type=int, default=8)
    ap.add_argument("--map-bound", type=int, default=(1 << 39) - 1)
    args = ap.parse_args()
    batched = workloads.batched_ranges(seed=0)
    served = [(a, b) for _, a, b in workloads.served_requests(seed=1)[:args.served]]
    top = max(max(b for _, b in batched), max(b for _, b in served)) + 64
    t0 = time.time()
    with ffo.Context(top, map_bound=args.map_bound, threads=args.threads) as ctx:
        print(f"map to {args.map_bound} sieved in {time.time() - t0:.0f} s", file=sys.stderr,
              flush=True)
        for name, arg_lists, desc in (
                ("batched_seed0.json", batched,
                 "256 ranges from seed 0: start U{5..2^21}, length floor(2^U[8,18])"),
                ("served_seed1.json", served,
                 f"the first {len(served)} requests of the seed-1 served stream: limit "
                 f"U{{69..2^22}}, length floor(2^U[6,20]), start max(5, limit-length+1)")):
            rows, groups = fixtures(ffo, ctx, arg_lists, args.threads, name)
            doc = {"workload": desc, "oracle_map_bound": args.map_bound,
                   "union_intervals": groups,
                   "generator": "tests/golden/make_workload_golden.py (CPU restatement, oracle/)",
                   "ranges": rows}
            with open(os.path.join(OUT, name), "w") as f:
                json.dump(doc, f, indent=0)
            print(f"wrote {name}: {len(rows)} ranges at {time.time() - t0:.0f} s",
                  file=sys.stderr, flush=True)


if __name__ == "__main__":
    main()
