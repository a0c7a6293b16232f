#!/usr/bin/env python
"""bench.py -- throughput of the plain GPU method on one range: sieve + Freudenthal search
over the odd sums 5..2^21 (`ff_sieve 5 2097152`), byte-identical to the reference.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One step = the whole job for the range: the prime map sieved on the device (the reference's
16 GiB map for values up to 274,877,906,959, extended to the 21.3 GiB that every probe of
the search needs so that none falls back to Miller-Rabin), then every odd sum of the range
searched, leaving one packed record per sum in HBM. `value` is odd sums per second of that
job on device-resident data (CUDA events on the launching stream, max over ranks); `e2e` is
the same metric through the public call a user makes (ffb_run: sieve, search, records copied
to the host, the text emitted in ff_seg's order), timed on the host clock. After the timed
steps the records are emitted as text and checked against the reference's SHA-256 of the
2^21 leg; a mismatch fails the run.

--impl reference times the reference program itself (ff_seg, compiled from the
reference's source) on the host cores: a bounded sample of the same job (see
reference_arm()).

With N > 1 ranks (torchrun), each rank sieves an equal slab of the map and an NCCL
all-gather assembles the whole map on every rank; the sums are split into cost-balanced
contiguous shards, one per GPU, searched with no exchange, and the records are gathered to
rank 0 (strong scaling: the job is fixed).

The side sections (batched, served, sieve sweep) run on rank 0 of a 1-GPU run; a compact
summary of every section is the last key of the JSON line.
"""
import argparse
import ctypes
import hashlib
import json
import math
import os
import re
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "ff-gpu_b200"))

LIMIT = 2097152
METRIC = "sums/sec byte-identical at sumLimit=2^21; served p50/p99 latency vs plain"
UNIT = "sums/s"
NORM = re.compile(rb"(Prime|Freudenthal) time: [0-9]+")
DEFAULT_TILE = 216 * 1024   # the sieve's shared-memory tile when the caller does not choose

# Integer operations per occurrence of each primitive of the reference search, counted as
# the 32-bit integer instructions (IMAD or ALU) an implementation needs:
#   isprime_calls  IsPrime from the map: parity test, bound compare, byte index, load, bit
#                  shift, mask                                                          6
#   splits         one (evenTerm, oddTerm) decomposition: b = s - o*2^k, o mod 3 and b mod 3
#                  (multiply-high), the 64-bit pair sums and the branch                 12
#   abop_calls     AllButOne... set-up: the 64-bit product, isqrt64, the first pair     18
#   trial_steps    one trial division of the product: a 64-bit by 32-bit quotient by
#                  reciprocal multiply and the exactness test                           10
#   divisors       one divisor pair: the 64-bit multiple, the 64-bit quotient product/d,
#                  the pair sum, the bound test and the list append                     18
# The counts per job come from the instrumented CPU restatement of the reference
# (tests/golden/search_work.json, made by tests/golden/make_search_work.py).
OP_COST = {"isprime_calls": 6, "splits": 12, "abop_calls": 18, "trial_steps": 10, "divisors": 18}

# DRAM bytes (read + written) per launch of each kernel on the 2^21 job, from one ncu capture
# of this bench's workload (dram__bytes_read.sum + dram__bytes_write.sum, one pass, full
# size; the command and the figures are in profiles/launches_ff_sieve_5_2097152.md).
NCU_TRAFFIC_2_21 = {"sieve_tiles": 0.03426e9 + 22.8534e9, "search_kernel": 463.360e9 + 2.707e9}


def odd_sums(lo, hi):
    return (hi - lo) // 2 + 1 if hi >= lo else 0


def norm(b):
    return NORM.sub(rb"\1 time: N", b)


def golden(name):
    with open(os.path.join(ROOT, "tests", "golden", name)) as f:
        return json.load(f)


# ---------------------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------------------
# roofline helpers
# ---------------------------------------------------------------------------------------
def hbm_peak():
    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peaks = json.load(f)
    except OSError:
        pass
    if "hbm_gbs" in peaks:
        return float(peaks["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
    return 6650.0, "fallback (6.65 TB/s, an earlier measurement on this pool)"


def odd_primes_upto(n):
    import numpy as np
    if n < 3:
        return np.zeros(0, dtype=np.int64)
    s = np.ones((n - 1) // 2, dtype=bool)   # index j -> 2j+3
    for j in range(int((math.isqrt(n) - 1) // 2)):
        if s[j]:
            p = 2 * j + 3
            s[(p * p - 3) // 2::p] = False
    return 2 * np.nonzero(s)[0].astype(np.int64) + 3


def sieve_marks(mpv, tile_bytes):
    """Shared-memory marks sieve_tiles makes for the map of values 0..mpv: the comb primes
    (47 <= p <= tile bits / 2048) mark every odd multiple from p^2, the larger primes the
    multiples p*k, k >= p, with k prime to 30 (the patterns cover 3..43)."""
    import numpy as np
    p = odd_primes_upto(math.isqrt(mpv))
    p = p[p >= 47]
    pcomb = tile_bytes * 8 // 2048
    comb = p[p <= pcomb]
    wheel = p[p > pcomb]
    n_comb = int(((mpv - comb * comb) // (2 * comb) + 1).sum())

    def coprime30_upto(x):   # #{1 <= k <= x : gcd(k, 30) = 1}
        r = x % 30
        small = np.zeros_like(x)
        for res in (1, 7, 11, 13, 17, 19, 23, 29):
            small += (r >= res)
        return 8 * (x // 30) + small
    kmax = mpv // wheel
    n_wheel = int((coprime30_upto(kmax) - coprime30_upto(wheel - 1)).sum())
    return n_comb, n_wheel


def search_ops():
    w = golden("search_work.json")["per_job"]
    return sum(w[k] * c for k, c in OP_COST.items()), w


# ---------------------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------------------
def ours(args, rank, world, dist):
    import torch
    import ffb200 as ffb
    from shard import gather_map, gather_records, map_slab, shard_bounds
    lib = ffb.load()
    dev = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(dev)
    peaks = ffb.measure_peaks(dev)
    g, _ = ffb.geometry(5, LIMIT)
    lo, hi = 5, LIMIT - 1                                  # odd sums of `ff_sieve 5 2097152`
    a, b = shard_bounds(lo, hi, world, rank)
    # the map: the reference's map, or the larger bound under which every probe of the
    # search is a map lookup (ffb_probe_bound; the output is the same either way,
    # Miller-Rabin being exact)
    mpv = max(g.maxPrimeMapValue, lib.ffb_probe_bound(hi))
    if args.map_bound:          # a smaller map: probes above it go to the Miller-Rabin variant
        mpv = min(mpv, (args.map_bound + 1) // 16 * 16 - 1)
    map_bytes = (mpv + 1 + 15) >> 4
    if world > 1:
        seg_lo, seg_hi, slab = map_slab(mpv, world, rank)
        d_map = torch.empty(world * slab + 256, dtype=torch.uint8, device="cuda")
    else:
        seg_lo, seg_hi, slab = 0, mpv + 1, 0
        d_map = torch.empty(map_bytes + 256, dtype=torch.uint8, device="cuda")
    nsums = odd_sums(a, b)
    d_rec = torch.empty(max(nsums, 1), dtype=torch.int64, device="cuda")
    stream = torch.cuda.Stream()
    sp = ctypes.c_void_p(stream.cuda_stream)

    def step(ev=None):
        with torch.cuda.stream(stream):
            if ev:
                ev[0].record(stream)
            if world > 1:
                if seg_hi > seg_lo:
                    assert lib.ffb_sieve_map_range_async(dev, seg_lo, seg_hi,
                                                         d_map.data_ptr() + (seg_lo >> 4), sp) == 0
                gather_map(dist, d_map, slab)
            else:
                assert lib.ffb_sieve_map_async(dev, mpv, d_map.data_ptr(), sp) == 0
            if ev:
                ev[1].record(stream)
            if a <= b:
                assert lib.ffb_search_async(dev, d_map.data_ptr(), mpv, a, b, d_rec.data_ptr(), sp) == 0
            if ev:
                ev[2].record(stream)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    assert ffb.take_errors(dev) == 0
    stats = (ctypes.c_uint64 * 2)()
    lib.ffb_search_stats(dev, stats, 1)
    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(args.steps)]
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    clocks = ClockSampler(dev)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    t0.record(stream)
    for k in range(args.steps):
        step(evs[k])
    t1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    if dist:
        dist.barrier()
    total_ms = t0.elapsed_time(t1)
    sieve_ms = statistics.mean(e[0].elapsed_time(e[1]) for e in evs)
    search_ms = statistics.mean(e[1].elapsed_time(e[2]) for e in evs)
    flags = ffb.take_errors(dev)
    if flags:
        raise RuntimeError(f"device error flags {flags:#x}")
    lib.ffb_search_stats(dev, stats, 1)
    probes_per_step = stats[0] // args.steps
    stage2_per_step = stats[1] // args.steps
    # the records of all shards on rank 0, emitted as ff_seg's text and checked against the
    # reference's hash of the leg (outside the timed region; a mismatch fails the run)
    if dist and world > 1:
        full = gather_records(dist, d_rec, lo, hi, world, rank)
    else:
        full = d_rec
    verified = None
    if rank == 0:
        import numpy as np
        text = ffb.emit((5, LIMIT), full.cpu().numpy().view(np.uint64), lo)
        want = golden("legs.json").get(str(LIMIT), {}).get("sha256")
        got = hashlib.sha256(norm(text)).hexdigest()
        if want is not None and got != want:
            raise RuntimeError(f"the job's text differs from the reference leg: sha256 {got}")
        verified = {"sha256": got, "equals_reference_leg": want is not None,
                    "solutions": text.count(b") sum =")}
    t = torch.tensor([total_ms, sieve_ms, search_ms], dtype=torch.float64, device="cuda")
    if dist:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    total_ms, sieve_ms, search_ms = t.tolist()
    ms_per_step = total_ms / args.steps
    job_sums = odd_sums(lo, hi)
    value = job_sums / (ms_per_step / 1e3)

    # e2e through the public call (rank 0, the whole job on one GPU)
    e2e = None
    if rank == 0 and not args.no_e2e:
        ctx = lib.ffb_context_create(dev)
        p, n = ctypes.c_void_p(), ctypes.c_size_t()
        for _ in range(max(1, args.warmup)):
            assert lib.ffb_run(ctx, 2, 5, LIMIT, ctypes.byref(p), ctypes.byref(n)) == 0
            lib.ffb_free(p)
        times = []
        text_len = 0
        for _ in range(args.steps):
            s = time.perf_counter()
            assert lib.ffb_run(ctx, 2, 5, LIMIT, ctypes.byref(p), ctypes.byref(n)) == 0
            times.append(time.perf_counter() - s)
            text_len = n.value
            lib.ffb_free(p)
        lib.ffb_context_destroy(ctx)
        e2e = {"value": job_sums / statistics.mean(times), "unit": UNIT,
               "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 8 * job_sums,
               "text_bytes_per_step": text_len, "ms_per_step": 1e3 * statistics.mean(times),
               "step_ms": [round(1e3 * t, 2) for t in times]}

    hbm, hbm_src = hbm_peak()
    # sieve: HBM bytes written once, and the shared-memory marks against the measured atomic
    # throughput (comb marks conflict-free, one-thread-per-prime marks on random banks)
    sieve_bytes = (seg_hi - seg_lo + 15) >> 4 if world > 1 else map_bytes
    n_comb, n_wheel = sieve_marks(mpv, DEFAULT_TILE)
    if world > 1:
        n_comb, n_wheel = n_comb / world, n_wheel / world
    mark_floor_s = n_comb / peaks["atomsConflictFreePerS"] + n_wheel / peaks["atomsRandomPerS"]
    sieve_kernel_s = sieve_ms / 1e3
    traffic_src = "ncu capture of this workload on one B200 (profiles/launches_ff_sieve_5_2097152.md)"
    known = LIMIT == 2097152 and not args.map_bound
    sieve_roof = {
        "kernel": "sieve_tiles", "bound": "hbm", "achieved": sieve_bytes / sieve_kernel_s / 1e9,
        "peak": hbm, "unit": "GB/s", "frac": sieve_bytes / sieve_kernel_s / 1e9 / hbm,
        "traffic": NCU_TRAFFIC_2_21["sieve_tiles"] / world if known else None,
        "traffic_source": traffic_src if known else None,
        "peak_source": hbm_src, "algorithmic_bytes": sieve_bytes,
        "marks": n_comb + n_wheel, "marks_per_s": (n_comb + n_wheel) / sieve_kernel_s,
        "marking_floor_ms": 1e3 * mark_floor_s,
        "frac_of_marking_floor": mark_floor_s / sieve_kernel_s,
        "note": "algorithmic bytes = bitmap bytes written once; marking floor = marks at the "
                "measured shared-memory atomicAnd rates (ffb_measure_peaks)"
                + ("; sieve_ms includes the NCCL all-gather of the map" if world > 1 else "")}
    ops, work = search_ops()
    if world > 1:
        share = (b * b - a * a) / (hi * hi - lo * lo) if a <= b else 0.0
        ops *= share
    search_roof = {
        "kernel": "search_kernel", "bound": "int_alu", "achieved": ops / (search_ms / 1e3),
        "peak": peaks["intOpsPerS"], "unit": "int ops/s",
        "frac": ops / (search_ms / 1e3) / peaks["intOpsPerS"],
        "traffic": NCU_TRAFFIC_2_21["search_kernel"] * (ops / search_ops()[0]) if known else None,
        "traffic_source": traffic_src if known else None,
        "peak_source": "measured (ffb_measure_peaks: integer multiply-add and ALU chains, "
                       "one IMAD to two ALU operations, whole GPU)",
        "algorithmic_ops": ops, "op_cost": OP_COST, "work_per_job": work,
        "stage1_probes": probes_per_step, "stage2_items": stage2_per_step,
        "note": "algorithmic ops = the reference search's primitive counts (instrumented CPU "
                "restatement) x the op_cost table; the kernel is bound by map-probe latency"}
    roof, other = (search_roof, sieve_roof) if search_ms >= sieve_ms else (sieve_roof, search_roof)

    def optional(fn, *a):
        # a side section that fails (e.g. a box with less free memory) is reported in its
        # place; the measured line above it is printed either way
        try:
            return fn(*a)
        except Exception as e:  # noqa: BLE001
            print(f"bench.py: {fn.__name__} failed: {e!r}", file=sys.stderr, flush=True)
            return {"error": repr(e)[:300]}

    side = rank == 0 and world == 1 and LIMIT == 2097152
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = optional(cpu_baseline, args)
    batched = None
    if side and not args.no_batched:
        batched = optional(batched_section, args, dev)
    served = None
    if side and args.served_requests > 0:
        del d_map
        torch.cuda.empty_cache()
        served = optional(served_section, args, dev)
    sweep = None
    if side and not args.no_sieve_sweep:
        sweep = optional(sieve_sweep_section, args, dev, hbm, peaks)
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "u32/u64 integer", "data": "synthetic",
            "config": {"workload": f"ff_sieve 5 {LIMIT}: prime map sieved on the device (values up "
                                   f"to {mpv}, {map_bytes / 2**30:.1f} GiB; reference mpv "
                                   f"{g.maxPrimeMapValue}) + search of {job_sums} odd sums",
                       "sum_start": 5, "sum_limit": LIMIT, "map_bytes": map_bytes,
                       "l2": "inputs larger than L2 (the map is rewritten every step)",
                       "parallelism": (f"map slabs + NCCL all-gather, sum shards x{world}"
                                       if world > 1 else "1 GPU")},
            "kernel_ms": {"sieve_tiles": sieve_ms, "search_kernel": search_ms},
            "roofline": roof, "roofline_other": other, "peaks": peaks, "verified": verified,
            "cpu_baseline": cpu, "e2e": e2e, "clocks": clk,
            "sieve_sweep": sweep, "batched": batched, "served": served,
            "gpu_launches": 3 * args.steps,   # list_primes, sieve_tiles, search_kernel per step
        }
        line["summary"] = summary(line)
        print(json.dumps(line), flush=True)


def summary(line):
    """The numbers of every section in a few keys (printed last in the line)."""
    def g(d, *ks):
        for k in ks:
            if not isinstance(d, dict) or k not in d:
                return None
            d = d[k]
        return d
    s = {"value": line["value"], "e2e": g(line, "e2e", "value"),
         "sieve_ms": g(line, "kernel_ms", "sieve_tiles"),
         "search_ms": g(line, "kernel_ms", "search_kernel"),
         "roofline_frac": g(line, "roofline", "frac"),
         "cpu_reference": g(line, "cpu_baseline", "value"),
         "cpu_reference_nproc_threads": g(line, "cpu_baseline", "threads_nproc_minus_1", "value")}
    b = line.get("batched") or {}
    if "value" in b:
        s["batched"] = {"requested_sums_per_s": b["value"],
                        "distinct_sums_per_s": b.get("distinct_sums_per_s"),
                        "vs_plain": b.get("vs_plain"), "cpu_sums_per_s": g(b, "cpu_baseline", "value")}
    v = line.get("served") or {}
    if "saturation" in v:
        sat = v["saturation"]
        s["served"] = {"requests": sat["requests"], "sums_per_s": sat["value"],
                       "vs_plain": v.get("vs_plain"), "p50_ms": sat["latency_ms"]["p50"],
                       "p99_ms": sat["latency_ms"]["p99"], "p999_ms": sat["latency_ms"]["p999"],
                       "loads": [{"load": r["load"], "p50_ms": r["latency_ms"]["p50"],
                                  "p99_ms": r["latency_ms"]["p99"], "p999_ms": r["latency_ms"]["p999"]}
                                 for r in v.get("rates", [])],
                       "cpu_sums_per_s": g(v, "cpu_baseline", "value")}
    w = line.get("sieve_sweep") or {}
    if "rows" in w:
        s["sieve_sweep"] = {r["N"]: {"tile": r["best"]["tile"], "GB/s": r["best"]["GB/s"],
                                     "cpu_GB/s": g(r, "cpu", "GB/s")} for r in w["rows"]}
    return s


# ---------------------------------------------------------------------------------------
# CPU baselines of the side configurations: the restatement oracle, multithreaded on the
# host's cores, on a bounded sample (test infrastructure used only as the CPU comparator)
# ---------------------------------------------------------------------------------------
def oracle_union_rate(arg_lists, windows=48, width=256):
    """Odd sums per second of the CPU restatement searching the union of the ranges' sums
    (each shared sum once, as the GPU batch does) with all host cores; measured on `windows`
    windows of `width` consecutive odd sums spread over the union by position and scaled.
    The map covers values up to 2^34 (Miller-Rabin above, exact); its sieve is not timed."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ffo
    spans = []
    for a, b in arg_lists:
        gg, _ = ffo.geometry(*ffo.parse_args(a, b))
        for f, l in ffo.schedule(gg.sum_start, gg.sum_limit, gg.max_prime_map_value):
            f |= 1
            l -= 1 - (l & 1)
            if f <= l:
                spans.append((f, l))
    spans.sort()
    union = []
    for f, l in spans:
        if union and f <= union[-1][1] + 2:
            union[-1][1] = max(union[-1][1], l)
        else:
            union.append([f, l])
    total = sum(odd_sums(f, l) for f, l in union)
    # window start positions: evenly spaced ordinals of the union's sums
    cum, acc = [], 0
    for f, l in union:
        cum.append(acc)
        acc += odd_sums(f, l)
    threads = os.cpu_count() or 1
    sampled, secs = 0, 0.0
    top = max(l for _, l in union)
    with ffo.Context(top + 2, map_bound=(1 << 34) - 1, threads=threads) as c:
        for i in range(windows):
            pos = (2 * i + 1) * total // (2 * windows)
            j = max(k for k in range(len(union)) if cum[k] <= pos)
            f, l = union[j]
            s0 = f + 2 * (pos - cum[j])
            s1 = min(l, s0 + 2 * (width - 1))
            t = time.perf_counter()
            c.eval_range(s0, s1, threads=threads)
            secs += time.perf_counter() - t
            sampled += odd_sums(s0, s1)
    return {"value": sampled / secs, "unit": "distinct sums/s", "cores": threads, "kind": "port",
            "union_sums": total, "est_union_s": total * secs / sampled,
            "sample": f"{windows} windows of {width} odd sums over the union of the ranges' sums "
                      f"({sampled} sums), oracle map to 2^34 + Miller-Rabin above, sieve untimed"}


# ---------------------------------------------------------------------------------------
# batched mode: 256 ranges (seed 0) against the plain method once per range
# ---------------------------------------------------------------------------------------
def range_sums(a, b):
    s = max(a | 1, 5)
    return (b - s) // 2 + 1 if b >= s else 0


def batched_section(args, dev):
    import ffb200 as ffb
    import workloads
    lib = ffb.load()
    ranges = workloads.batched_ranges(seed=0)
    sums = sum(range_sums(a, b) for a, b in ranges)
    t0 = time.perf_counter()
    batch = ffb.Batch(ranges, dev=dev, autotune=True)
    setup_s = time.perf_counter() - t0
    try:
        for _ in range(max(1, args.warmup)):
            batch.run()
        times, dev_ms = [], []
        for _ in range(args.steps):
            s = time.perf_counter()
            texts = batch.run()
            times.append(time.perf_counter() - s)
            info = batch.info()
            dev_ms.append(info["sieveMs"] + info["searchMs"])
        info = batch.info()
    finally:
        batch.close()
    fix = golden("batched_seed0.json")["ranges"]
    mismatches = sum(1 for r, t in zip(fix, texts) if hashlib.sha256(norm(t)).hexdigest() != r["sha256"])
    # the plain method, one ffb_run per range, on an evenly spaced sample of the ranges
    ctx = lib.ffb_context_create(dev)
    sample = ranges[::16]
    p, n = ctypes.c_void_p(), ctypes.c_size_t()
    plain_t, plain_sums = 0.0, 0
    try:
        assert lib.ffb_run(ctx, 2, sample[0][0], sample[0][1], ctypes.byref(p), ctypes.byref(n)) == 0
        lib.ffb_free(p)
        for a, b in sample:
            s = time.perf_counter()
            assert lib.ffb_run(ctx, 2, a, b, ctypes.byref(p), ctypes.byref(n)) == 0
            plain_t += time.perf_counter() - s
            lib.ffb_free(p)
            plain_sums += range_sums(a, b)
    finally:
        lib.ffb_context_destroy(ctx)
    t_batch = statistics.mean(times)
    value = sums / t_batch
    plain = plain_sums / plain_t
    cpu = None if args.no_cpu_baseline else oracle_union_rate(ranges)
    out = {"workload": "256 ranges from seed 0 (start U{5..2^21}, length floor(2^U[8,18]))",
           "value": value, "unit": "requested sums/s", "ms_per_batch": 1e3 * t_batch,
           "device_ms_per_batch": statistics.mean(dev_ms), "sums_per_batch": sums,
           "distinct_sums": info["sums"], "distinct_sums_per_s": info["sums"] / t_batch,
           "intervals": info["intervals"], "map_bytes": info["mapBytes"],
           "tuned": {k: info[k] for k in ("sieveTileBytes", "searchWarps", "searchChunk",
                                            "searchGroup") if k in info},
           "setup_s_incl_autotune": setup_s, "oracle_mismatches": mismatches,
           "plain_one_launch_per_range": {"value": plain, "unit": UNIT,
                                          "sample": f"{len(sample)} of the 256 ranges (every 16th)"},
           "vs_plain": value / plain}
    if cpu:
        cpu["est_batch_s"] = cpu["est_union_s"]
        cpu["value_requested"] = sums / cpu["est_union_s"]
        out["cpu_baseline"] = {**cpu, "value": cpu["value_requested"], "unit": "requested sums/s"}
        out["vs_cpu"] = value / cpu["value_requested"]
    return out


# ---------------------------------------------------------------------------------------
# sieve sweep: the map for N = 2^24, 2^28, 2^32 with the shared-memory tile swept
# ---------------------------------------------------------------------------------------
def sieve_sweep_section(args, dev, hbm, peaks):
    import torch
    import ffb200 as ffb
    lib = ffb.load()
    stream = torch.cuda.Stream()
    sp = ctypes.c_void_p(stream.cuda_stream)
    out = []
    for logn in (24, 28, 32):
        n = 1 << logn
        nbytes = (n + 1 + 15) >> 4
        d = torch.empty(nbytes + 256, dtype=torch.uint8, device="cuda")
        row = {"N": f"2^{logn}", "map_bytes": nbytes, "tiles": {}}
        for kb in (64, 96, 128, 160, 192, 216):
            for _ in range(3):
                assert lib.ffb_sieve_map_tiled_async(dev, n, d.data_ptr(), kb * 1024, sp) == 0
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            reps = 20 if logn < 32 else 5
            e0.record(stream)
            for _ in range(reps):
                assert lib.ffb_sieve_map_tiled_async(dev, n, d.data_ptr(), kb * 1024, sp) == 0
            e1.record(stream)
            e1.synchronize()
            ms = e0.elapsed_time(e1) / reps
            gbs = nbytes / (ms / 1e3) / 1e9
            nc, nw = sieve_marks(n, kb * 1024)
            row["tiles"][f"{kb}KB"] = {"ms": ms, "GB/s": gbs, "frac_of_hbm": gbs / hbm,
                                       "marks_per_s": (nc + nw) / (ms / 1e3)}
        best = max(row["tiles"].items(), key=lambda kv: kv[1]["GB/s"])
        row["best"] = {"tile": best[0], **best[1]}
        if not args.no_cpu_baseline:
            row["cpu"] = cpu_segment_fill(n)
        out.append(row)
        del d
    assert ffb.take_errors(dev) == 0
    return {"workload": "prime map for values up to N (list made on the device, sieve only); "
                        "a 2^24 or 2^28 map fits in L2, so only the 2^32 line is HBM-sized; "
                        "host launch overhead included (one call per sieve)", "rows": out}


def cpu_segment_fill(n):
    """The restated SegmentFill (oracle ffo_build_map: the map of values 0..n in byte-aligned
    chunks, one per thread) on all host cores."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ffo
    threads = os.cpu_count() or 1
    ffo.build_map(min(n, 1 << 20), threads=threads)   # warm-up
    t = time.perf_counter()
    ffo.build_map(n, threads=threads)
    s = time.perf_counter() - t
    nbytes = (n + 1 + 15) >> 4
    return {"s": s, "GB/s": nbytes / s / 1e9, "cores": threads, "kind": "port"}


# ---------------------------------------------------------------------------------------
# served mode: a Poisson stream of requests (seed 1) against the serving loop
# ---------------------------------------------------------------------------------------
def pct(xs, q):
    xs = sorted(xs)
    if not xs:
        return None
    k = min(len(xs) - 1, max(0, int(round(q * (len(xs) - 1)))))
    return xs[k]


def serve_stream(ffb, dev, reqs, budget, **cfg):
    """Submits reqs [(arrival_s, start, limit)] at their arrival times (arrival 0 = now) to a
    fresh server, drains the output on a second thread; returns per-request figures."""
    srv = ffb.Server(dev=dev, budget_bytes=budget, **cfg)
    try:
        got = {"bytes": 0, "chunks": 0, "done": 0, "failed": 0}

        def consume():
            while got["done"] + got["failed"] < len(reqs):
                c = srv.next(1000, keep_text=False)
                if c is None:
                    continue
                got["chunks"] += 1
                got["bytes"] += c[3]
                if c[2] == 1:
                    got["done"] += 1
                elif c[2] < 0:
                    got["failed"] += 1
        th = threading.Thread(target=consume, daemon=True)
        th.start()
        t0 = time.perf_counter()
        ids = []
        for t, a, b in reqs:
            d = t0 + t - time.perf_counter()
            if d > 0:
                time.sleep(d)
            ids.append(srv.submit(a, b))
        srv.drain()
        th.join(timeout=60)
        info = srv.info()
        ri = [srv.request_info(i) for i in ids]
    finally:
        srv.close()
    lat = [(r["doneUs"] - r["submitUs"]) / 1e3 for r in ri]
    first = [(r["firstChunkUs"] - r["submitUs"]) / 1e3 for r in ri]
    span_s = (max(r["doneUs"] for r in ri) - min(r["submitUs"] for r in ri)) / 1e6
    sums = sum(r["sums"] for r in ri)
    return {"requests": len(reqs), "sums": sums, "span_s": span_s, "value": sums / span_s,
            "requests_per_s": len(reqs) / span_s,
            "latency_ms": {"p50": pct(lat, 0.50), "p99": pct(lat, 0.99), "p999": pct(lat, 0.999),
                           "max": max(lat)},
            "first_chunk_ms": {"p50": pct(first, 0.50), "p99": pct(first, 0.99)},
            "failed": got["failed"], "text_bytes": got["bytes"], "chunks": got["chunks"],
            "launches": info["launches"], "sums_searched": info["sumsSearched"],
            "search_device_ms": info["searchMs"], "sieve_device_ms": info["sieveMs"],
            "map_bytes": info["mapBytes"], "map_max_value": info["mapMaxValue"],
            "max_queued": info["maxQueued"], "budget_bytes": info["budget"]["budget"],
            "stage1_probes": info["stage1Probes"], "stage2_items": info["stage2Items"],
            "mr_candidates": info["mrCandidates"], "mr_base2_passed": info["mrBase2Passed"],
            "backing_bytes": info["budget"]["backing"], "scratch_bytes": info["budget"]["scratch"]}


def served_section(args, dev):
    import ffb200 as ffb
    import workloads
    lib = ffb.load()
    n = args.served_requests
    budget = 8 << 30
    stream = workloads.served_requests(seed=1, n=10000, rate=1.0)
    base = stream[:n]
    # capacity: the first n requests at once
    sat = serve_stream(ffb, dev, [(0.0, a, b) for _, a, b in base], budget)
    cap_rps = sat["requests_per_s"]
    # offered loads on a prefix: the seed-1 arrival gaps rescaled to a fraction of capacity
    pre = stream[:min(n, args.served_load_requests)]
    runs = []
    for frac in args.served_loads:
        rate = frac * cap_rps
        reqs = [(t / rate, a, b) for t, a, b in pre]
        r = serve_stream(ffb, dev, reqs, budget)
        r["rate_per_s"] = rate
        r["load"] = frac
        runs.append(r)
    # the same prefix at a budget whose backing holds every probe of sums up to 2^22 (no
    # Miller-Rabin): what the 8 GiB cap costs
    full_budget = (((lib.ffb_probe_bound(1 << 22) + 1) >> 4) + (1 << 20) + (1 << 30) + (64 << 20))
    full_budget = (full_budget + (1 << 30) - 1) >> 30 << 30
    sat_full = serve_stream(ffb, dev, [(0.0, a, b) for _, a, b in pre], full_budget)
    # the plain method once per request (ffb_run: its own map sieved, then the search)
    ctx = lib.ffb_context_create(dev)
    k = max(1, n // args.served_plain)
    sample = base[k // 2::k]
    p, m = ctypes.c_void_p(), ctypes.c_size_t()
    plain_t, plain_sums, plain_lat = 0.0, 0, []
    try:
        assert lib.ffb_run(ctx, 2, 5, 65536, ctypes.byref(p), ctypes.byref(m)) == 0
        lib.ffb_free(p)
        for _, a, b in sample:
            s = time.perf_counter()
            assert lib.ffb_run(ctx, 2, a, b, ctypes.byref(p), ctypes.byref(m)) == 0
            dt = time.perf_counter() - s
            lib.ffb_free(p)
            plain_t += dt
            plain_lat.append(1e3 * dt)
            g, _ = ffb.geometry(a, b)
            plain_sums += sum((min(l, g.sumLimit) - (f | 1)) // 2 + 1
                              for f, l in ffb.schedule(g.sumStart, g.sumLimit, g.maxPrimeMapValue)
                              if (f | 1) <= l)
    finally:
        lib.ffb_context_destroy(ctx)
    # the plain method's time for the whole mix, estimated from the sample by request count
    # (each request pays its own sieve, so time is not proportional to sums): the sample is
    # every k-th request in arrival order, unbiased for the per-request mean time
    plain_total_s = plain_t * len(base) / len(sample)
    plain = sat["sums"] / plain_total_s
    out = {"workload": f"first {n} of the 10,000 seed-1 requests (limit U{{69..2^22}}, "
                       f"length floor(2^U[6,20]), start max(5, limit-length+1)) submitted at "
                       f"once (saturation); offered loads and the full-map budget on the first "
                       f"{len(pre)}, Poisson arrivals of the seed-1 stream rescaled to each rate",
           "budget": "8 GiB (computeBudget: f 0.90, cap 8 GiB)",
           "saturation": sat, "rates": runs,
           "saturation_full_map": {**{k: sat_full[k] for k in (
               "requests", "value", "requests_per_s", "span_s", "latency_ms", "map_bytes",
               "map_max_value", "budget_bytes", "mr_candidates")}},
           "plain_one_launch_per_request": {
               "value": plain, "unit": UNIT, "latency_ms_p50": pct(plain_lat, 0.5),
               "est_total_s": plain_total_s, "sample_sums_per_s": plain_sums / plain_t,
               "sample": f"every {k}th of the {n} requests ({len(sample)}), one ffb_run each; "
                         f"the mix's time = mean time per request x {n}"},
           "vs_plain": sat["value"] / plain}
    if not args.no_cpu_baseline:
        cpu = oracle_union_rate([(a, b) for _, a, b in base])
        cpu["value_requested"] = sat["sums"] / cpu["est_union_s"]
        out["cpu_baseline"] = {**cpu, "value": cpu["value_requested"], "unit": "requested sums/s"}
        out["vs_cpu"] = sat["value"] / cpu["value_requested"]
    return out


# ---------------------------------------------------------------------------------------
# the reference's CPU program
# ---------------------------------------------------------------------------------------
def ref_binary(threads=31):
    """ff_seg built from the reference source with THREADS = `threads` (oracle/_ref)."""
    exe = os.path.join(ROOT, "oracle", "_ref", "ff_seg" if threads == 31 else f"ff_seg_t{threads}")
    return exe if os.path.exists(exe) else None


# The sample: 8192 odd sums around 0.505 * 2^21, where the per-sum search cost equals the
# average over 5..2^21 (the cumulative cost grows as ~s^2.05); ff_seg's own timers give its
# sieve time for the sample's limit and its search time for the sample.
SAMPLE = (1073537, 1089919)


def run_ff_seg(exe, lo, hi):
    d = tempfile.mkdtemp()
    try:
        out = subprocess.run([exe, str(lo), str(hi)], cwd=d, capture_output=True, check=True).stdout
    finally:
        try:
            os.rmdir(d)
        except OSError:
            pass
    p = int(re.search(rb"Prime time: (\d+)", out).group(1))
    f = int(re.search(rb"Freudenthal time: (\d+)", out).group(1))
    return p, f, out


def map_bytes_for(limit):
    mgp = (limit + 1) >> 1
    size = (max(((mgp * mgp) >> 2) + 2, 2) + 15) >> 4
    return size


def ref_sample_value(exe):
    lo, hi = SAMPLE
    p_us, f_us, _ = run_ff_seg(exe, lo, hi)
    n = odd_sums(lo, hi)
    total = odd_sums(5, LIMIT - 1)
    # the full job's sieve scaled from the sample's map to the 2^21 map, charged per sum
    p_full = p_us * map_bytes_for(LIMIT) / map_bytes_for(hi)
    t = (f_us + p_full * n / total) / 1e6
    return n / t, {"prime_us": p_us, "freudenthal_us": f_us, "prime_full_est_us": p_full}


def cpu_baseline(args):
    exe = ref_binary(31)
    if not exe:
        return {"value": None, "unit": UNIT, "cores": 0, "kind": "reference",
                "sample": "reference binary not built (oracle/_ref)"}
    cores = os.cpu_count() or 1
    v, info = ref_sample_value(exe)
    out = {"value": v, "unit": UNIT, "cores": min(31, cores), "threads": 31, "host_cores": cores,
           "kind": "reference",
           "sample": f"ff_seg (THREADS=31, the reference's default) on odd sums {SAMPLE[0]}.."
                     f"{SAMPLE[1]} (8192 sums of average cost); its sieve time scaled to the "
                     f"2^21 map and charged per sum", **info}
    t = cores - 1
    exe_t = ref_binary(t)
    if exe_t and t != 31:
        v2, info2 = ref_sample_value(exe_t)
        out["threads_nproc_minus_1"] = {"value": v2, "threads": t, **info2}
    return out


def reference_arm(args, rank):
    if rank != 0:
        return
    exe = ref_binary(31)
    if not exe:
        print(json.dumps({"impl": "reference", "unavailable": "reference binary oracle/_ref/ff_seg "
                                                               "not built (needs the reference checkout)"}))
        return
    vals, infos = [], []
    for _ in range(args.warmup):
        ref_sample_value(exe)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        v, info = ref_sample_value(exe)
        vals.append(v)
        infos.append(info)
    wall = time.perf_counter() - t0
    value = statistics.mean(vals)
    cores = os.cpu_count() or 1
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 0,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * wall / args.steps,
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
        "dtype": "u32/u64 integer", "data": "synthetic",
        "config": {"workload": "ff_sieve 5 2097152 (bounded sample)", "sum_start": 5,
                   "sum_limit": LIMIT},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": min(31, cores),
                         "threads": 31, "host_cores": cores, "kind": "reference",
                         "sample": f"ff_seg (THREADS=31, reference source) on odd sums "
                                   f"{SAMPLE[0]}..{SAMPLE[1]}; sieve time scaled to the 2^21 map "
                                   f"and charged per sum", "last": infos[-1]},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def main():
    global LIMIT
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the public-call timing")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched-mode section")
    ap.add_argument("--no-sieve-sweep", action="store_true", help="skip the sieve sweep section")
    ap.add_argument("--served-requests", type=int, default=1000,
                    help="requests of the seed-1 served stream replayed at saturation (0: skip; "
                         "10000: the whole stream)")
    ap.add_argument("--served-load-requests", type=int, default=300,
                    help="requests of the stream replayed at each offered load")
    ap.add_argument("--served-loads", type=lambda v: [float(x) for x in v.split(",")],
                    default=[0.5, 0.8], help="offered loads, as fractions of the measured capacity")
    ap.add_argument("--served-plain", type=int, default=16,
                    help="requests timed through the plain method for the comparison")
    ap.add_argument("--map-bound", type=int, default=0,
                    help="cap the map at this value (probes above it take the Miller-Rabin "
                         "search variant); 0 = the bound covering every probe")
    ap.add_argument("--limit", type=int, default=2097152,
                    help="sumLimit of the job (2^21 for the reported line; smaller for profiling)")
    args = ap.parse_args()
    LIMIT = args.limit
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if args.impl == "reference":
        reference_arm(args, rank)
        return
    dist = None
    if world > 1:
        import datetime
        import torch
        import torch.distributed as tdist
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        dist = tdist
    try:
        ours(args, rank, world, dist)
    finally:
        if dist:
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
