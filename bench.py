#!/usr/bin/env python
"""bench.py -- throughput of the plain GPU method on one range: sieve + Freudenthal search
over the odd sums 5..2^21 (`ff_sieve 5 2097152`), byte-identical to the reference.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One step = the whole job for the range: the prime map sieved on the device (the reference's
16 GiB map for values up to 274,877,906,959, extended to the 21.3 GiB that every probe of
the search needs so that none falls back to Miller-Rabin), then every odd sum of the range
searched, leaving one packed record per sum in HBM. `value` is odd sums per second of that job on
device-resident data (CUDA events on the launching stream, max over ranks); `e2e` is the
same metric through the public call a user makes (ffb_run: sieve, search, records copied
to the host, the text emitted in ff_seg's order), timed on the host clock.

--impl reference times the reference program itself (ff_seg, compiled from the
reference's source) on the host cores: a bounded sample of the same job (see
reference_arm()).

With N > 1 ranks (torchrun), the sums are split into cost-balanced contiguous shards, one
per GPU; each rank sieves the map its shard needs and searches its shard, and the records
are gathered to rank 0 over NCCL (strong scaling: the job is fixed).
"""
import argparse
import ctypes
import json
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


def odd_sums(lo, hi):
    return (hi - lo) // 2 + 1 if hi >= lo else 0


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
# our arm
# ---------------------------------------------------------------------------------------
def geometry_for(ffb, limit):
    g, _ = ffb.geometry(5, limit)
    return g


def ours(args, rank, world, dist):
    import torch
    import ffb200 as ffb
    from shard import shard_bounds, gather_records
    lib = ffb.load()
    dev = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(dev)
    g = geometry_for(ffb, LIMIT)
    lo, hi = 5, LIMIT - 1                                  # odd sums of `ff_sieve 5 2097152`
    a, b = shard_bounds(lo, hi, world, rank)
    # the map this shard's probes need: the reference's map for the shard's top sum, or the
    # larger bound under which every probe of the search is a map lookup (ffb_probe_bound;
    # the output is the same either way, Miller-Rabin being exact)
    gs = geometry_for(ffb, b + 1)
    mpv = max(gs.maxPrimeMapValue, lib.ffb_probe_bound(b))
    if args.map_bound:          # a smaller map: probes above it go to the Miller-Rabin variant
        mpv = min(mpv, (args.map_bound + 1) // 16 * 16 - 1)
    nsums = odd_sums(a, b)
    d_map = torch.empty(((mpv + 1 + 15) >> 4) + 64, dtype=torch.uint8, device="cuda")
    d_rec = torch.empty(max(nsums, 1), dtype=torch.int64, device="cuda")
    stream = torch.cuda.Stream()
    sp = ctypes.c_void_p(stream.cuda_stream)

    def step(ev=None):
        if ev:
            ev[0].record(stream)
        assert lib.ffb_sieve_map_async(dev, mpv, d_map.data_ptr(), sp) == 0
        if ev:
            ev[1].record(stream)
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
    # records of all shards to rank 0 (the exchange of the sharded job)
    if dist and world > 1:
        gather_records(dist, d_rec, lo, hi, world, rank)
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
               "text_bytes_per_step": text_len, "ms_per_step": 1e3 * statistics.mean(times)}

    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peaks = json.load(f)
    except OSError:
        pass
    hbm_peak = peaks.get("hbm_gbs", 6650.0)
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"
    map_bytes = (mpv + 1 + 15) >> 4
    # dominant kernel of the step
    if sieve_ms >= search_ms:
        achieved = map_bytes / (sieve_ms / 1e3) / 1e9
        roof = {"kernel": "sieve_tiles", "bound": "hbm", "achieved": achieved, "peak": hbm_peak,
                "unit": "GB/s", "frac": achieved / hbm_peak, "traffic": None,
                "algorithmic_bytes": map_bytes, "peak_source": peak_src,
                "note": "algorithmic bytes = bitmap bytes written once"}
    else:
        # search: each stage-1 probe (2^k + o*b - 2) reads one random 32-byte sector of the
        # multi-GB map; the records are written once. Algorithmic bytes per step =
        # 32 B x stage-1 probes + 8 B x sums (counted on the device in the timed steps).
        alg = 32 * probes_per_step + 8 * nsums
        achieved = alg / (search_ms / 1e3) / 1e9
        roof = {"kernel": "search_kernel", "bound": "hbm", "achieved": achieved, "peak": hbm_peak,
                "unit": "GB/s", "frac": achieved / hbm_peak, "traffic": None,
                "algorithmic_bytes": alg, "stage1_probes": probes_per_step,
                "stage2_items": stage2_per_step, "peak_source": peak_src,
                "note": "latency-bound integer kernel; see profiles/ for pipe utilisation"}
    def optional(fn, *a):
        # a side section that fails (e.g. a box with less free memory) is reported in its
        # place; the measured line above it is printed either way
        try:
            return fn(*a)
        except Exception as e:  # noqa: BLE001
            print(f"bench.py: {fn.__name__} failed: {e!r}", file=sys.stderr, flush=True)
            return {"error": repr(e)[:300]}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = optional(cpu_baseline, args)
    batched = None
    if rank == 0 and world == 1 and not args.no_batched and LIMIT == 2097152:
        batched = optional(batched_section, args, dev)
    served = None
    if rank == 0 and world == 1 and args.served_requests > 0 and LIMIT == 2097152:
        del d_map
        torch.cuda.empty_cache()
        served = optional(served_section, args, dev)
    sweep = None
    if rank == 0 and world == 1 and not args.no_sieve_sweep and LIMIT == 2097152:
        sweep = optional(sieve_sweep_section, args, dev, hbm_peak)
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
                       "parallelism": f"sum shards x{world}" if world > 1 else "1 GPU"},
            "kernel_ms": {"sieve_tiles": sieve_ms, "search_kernel": search_ms},
            "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "clocks": clk,
            "batched": batched, "served": served, "sieve_sweep": sweep,
            "gpu_launches": 2 * args.steps,
        }
        print(json.dumps(line), flush=True)


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
            batch.run()
            times.append(time.perf_counter() - s)
            info = batch.info()
            dev_ms.append(info["sieveMs"] + info["searchMs"])
        info = batch.info()
    finally:
        batch.close()
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
    value = sums / statistics.mean(times)
    plain = plain_sums / plain_t
    return {"workload": "256 ranges from seed 0 (start U{5..2^21}, length floor(2^U[8,18]))",
            "value": value, "unit": UNIT, "ms_per_batch": 1e3 * statistics.mean(times),
            "device_ms_per_batch": statistics.mean(dev_ms), "sums_per_batch": sums,
            "distinct_sums": info["sums"], "intervals": info["intervals"],
            "map_bytes": info["mapBytes"], "sieve_tile_bytes": info["sieveTileBytes"],
            "search_warps": info["searchWarps"], "setup_s_incl_autotune": setup_s,
            "plain_one_launch_per_range": {"value": plain, "unit": UNIT,
                                           "sample": f"{len(sample)} of the 256 ranges (every 16th)"},
            "vs_plain": value / plain}


# ---------------------------------------------------------------------------------------
# sieve sweep: the map for N = 2^24, 2^28, 2^32 with the shared-memory tile swept
# ---------------------------------------------------------------------------------------
def sieve_sweep_section(args, dev, hbm_peak):
    import torch
    import ffb200 as ffb
    lib = ffb.load()
    stream = torch.cuda.Stream()
    sp = ctypes.c_void_p(stream.cuda_stream)
    marks = {24: 1.53e7, 28: 2.66e8, 32: 4.55e9}   # odd multiples >= p^2 of odd primes <= sqrt(N)
    out = []
    for logn in (24, 28, 32):
        n = 1 << logn
        nbytes = (n + 1 + 15) >> 4
        d = torch.empty(nbytes + 64, dtype=torch.uint8, device="cuda")
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
            row["tiles"][f"{kb}KB"] = {"ms": ms, "GB/s": gbs, "frac_of_hbm": gbs / hbm_peak,
                                       "marks_per_s": marks[logn] / (ms / 1e3)}
        best = max(row["tiles"].items(), key=lambda kv: kv[1]["GB/s"])
        row["best"] = {"tile": best[0], **best[1]}
        out.append(row)
        del d
    return {"workload": "prime map for values up to N (host prime list to sqrt N, sieve only); "
                        "a 2^24 or 2^28 map fits in L2, so only the 2^32 line is HBM-sized; "
                        "host launch overhead included (one call per sieve)", "rows": out}


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
    base = workloads.served_requests(seed=1, n=10000, rate=1.0)[:n]
    # capacity: the whole prefix at once
    sat = serve_stream(ffb, dev, [(0.0, a, b) for _, a, b in base], budget)
    cap_rps = sat["requests_per_s"]
    # the same at a budget whose backing holds every probe of sums up to 2^22 (no
    # Miller-Rabin): what the 8 GiB cap costs
    full_budget = (((lib.ffb_probe_bound(1 << 22) + 1) >> 4) + (1 << 20) + (1 << 30) + (64 << 20))
    full_budget = (full_budget + (1 << 30) - 1) >> 30 << 30
    sat_full = serve_stream(ffb, dev, [(0.0, a, b) for _, a, b in base], full_budget)
    runs = []
    for frac in args.served_loads:
        rate = frac * cap_rps
        # the same requests, arrival gaps of the seed-1 stream rescaled to this rate
        reqs = [(t / rate, a, b) for t, a, b in base]
        r = serve_stream(ffb, dev, reqs, budget)
        r["rate_per_s"] = rate
        r["load"] = frac
        runs.append(r)
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
    sat_full_vs_plain = sat_full["value"] / plain
    return {"workload": f"first {n} of the 10,000 seed-1 requests (limit U{{69..2^22}}, "
                        f"length floor(2^U[6,20]), start max(5, limit-length+1)); Poisson "
                        f"arrivals of the seed-1 stream rescaled to each rate",
            "budget": "8 GiB (computeBudget: f 0.90, cap 8 GiB)",
            "saturation": sat, "rates": runs,
            "saturation_full_map": {**{k: sat_full[k] for k in (
                "value", "requests_per_s", "span_s", "latency_ms", "map_bytes", "map_max_value",
                "budget_bytes", "mr_candidates")}},
            "plain_one_launch_per_request": {
                "value": plain, "unit": UNIT, "latency_ms_p50": pct(plain_lat, 0.5),
                "est_total_s": plain_total_s, "sample_sums_per_s": plain_sums / plain_t,
                "sample": f"every {n // len(sample)}th of the {n} requests ({len(sample)}), one "
                          f"ffb_run each; the mix's time = mean time per request x {n}"},
            "vs_plain": sat["value"] / plain, "full_map_vs_plain": sat_full_vs_plain}


# ---------------------------------------------------------------------------------------
# the reference's CPU program
# ---------------------------------------------------------------------------------------
def ref_binary():
    """ff_seg built from the reference source with the largest THREADS <= cores-1."""
    cores = os.cpu_count() or 1
    best, best_t = None, 0
    for t in (31, 63, 127, 255):
        exe = os.path.join(ROOT, "oracle", "_ref", "ff_seg" if t == 31 else f"ff_seg_t{t}")
        if os.path.exists(exe) and (t <= cores - 1 or best is None):
            if t > best_t:
                best, best_t = exe, t
    return best, best_t


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
    import math
    mgp = (limit + 1) >> 1
    size = (max(((mgp * mgp) >> 2) + 2, 2) + 15) >> 4
    return size


def ref_sample_value(exe, threads):
    lo, hi = SAMPLE
    p_us, f_us, _ = run_ff_seg(exe, lo, hi)
    n = odd_sums(lo, hi)
    total = odd_sums(5, LIMIT - 1)
    # the full job's sieve scaled from the sample's map to the 2^21 map, charged per sum
    p_full = p_us * map_bytes_for(LIMIT) / map_bytes_for(hi)
    t = (f_us + p_full * n / total) / 1e6
    return n / t, {"prime_us": p_us, "freudenthal_us": f_us, "prime_full_est_us": p_full}


def cpu_baseline(args):
    exe, threads = ref_binary()
    if not exe:
        return {"value": None, "unit": UNIT, "cores": 0, "kind": "reference",
                "sample": "reference binary not built (oracle/_ref)"}
    v, info = ref_sample_value(exe, threads)
    return {"value": v, "unit": UNIT, "cores": min(threads, os.cpu_count() or threads),
            "threads": threads, "host_cores": os.cpu_count(), "kind": "reference",
            "sample": f"ff_seg (THREADS={threads}) on odd sums {SAMPLE[0]}..{SAMPLE[1]} "
                      f"(8192 sums of average cost); its sieve time scaled to the 2^21 map and "
                      f"charged per sum", **info}


def reference_arm(args, rank):
    if rank != 0:
        return
    exe, threads = ref_binary()
    if not exe:
        print(json.dumps({"impl": "reference", "unavailable": "reference binary oracle/_ref/ff_seg "
                                                               "not built (needs the reference checkout)"}))
        return
    vals, infos = [], []
    for _ in range(args.warmup):
        ref_sample_value(exe, threads)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        v, info = ref_sample_value(exe, threads)
        vals.append(v)
        infos.append(info)
    wall = time.perf_counter() - t0
    value = statistics.mean(vals)
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 0,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * wall / args.steps,
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
        "dtype": "u32/u64 integer", "data": "synthetic",
        "config": {"workload": "ff_sieve 5 2097152 (bounded sample)", "sum_start": 5,
                   "sum_limit": LIMIT},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": min(threads, os.cpu_count() or threads),
                         "threads": threads, "host_cores": os.cpu_count(), "kind": "reference",
                         "sample": f"ff_seg (THREADS={threads}, reference source) on odd sums "
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
    ap.add_argument("--served-requests", type=int, default=300,
                    help="requests of the seed-1 served stream to replay (0: skip)")
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
