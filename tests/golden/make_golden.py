"""Regenerates the golden fixtures of tests/golden/ from the REFERENCE program.

Runs oracle/_ref/ff_seg (the reference's reference/segmentedSieve.C compiled from its own
source by `make -C oracle ref`) in a fresh working directory per run (it refuses to run
where ffPlayground exists), normalises the two timing lines the way the reference's
scripts/verify.sh does, and writes:

  out_ff_seg_65536.txt   the 5..65536 leg (checked against goldens/SHA256SUMS of the
                         reference before it is written)
  legs.json              per leg: sha256 of the normalised stdout and the solution count,
                         taken from the reference's goldens/SHA256SUMS and scripts/verify.sh
  small_ranges.json      stdout of ff_seg for short ranges, partition-quirk ranges
                         (fewer than 62 sums) and limits that take main's two-call split
  pen_blocks.json        with --pen-blocks (only this file is written then): per leg, the
                         sha256 and line count of the solution block (the `) sum` lines) of
                         the reference's goldens/out_pen_<leg>.txt and out_pen2_<leg>.txt,
                         the second comparison of scripts/verify.sh:146-154
  dump_maps.json         with --dump-maps (only this file is written then): for argument
                         lists of `ff_seg --dump-map <file> ...`, the size and sha256 of the
                         dumped prime map and the stdout printed before the dump
  above_2_21.json        with --above-2-21 (only this file is written then): stdout of ff_seg
                         for short ranges with limits between 2.2M and 3.2M (above the legs)

Needs the reference checkout ($FF_REF_DIR, default ../reference beside the repository);
run from the repository root:
    python tests/golden/make_golden.py [--dump-maps | --pen-blocks | --above-2-21]
"""
import hashlib
import json
import math
import os
import random
import re
import subprocess
import tempfile

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
REF_BIN = os.path.join(ROOT, "oracle", "_ref", "ff_seg")
# the reference checkout: $FF_REF_DIR, by default a sibling of this repository
REF_TREE = os.environ.get("FF_REF_DIR", os.path.join(os.path.dirname(ROOT), "reference"))
OUT = os.path.join(ROOT, "tests", "golden")
NORM = re.compile(rb"(Prime|Freudenthal) time: [0-9]+")


def ff_seg(*args):
    d = tempfile.mkdtemp()
    try:
        out = subprocess.run([REF_BIN] + [str(a) for a in args], cwd=d, capture_output=True,
                             check=True).stdout
    finally:
        os.rmdir(d)
    return NORM.sub(rb"\1 time: N", out)


def pmap_limit(L):
    """isqrt64((mpv-2)<<2)<<1 for the map main sizes from L (no estimate branch at L >= 69)."""
    mgp = (L + 1) >> 1
    size = (max(((mgp * mgp) >> 2) + 2, 2) + 15) >> 4
    mpv = (size << 4) - 1
    return math.isqrt((mpv - 2) << 2) << 1


def main():
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref"], check=True)
    sums = {}
    with open(os.path.join(REF_TREE, "goldens", "SHA256SUMS")) as f:
        for line in f:
            h, name = line.split()
            sums[name] = h
    counts = {65536: 2357, 131072: 4776, 262144: 9163, 524288: 18408, 1048576: 35556,
              2097152: 71424}   # scripts/verify.sh:41-44
    legs = {str(L): {"sha256": sums[f"out_ff_seg_{L}.txt"], "solutions": c}
            for L, c in counts.items()}
    with open(os.path.join(OUT, "legs.json"), "w") as f:
        json.dump(legs, f, indent=1, sort_keys=True)

    leg = ff_seg(5, 65536)
    assert hashlib.sha256(leg).hexdigest() == legs["65536"]["sha256"], "65536 leg differs"
    with open(os.path.join(OUT, "out_ff_seg_65536.txt"), "wb") as f:
        f.write(leg)

    rnd = random.Random(20261203)
    cases = [[], [100], [3000], [5, 5], [4, 17], [0, 3], [7, 9], [43105, 43116], [40777, 40837],
             [1, 2627], [5, 1000], [99, 98]]
    for _ in range(120):
        s = rnd.randint(5, 200000)
        n = rnd.choice([0, 1, 2, 3, 5, 10, 30, 60, 61, 62, 63, 64, 100, 123, 200, 1000])
        cases.append([s, s + n])
    split = [L for L in range(69, 300000) if L > pmap_limit(L)]
    for L in rnd.sample(split, 40):
        cases.append([max(5, L - rnd.choice([0, 1, 2, 3, 10, 61, 62, 100, 1000])), L])
    for L in rnd.sample(split, 5):
        cases.append([L])
    out = []
    for c in cases:
        text = ff_seg(*c)
        out.append({"args": c, "sha256": hashlib.sha256(text).hexdigest(),
                    "text": text.decode() if len(text) < 20000 else None})
    with open(os.path.join(OUT, "small_ranges.json"), "w") as f:
        json.dump(out, f, indent=0)
    print(f"wrote {len(out)} small ranges, legs.json, out_ff_seg_65536.txt")


def dump_maps():
    """ff_seg --dump-map <file> <args> (reference/segmentedSieve.C:830-839, 883-897)."""
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref"], check=True)
    cases = [[], [100], [4, 17], [1000, 3000], [5, 65536], [5, 131072], [5, 262144],
             [300001, 300100]]
    out = []
    for c in cases:
        d = tempfile.mkdtemp()
        dump = os.path.join(d, "map.bin")
        try:
            res = subprocess.run([REF_BIN, "--dump-map", dump] + [str(a) for a in c], cwd=d,
                                 capture_output=True, check=True)
            with open(dump, "rb") as f:
                data = f.read()
        finally:
            if os.path.exists(dump):
                os.remove(dump)
            os.rmdir(d)
        out.append({"args": c, "bytes": len(data), "sha256": hashlib.sha256(data).hexdigest(),
                    "stdout": res.stdout.decode()})
    with open(os.path.join(OUT, "dump_maps.json"), "w") as f:
        json.dump(out, f, indent=1)
    print(f"wrote {len(out)} map dumps to dump_maps.json")


def pen_blocks():
    """Solution blocks of the pen/pen2 goldens (scripts/verify.sh:146-154: grep ') sum')."""
    out = {}
    for leg in (65536, 131072, 262144, 524288, 1048576):
        row = {}
        for kind in ("pen", "pen2", "ff_seg"):
            with open(os.path.join(REF_TREE, "goldens", f"out_{kind}_{leg}.txt"), "rb") as f:
                lines = [ln for ln in f.read().split(b"\n") if b") sum" in ln]
            block = b"".join(ln + b"\n" for ln in lines)
            row[kind] = {"sha256": hashlib.sha256(block).hexdigest(), "lines": len(lines)}
        out[str(leg)] = row
    with open(os.path.join(OUT, "pen_blocks.json"), "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
    print(f"wrote pen_blocks.json for {len(out)} legs")


def above_2_21():
    """ff_seg on short ranges whose limits lie above 2^21 (the served configuration's limits
    reach 2^22): each run sieves the reference's own map, limit^2/256 bytes (19 to 40 GB
    here), so the limits stop where this machine's memory does."""
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref"], check=True)
    cases = [[2200001, 2201000], [2500001, 2500300], [2750001, 2750150], [2999999, 3000100],
             [3100001, 3100063], [3199901, 3200000]]
    out = []
    for c in cases:
        text = ff_seg(*c)
        out.append({"args": c, "sha256": hashlib.sha256(text).hexdigest(), "text": text.decode()})
        print(f"ff_seg {c}: {text.count(b') sum =')} solutions", flush=True)
    with open(os.path.join(OUT, "above_2_21.json"), "w") as f:
        json.dump(out, f, indent=0)
    print(f"wrote {len(out)} ranges to above_2_21.json")


if __name__ == "__main__":
    import sys
    if "--above-2-21" in sys.argv:
        above_2_21()
    elif "--dump-maps" in sys.argv:
        dump_maps()
    elif "--pen-blocks" in sys.argv:
        pen_blocks()
    else:
        main()
