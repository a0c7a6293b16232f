"""Host side of the product without a GPU: the library loads and exports every symbol of
include/*.h, and its planning code (geometry, headers, schedule, line format) agrees with
the oracle and with the reference binary's outputs."""
import os
import random
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_c_symbols():
    """Function names declared at file scope of include/ffb200.h (extern "C" block)."""
    with open(os.path.join(ROOT, "include", "ffb200.h")) as f:
        text = f.read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = set()
    for m in re.finditer(r"^[A-Za-z_][\w\s\*]*?\b([A-Za-z_]\w*)\s*\(", text, flags=re.M):
        name = m.group(1)
        if name not in {"typedef", "if", "sizeof"} and not text[m.start():m.end()].startswith("typedef"):
            names.add(name)
    return names


def test_library_exports_every_declared_symbol(ffb):
    lib = ffb.load()
    names = declared_c_symbols()
    # the binding declares exactly the header's functions (29 entry points)
    assert names == set(ffb.SIGNATURES), names ^ set(ffb.SIGNATURES)
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_cxx_symbols_exported():
    out = subprocess.run(["nm", "-DC", os.path.join(ROOT, "ff-gpu_b200", "lib", "libffb200.so")],
                         capture_output=True, text=True, check=True).stdout
    for sym in ("GpuPrime::IsPrime(unsigned long) const", "GpuPrime::AskMillerRabin(unsigned long) const",
                "PrintOutputTags(GpuPrime const&, unsigned long, bool)",
                "FormatGpuSearchResult(GpuPrime const&, unsigned int, GpuRecord const&)",
                "GpuSearchEmit(GpuPrime const&, GpuRecord const*, unsigned int)"):
        assert sym in out, sym


def test_gpu_record_layout(ffb):
    import ctypes
    assert ctypes.sizeof(ffb.GpuRecord) == 32
    assert ffb.GpuRecord.low.offset == 8 and ffb.GpuRecord.tag.offset == 24


def test_getters_without_device(ffb):
    # no GPU here: every getter reports "no device" instead of failing
    lib = ffb.load()
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is visible")
    for g in ("SieveSlabGetLaunchFn_sm_100a", "SieveSlabEngineGetLaunchFn_sm_100a",
              "SievePoolGet_sm_100a", "SearchKernelGetLaunchFn_sm_100a",
              "SieveSlabGetLaunchFn_gfx1201", "SearchKernelGetLaunchFn_gfx1201"):
        assert getattr(lib, g)(0) is None
    assert lib.GpuSearchLaunch(0, b"amd", None, 0, 5, 5, None, None) == -1


def _limits():
    rnd = random.Random(11)
    ls = [5, 6, 7, 17, 20, 68, 69, 100, 2627, 65536, 65537, 131071, 2097152, 4194304,
          4834000, 4900000, 6000000, 16777216, 33554432]
    ls += [rnd.randint(5, 1 << 25) for _ in range(300)]
    return ls


def test_geometry_headers_match_oracle(ffb, oracle):
    for L in _limits():
        g, hdr = ffb.geometry(5, L)
        og, ohdr = oracle.geometry(5, L)
        assert hdr == ohdr, L
        assert g.maxPrimeMapValue == og.max_prime_map_value
        assert g.pmapSumLimit == og.pmap_sum_limit


def test_argument_handling_matches_oracle(ffb, oracle):
    for args in [(), (100,), (6, 100), (99, 98), (0, 3), (1, 2627), (4, 17)]:
        g, _ = ffb.geometry(*args)
        assert (g.sumStart, g.sumLimit) == oracle.parse_args(*args), args


def test_schedule_matches_oracle(ffb, oracle):
    rnd = random.Random(5)
    cases = [(5, L) for L in (5, 7, 17, 66, 67, 68, 100, 2627, 65536, 2097152)]
    for _ in range(2000):
        s = rnd.randint(5, 1 << 22) | 1
        n = rnd.choice([0, 1, 2, 5, 30, 61, 62, 63, 64, 124, 1000, rnd.randint(0, 1 << 20)])
        cases.append((s, s + n))
    for s, l in cases:
        mpv = oracle.geometry(s, l)[0].max_prime_map_value
        assert ffb.schedule(s, l, mpv) == oracle.schedule(s, l, mpv), (s, l)


def test_format_line_matches_oracle(ffb, oracle):
    rnd = random.Random(3)
    with oracle.Context(1 << 20, map_bound=1 << 20) as ctx:
        lib = oracle.load()
        import ctypes
        buf = ctypes.create_string_buffer(256)
        terms = [4, 8, 16, 512, 1024, 2 ** 20, 3, 9, 13, 15, 21, 1048573, 999983]
        terms += [rnd.randint(3, 1 << 20) for _ in range(500)]
        for i in range(2000):
            a, b = rnd.choice(terms), rnd.choice(terms)
            lo, hi = min(a, b), max(a, b)
            count = rnd.choice([1, 9, 10, 999, 71424, 1234567])
            n = lib.ffo_format_line(ctx.h, count, lo + hi, lo, hi, buf, len(buf))
            want = buf.raw[:n]
            got = ffb.format_line(count, lo + hi, lo, hi, ctx.is_prime(lo), ctx.is_prime(hi))
            assert got == want, (lo, hi)


def test_golden_lines_reformat(ffb, golden):
    # every solution line of the 65536 leg re-created by the product's formatter
    for line in golden["leg65536"].splitlines(keepends=True):
        m = re.match(rb"\s*(\d+)\) sum =\s*(\d+), product =\s*\d+,  low term =\s*(\d+)(.*?)high term =\s*(\d+)(.*)\n",
                     line)
        if not m:
            continue
        got = ffb.format_line(int(m[1]), int(m[2]), int(m[3]), int(m[5]),
                              b"prime" in m[4], b"prime" in m[6])
        assert got == line


def test_cli_usage():
    exe = os.path.join(ROOT, "ff-gpu_b200", "bin", "ff_sieve")
    r = subprocess.run([exe, "--help"], capture_output=True, text=True)
    assert r.returncode == 0 and "usage" in r.stderr
    r = subprocess.run([exe, "--bogus"], capture_output=True, text=True)
    assert r.returncode == 1
