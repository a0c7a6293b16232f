"""Batched mode (ffb_batch_*): many ranges in one sieve + one work-queue search launch,
replayed from a CUDA graph. Each range's text must be exactly ff_seg's for that range."""
import hashlib
import re

import pytest

pytestmark = pytest.mark.gpu
NORM = re.compile(rb"(Prime|Freudenthal) time: [0-9]+")


def norm(b):
    return NORM.sub(rb"\1 time: N", b)


def as_pair(args):
    """ff_seg's argument forms as the (start, limit) pair with the same meaning."""
    if len(args) == 0:
        return 5, 2627
    if len(args) == 1:
        return 5, args[0]
    return args[0], args[1]


def test_reference_binary_ranges_as_one_batch(ffb, golden):
    cases = golden["small"]
    with ffb.Batch([as_pair(c["args"]) for c in cases], autotune=False) as b:
        texts = b.run()
        info = b.info()
    bad = [c["args"] for c, t in zip(cases, texts)
           if hashlib.sha256(norm(t)).hexdigest() != c["sha256"]]
    assert not bad, bad
    assert info["ranges"] == len(cases) and info["intervals"] >= 1
    assert ffb.take_errors(0) == 0


def test_batched_config_matches_oracle(ffb):
    """All 256 ranges of the batched configuration (seed 0), run as one batch and replayed
    from the graph, each equal to the oracle's text for that range (tests/golden/
    batched_seed0.json, made by tests/golden/make_workload_golden.py); a spread of them also
    equal to the single-range pipeline."""
    import json
    import os
    import workloads
    ranges = workloads.batched_ranges(seed=0)
    assert len(ranges) == 256
    with open(os.path.join(os.path.dirname(__file__), "golden", "batched_seed0.json")) as f:
        fix = json.load(f)["ranges"]
    assert [tuple(r["args"]) for r in fix] == ranges
    with ffb.Batch(ranges, autotune=True) as b:
        first = b.run()
        second = b.run()          # graph replay
        info = b.info()
    assert len(first) == 256
    assert [norm(t) for t in first] == [norm(t) for t in second]
    bad = [r["args"] for r, t in zip(fix, first) if hashlib.sha256(norm(t)).hexdigest() != r["sha256"]]
    assert not bad, bad
    ctx = ffb.load().ffb_context_create(0)
    try:
        for i in range(0, 256, 51):        # a spread against the single-range pipeline
            assert norm(first[i]) == norm(ffb.run(*ranges[i], ctx=ctx)), ranges[i]
    finally:
        ffb.load().ffb_context_destroy(ctx)
    assert info["autotuned"] in (1, 2)
    assert info["sieveTileBytes"] in {k * 1024 for k in (64, 96, 128, 160, 192, 216)}
    assert info["searchWarps"] in (4, 8, 16)
    assert info["searchGroup"] in (1, 2, 4)
    assert info["searchChunk"] in ((16, 32, 64) if info["searchGroup"] == 1 else (32 * info["searchGroup"],))
    assert info["sieveMs"] > 0 and info["searchMs"] > 0      # replayed graph timestamps
    assert ffb.take_errors(0) == 0
