"""Serving loop (ffb_serve_*): requests continuously batched over a resident prime map.

Every request's text must be exactly ff_seg's for its arguments, whether it ran alone or
in a mix with others, and whether its probes were answered by the resident map or (above
a map cut short by a small budget) by Miller-Rabin.
"""
import hashlib
import re

import pytest

pytestmark = pytest.mark.gpu
NORM = re.compile(rb"(Prime|Freudenthal) time: [0-9]+")


def norm(b):
    return NORM.sub(rb"\1 time: N", b)


def sha(b):
    return hashlib.sha256(norm(b)).hexdigest()


def test_reference_binary_ranges_in_one_mix(ffb, golden):
    """All 177 reference-binary cases submitted at once (one mix), then a spread of them
    again one at a time on the drained server: identical texts, equal to ff_seg's."""
    cases = golden["small"]
    with ffb.Server(budget_bytes=8 << 30) as srv:
        ids = [srv.submit(*c["args"]) for c in cases]
        texts = srv.collect(ids)
        bad = [c["args"] for c, t in zip(cases, texts) if t is None or sha(t) != c["sha256"]]
        assert not bad, bad
        info = srv.info()
        assert info["completed"] == len(cases) and info["failed"] == 0
        assert info["launches"] >= 1 and info["sumsRequested"] >= info["sumsSearched"]
        for i in range(0, len(cases), 16):
            rid = srv.submit(*cases[i]["args"])
            (alone,) = srv.collect([rid])
            assert norm(alone) == norm(texts[i]), cases[i]["args"]
            ri = srv.request_info(rid)
            assert ri["state"] == 2 and ri["textBytes"] == len(alone)
            assert ri["bodyHash"] == srv.request_info(ids[i])["bodyHash"]


def test_small_budget_answers_above_the_map_by_miller_rabin(ffb, golden):
    """An 80 MiB budget leaves a 4 MiB map (values below 2^26): most probes of the larger
    cases go to Miller-Rabin, and the texts stay ff_seg's."""
    cases = [c for c in golden["small"] if len(c["args"]) == 2 and c["args"][1] >= 1 << 15]
    assert len(cases) >= 10
    with ffb.Server(budget_bytes=80 << 20) as srv:
        info = srv.info()
        b = info["budget"]
        assert b["budget"] == 80 << 20
        assert b["scratch"] == int(0.15 * (80 << 20))
        assert b["backing"] == ((b["budget"] - b["scratch"] - (64 << 20)) // 4096) * 4096
        ids = [srv.submit(*c["args"]) for c in cases]
        texts = srv.collect(ids)
        info = srv.info()
    assert info["mapMaxValue"] < 16 * b["backing"]
    top = max(c["args"][1] for c in cases)
    assert info["mapMaxValue"] < ffb.load().ffb_probe_bound(top)
    bad = [c["args"] for c, t in zip(cases, texts) if t is None or sha(t) != c["sha256"]]
    assert not bad, bad


def test_served_stream_identity_alone_vs_mix(ffb, oracle):
    """The first 120 requests of the seed-1 served stream submitted as one burst (many
    launches, each request sliced over several); ten of them again alone; the shortest
    ones also against the oracle."""
    import workloads
    reqs = workloads.served_requests(seed=1)[:120]
    with ffb.Server(budget_bytes=8 << 30, launch_work=16384) as srv:
        ids = [srv.submit(s, l) for _, s, l in reqs]
        mix = srv.collect(ids)
        assert all(t is not None for t in mix)
        infos = [srv.request_info(i) for i in ids]
        assert max(i["launches"] for i in infos) > 1          # requests were sliced
        for k in range(0, 120, 12):
            rid = srv.submit(reqs[k][1], reqs[k][2])
            (alone,) = srv.collect([rid])
            assert norm(alone) == norm(mix[k]), reqs[k]
    short = sorted(range(len(reqs)), key=lambda k: reqs[k][2] - reqs[k][1])[:6]
    for k in short:
        _, s, l = reqs[k]
        assert norm(mix[k]) == norm(oracle.run(s, l, map_bound=(1 << 30) - 1)), (s, l)


def test_served_stream_matches_oracle(ffb):
    """The first 300 requests of the seed-1 served stream (limits up to 2^22, 154 of them
    above 2^21) submitted as one burst under the 8 GiB budget (a map capped below the
    probes, Miller-Rabin above it): every request's streamed text equals the oracle's
    (tests/golden/served_seed1.json, made by tests/golden/make_workload_golden.py)."""
    import json
    import os
    import workloads
    with open(os.path.join(os.path.dirname(__file__), "golden", "served_seed1.json")) as f:
        fix = json.load(f)["ranges"]
    reqs = [(s, l) for _, s, l in workloads.served_requests(seed=1)[:len(fix)]]
    assert [tuple(r["args"]) for r in fix] == reqs and len(fix) >= 300
    assert sum(1 for _, l in reqs if l > 1 << 21) >= 100
    with ffb.Server(budget_bytes=8 << 30) as srv:
        ids = [srv.submit(s, l) for s, l in reqs]
        texts = srv.collect(ids)
        info = srv.info()
    assert info["failed"] == 0 and info["mapMaxValue"] < ffb.load().ffb_probe_bound(1 << 22)
    bad = [r["args"] for r, t in zip(fix, texts) if t is None or sha(t) != r["sha256"]]
    assert not bad, bad


def test_streamed_chunks_arrive_in_order(ffb):
    """A request sliced over many launches streams its chunks in order; the header leads."""
    with ffb.Server(budget_bytes=8 << 30, launch_work=2048) as srv:
        rid = srv.submit(1000001, 1100000)
        seqs, parts = [], []
        while True:
            got = srv.next(600000)
            assert got is not None
            r, seq, status, text = got
            assert r == rid and status >= 0
            seqs.append(seq)
            parts.append(text)
            if status == 1:
                break
        assert seqs == list(range(len(seqs))) and len(seqs) > 2
        assert parts[0].startswith(b"maxPrimeMapValue")
        whole = b"".join(parts)
        assert norm(whole) == norm(ffb.run(1000001, 1100000))


def test_rejected_requests(ffb):
    with ffb.Server(budget_bytes=1 << 30) as srv:
        with pytest.raises(ValueError):
            srv.submit(5, (1 << 25) + 2)
        rid = srv.submit(100, 50)           # the reference runs the one sum 101
        (t,) = srv.collect([rid])
        assert norm(t) == norm(ffb.run(100, 50))
