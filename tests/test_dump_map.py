"""`--dump-map` (reference/segmentedSieve.C:830-839, 883-897): the prime map ff_seg builds
for a range, byte for byte. Fixtures: tests/golden/dump_maps.json, made by running the
reference program (make_golden.py --dump-maps). The CPU tests pin the header lines and the
oracle's map against the reference's dumps and check the command's argument errors; the
GPU tests check the device-built dumps through the C ABI and the ff_sieve command."""
import hashlib
import json
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "ff-gpu_b200", "bin", "ff_sieve")


@pytest.fixture(scope="module")
def dumps():
    with open(os.path.join(ROOT, "tests", "golden", "dump_maps.json")) as f:
        return json.load(f)


def test_headers_match_the_reference(ffb, dumps):
    for d in dumps:
        _, hdr = ffb.geometry(*d["args"])
        assert hdr.decode() == d["stdout"], d["args"]


def test_oracle_map_matches_the_reference_dump(oracle, ffb, dumps):
    for d in dumps:
        if d["bytes"] > 70_000_000:
            continue
        g, _ = ffb.geometry(*d["args"])
        m = oracle.build_map(g.maxPrimeMapValue)[: d["bytes"]]
        assert len(m) == d["bytes"] == (g.maxPrimeMapValue + 15) >> 4, d["args"]
        assert hashlib.sha256(m.tobytes()).hexdigest() == d["sha256"], d["args"]


def test_cli_dump_map_without_a_file(ffb):
    if not os.path.exists(CLI):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "ff-gpu_b200"), "-j8"], check=True)
    r = subprocess.run([CLI, "--dump-map"], capture_output=True)
    assert r.returncode == 256 - 6
    assert r.stdout == b"--dump-map requires a file argument.\n"


@pytest.mark.gpu
def test_device_dumps_match_the_reference(ffb, dumps):
    for d in dumps:
        data, hdr = ffb.map_dump(*d["args"])
        assert len(data) == d["bytes"], d["args"]
        assert hashlib.sha256(data).hexdigest() == d["sha256"], d["args"]
        assert hdr.decode() == d["stdout"], d["args"]


@pytest.mark.gpu
def test_cli_dump_map_file(ffb, dumps, tmp_path):
    d = next(x for x in dumps if x["args"] == [5, 65536])
    out = tmp_path / "map.bin"
    r = subprocess.run([CLI, "--dump-map", str(out), "5", "65536"], capture_output=True)
    assert r.returncode == 0, r.stderr
    assert r.stdout.decode() == d["stdout"]
    assert hashlib.sha256(out.read_bytes()).hexdigest() == d["sha256"]
    bad = subprocess.run([CLI, "--dump-map", str(tmp_path / "no" / "such" / "dir"), "100"],
                         capture_output=True)
    assert bad.returncode == 256 - 6
    assert b"Cannot open dump file" in bad.stdout
