"""The checks of the reference's golden-diff harness (scripts/verify.sh:120-154) against
ff_sieve, run the way that harness runs its GPU binary:
`<bin> --devices nvidia --gpu-search 5 <leg>`. Per leg: exit code 0, the solution count of
scripts/verify.sh:41-44, the whole timing-normalised stdout byte-equal to ff_seg's golden,
and the solution block equal to those of the pen and pen2 goldens (sha256 fixtures in
tests/golden/pen_blocks.json, made from the reference's goldens by make_golden.py)."""
import hashlib
import json
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "ff-gpu_b200", "bin", "ff_sieve")
NORM = re.compile(rb"(Prime|Freudenthal) time: [0-9]+")


def block(text):
    lines = [ln for ln in text.split(b"\n") if b") sum" in ln]
    return b"".join(ln + b"\n" for ln in lines), len(lines)


@pytest.fixture(scope="module")
def pens():
    with open(os.path.join(ROOT, "tests", "golden", "pen_blocks.json")) as f:
        return json.load(f)


def test_pen_goldens_agree_with_ff_seg(pens, golden):
    """The three goldens share one solution block per leg, and the 65536 leg's text here
    gives the same block."""
    for leg, row in pens.items():
        assert row["pen"] == row["pen2"] == row["ff_seg"], leg
        assert row["ff_seg"]["lines"] == golden["legs"][leg]["solutions"], leg
    b, n = block(golden["leg65536"])
    assert hashlib.sha256(b).hexdigest() == pens["65536"]["pen"]["sha256"] and n == 2357


def test_rejects_other_vendors(ffb):
    if not os.path.exists(CLI):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "ff-gpu_b200"), "-j8"], check=True)
    r = subprocess.run([CLI, "--devices", "amd", "5", "100"], capture_output=True)
    assert r.returncode == 1 and r.stdout == b""


@pytest.mark.gpu
@pytest.mark.parametrize("leg", [65536, 131072, 262144, 524288, 1048576])
def test_verify_sh_leg(leg, pens, golden):
    r = subprocess.run([CLI, "--devices", "nvidia", "--gpu-search", "5", str(leg)],
                       capture_output=True)
    assert r.returncode == 0, r.stderr[-2000:]
    out = NORM.sub(rb"\1 time: N", r.stdout)
    b, n = block(out)
    assert n == golden["legs"][str(leg)]["solutions"]
    assert hashlib.sha256(out).hexdigest() == golden["legs"][str(leg)]["sha256"]
    assert hashlib.sha256(b).hexdigest() == pens[str(leg)]["pen"]["sha256"]
    assert hashlib.sha256(b).hexdigest() == pens[str(leg)]["pen2"]["sha256"]
