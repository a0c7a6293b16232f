import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "ff-gpu_b200")
for p in (PKG, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def ffb():
    """The product's C ABI (built on demand; no fallback when the build is missing)."""
    if not os.path.exists(os.path.join(PKG, "lib", "libffb200.so")):
        subprocess.run(["make", "-s", "-C", PKG, "-j8"], check=True)
    import ffb200
    ffb200.load()
    return ffb200


@pytest.fixture(scope="session")
def oracle():
    import ffo
    ffo.load()
    return ffo


@pytest.fixture(scope="session")
def golden():
    import json
    g = os.path.join(ROOT, "tests", "golden")
    with open(os.path.join(g, "legs.json")) as f:
        legs = json.load(f)
    with open(os.path.join(g, "small_ranges.json")) as f:
        small = json.load(f)
    with open(os.path.join(g, "out_ff_seg_65536.txt"), "rb") as f:
        leg65536 = f.read()
    return {"legs": legs, "small": small, "leg65536": leg65536}
