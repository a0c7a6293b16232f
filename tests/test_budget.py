"""The device budget of the reference (source/budget.cpp:15-51) that the serving loop
admits requests against, checked against the known answers of
test/source/budget_selftest.cpp:133-178 (synthetic free-memory figures, no GPU)."""
import pytest

GiB = 1 << 30
HEADROOM = 64 << 20


def test_uncapped_budget(ffb):
    free = 34182397952                       # ~31.8 GiB free (budget_selftest.cpp:135)
    b = ffb.compute_budget(free, 0.90)
    assert b["freeUsed"] == int(0.90 * free)
    assert b["budget"] == b["freeUsed"]
    assert b["scratch"] == GiB                # min(0.15 x budget, 1 GiB)
    assert b["backing"] == ((b["budget"] - b["scratch"] - HEADROOM) // 4096) * 4096
    assert b["slabCount"] == b["backing"] // GiB
    assert b["cap"] == (1 << 64) - 1


def test_capped_budgets(ffb):
    free = 34182397952
    b = ffb.compute_budget(free, 0.90, cap=20 * GiB)
    assert b["budget"] == 20 * GiB
    assert b["backing"] == 20 * GiB - GiB - HEADROOM
    assert b["slabCount"] == 18
    b = ffb.compute_budget(free, 0.90, cap=8 * GiB)      # the serving loop's 8 GiB budget
    assert b["budget"] == 8 * GiB
    assert b["backing"] == 8 * GiB - GiB - HEADROOM
    assert b["slabCount"] == 6
    # two 8 GiB-capped devices cannot hold the 2^21 map (2^34 + 1 bytes); 20 GiB caps can
    assert 2 * b["backing"] < (1 << 34) + 1
    assert 2 * (20 * GiB - GiB - HEADROOM) >= (1 << 34) + 1


def test_small_budgets(ffb):
    b = ffb.compute_budget(1 << 40, 0.90, cap=80 << 20)
    assert b["scratch"] == int(0.15 * (80 << 20))
    assert b["backing"] == ((80 << 20) - b["scratch"] - HEADROOM) // 4096 * 4096
    b = ffb.compute_budget(1 << 40, 0.90, cap=64 << 20)  # nothing left after the headroom
    assert b["backing"] == 0
    b = ffb.compute_budget(1 << 40, 0.90, cap=8 * GiB, scratch=3 * GiB)
    assert b["scratch"] == 3 * GiB and b["backing"] == 5 * GiB - HEADROOM


def test_shrink_steps_toward_the_floor(ffb):
    free = 20 * GiB                           # budget_selftest.cpp:167
    s1 = ffb.compute_budget(free, 0.90, shrink=True)
    assert s1["fraction"] == pytest.approx(0.70, abs=1e-9)
    assert s1["backing"] < ffb.compute_budget(free, 0.90)["backing"]
    s2 = ffb.compute_budget(free, s1["fraction"], shrink=True)
    assert s2["fraction"] == pytest.approx(0.60, abs=1e-9)
    assert s2["backing"] < s1["backing"]
    s3 = ffb.compute_budget(free, s2["fraction"], shrink=True)
    assert s3["fraction"] == pytest.approx(0.55, abs=1e-9)
    floor = ffb.compute_budget(free, 0.50, shrink=True)
    assert floor["fraction"] == 0.50
    assert floor["backing"] == ffb.compute_budget(free, 0.50)["backing"]


def test_bad_fraction(ffb):
    with pytest.raises(ValueError):
        ffb.compute_budget(GiB, 0.0)
    with pytest.raises(ValueError):
        ffb.compute_budget(GiB, 1.5)
