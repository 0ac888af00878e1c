"""The autotuner's host logic (no GPU): the fastest candidate wins, a
candidate that changes the result is an error, and results are kept per
device and workload in a JSON file."""
import pytest

from puzzlesearch_b200 import autotune


def test_tune_picks_fastest_and_checks_results():
    times = {1: 0.30, 2: 0.20, 3: 0.25}
    best, timings = autotune.tune([1, 2, 3], lambda c: (times[c], "same counts"))
    assert best == 2 and timings == times
    with pytest.raises(AssertionError):
        autotune.tune([1, 2], lambda c: (0.1, [1, 8, 56] if c == 1 else [1, 8, 57]))


def test_cache_round_trip(tmp_path):
    path = str(tmp_path / "tune.json")
    c = autotune.Cache(path)
    assert c.get("NVIDIA B200 (sm_100, 148 SMs)", "batch") is None
    c.put("NVIDIA B200 (sm_100, 148 SMs)", "batch", 3)
    c.put("NVIDIA B200 (sm_100, 148 SMs)", "pancake13-3bit", 16)
    again = autotune.Cache(path)
    assert again.get("NVIDIA B200 (sm_100, 148 SMs)", "batch") == 3
    assert again.get("NVIDIA B200 (sm_100, 148 SMs)", "pancake13-3bit") == 16
    assert again.get("other GPU", "batch") is None


def test_engine_shapes_cover_grid_and_window():
    """The engine tuner's default candidates span both dimensions it tunes."""
    shapes = autotune.ENGINE_SHAPES
    assert {b for b, _ in shapes} == {1, 2, 3, 4}
    assert {w for _, w in shapes} == {-2, -1, 0, 1}
    assert len(shapes) == len(set(shapes)) == 16
