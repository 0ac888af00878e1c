"""The autotuner on the GPU: every candidate launch shape gives the same
counts (the tuner checks it), the pick is one of the candidates, and a
cached pick is reused without timing again."""
import random

import pytest

import puzzlesearch_b200 as psb
from puzzlesearch_b200 import autotune

pytestmark = pytest.mark.gpu


def test_engine_blocks_per_sm(tmp_path):
    rng = random.Random(3)
    items = []
    for _ in range(96):
        p = [psb.PancakeSimple(8), psb.PancakeSimple(9), psb.SlidingTilePuzzleSimple(3, 3)][rng.randrange(3)]
        start = rng.randrange(p.IndexesCount()) if p.Name().startswith("Pancake") else 0
        items.append((p, start))
    cache = autotune.Cache(str(tmp_path / "tune.json"))
    best, timings = autotune.tune_engine(items, candidates=(1, 2, 4), pool_bytes=1 << 30, cache=cache, key="mix")
    assert best in (1, 2, 4) and set(timings) == {1, 2, 4}
    again, t2 = autotune.tune_engine(items, candidates=(1, 2, 4), pool_bytes=1 << 30, cache=cache, key="mix")
    assert again == best and t2 == {}
    # the tuned grid gives the single-instance counts
    eng = psb.Engine(max_instances=8, pool_bytes=1 << 30, blocks_per_sm=best)
    for tag, (p, s) in enumerate(items[:8]):
        assert eng.add(p, s, tag)
    done = {}
    while len(done) < 8:
        eng.step(8)
        done.update(eng.poll())
    eng.close()
    for tag, (p, s) in enumerate(items[:8]):
        assert done[tag] == psb.bfs(p, "two_bit", s)["counts"]


def test_window_bits():
    p = psb.PancakeSimple(10)
    best, timings = autotune.tune_window_bits(p, "three_bit", candidates=[10, 12, 14])
    assert best in (10, 12, 14) and set(timings) == {10, 12, 14}
    assert all(ms > 0 for ms in timings.values())
    assert psb.device_name().startswith("NVIDIA")


def test_engine_window_offsets(tmp_path):
    """Both engine dimensions: every (blocks per SM, window offset) pair gives
    the single-instance counts (the tuner checks that all candidates agree),
    and a cached tuple pick comes back as a tuple."""
    rng = random.Random(5)
    items = []
    for _ in range(48):
        p = [psb.PancakeSimple(9), psb.SlidingTilePuzzleSimple(2, 5), psb.FourPegHanoiSimple(9)][rng.randrange(3)]
        items.append((p, rng.randrange(p.IndexesCount()) if not p.Name().startswith("Sliding") else 0))
    cands = [(2, -2), (2, 0), (4, 1), (1, -1)]
    cache = autotune.Cache(str(tmp_path / "tune.json"))
    best, timings = autotune.tune_engine(items, candidates=cands, pool_bytes=1 << 30, cache=cache, key="mix2")
    assert best in cands and set(timings) == set(cands)
    assert autotune.tune_engine(items, candidates=cands, cache=autotune.Cache(str(tmp_path / "tune.json")),
                                key="mix2") == (best, {})
    eng = psb.Engine(max_instances=8, pool_bytes=1 << 30, blocks_per_sm=best[0], window_bits_offset=best[1])
    for tag, (p, s) in enumerate(items[:8]):
        assert eng.add(p, s, tag)
    done = {}
    while len(done) < 8:
        eng.step(8)
        done.update(eng.poll())
    eng.close()
    for tag, (p, s) in enumerate(items[:8]):
        assert done[tag] == psb.bfs(p, "two_bit", s)["counts"]


def test_far_marks():
    best, timings = autotune.tune_far_marks(psb.PancakeSimple(10))
    assert best in ("none", "near", "all") and set(timings) == {"none", "near", "all"}


def test_threads_per_block():
    """The shape variants (128 / 256 / 512 threads per block) give the same
    counts, and the tuner picks one of them."""
    for algo in ("two_bit", "three_bit"):
        best, timings = autotune.tune_threads(psb.PancakeSimple(10), algo)
        assert best in (128, 256, 512) and set(timings) == {128, 256, 512}
    r = psb.bfs(psb.SlidingTilePuzzleSimple(3, 3), "two_bit", 0, threads=512, levels=True)
    assert r["stats"]["threads"] == 512
    with pytest.raises(psb.PsbError):
        psb.bfs(psb.PancakeSimple(8), "two_bit", 0, threads=300)
