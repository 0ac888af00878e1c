"""SlidingTilePuzzleOptimized (Puzzles/SlidingTilePuzzleOptimized.cpp) on the
GPU: its packed index, its expand (kernel_sliding_tile_optimized,
Puzzles/SlidingPuzzleGpu.cu:211-269) and every search over it, against the
oracle (pinned to the reference class's own Parse / ToString, the Opt3x2 and
Opt4x4 known answers and the golden search counts, tests/test_oracle.py)."""
import random

import pytest

import oracle as O
import puzzlesearch_b200 as psb

pytestmark = pytest.mark.gpu

SHAPES = [(2, 2), (3, 2), (4, 2), (5, 2), (6, 2), (7, 2), (8, 2), (3, 3), (4, 3), (3, 4), (5, 3), (4, 4)]


def boards(spec, rng, n):
    """n random indexes of boards (and, every fourth, of the index space at large)."""
    N = O.info(spec)["indexes"]
    cells = spec[1] * spec[2]
    out = []
    while len(out) < n:
        i = rng.randrange(N)
        if len(out) % 4 and (i & 15) >= cells:
            continue
        out.append(i)
    return out


@pytest.mark.parametrize("w,h", SHAPES, ids=lambda v: str(v))
def test_expand_matches_oracle(w, h):
    spec = ["sliding_opt", w, h]
    p = psb.SlidingTilePuzzleOptimized(w, h)
    assert p.IndexesCount() == O.info(spec)["indexes"]
    rng = random.Random(w * 16 + h)
    parents = boards(spec, rng, 3000)
    ops = [rng.randrange(16) if k % 3 == 0 else 0 for k in range(len(parents))]
    assert tuple(p.Expand(parents, ops)) == tuple(O.expand(spec, parents, ops)), spec
    for i in parents[1::97]:
        try:
            s = O.to_string(spec, i)
        except ValueError:
            continue
        assert p.ToString(i) == s and p.Parse(s) == i


def test_parse_rejects_unsolvable_and_names():
    p = psb.SlidingTilePuzzleOptimized(3, 2)
    with pytest.raises(psb.PsbError):
        p.Parse("0 2 1 3 4 5")  # one inversion, odd width: the other parity class
    with pytest.raises(psb.PsbError):
        p.ToString(15)  # blank digit 15 names no 3x2 board
    assert p.Name() == "Sliding-Tile GPU Optimized (for 32-bit segment): 3 x 2"


@pytest.mark.parametrize("w,h", [(3, 2), (4, 2), (2, 4), (3, 3), (5, 2)], ids=lambda v: str(v))
@pytest.mark.parametrize("algo", ["two_bit", "three_bit", "frontier", "classic"])
def test_searches_bit_exact(w, h, algo):
    """Counts and final arrays of every in-memory search equal the oracle's,
    top-down and with bottom-up levels."""
    spec = ["sliding_opt", w, h]
    p = psb.SlidingTilePuzzleOptimized(w, h)
    start = p.Parse(" ".join(str(i) for i in range(w * h)))
    counts, fin = O.bfs(spec, algo, start, final=True)
    for direction in ("top_down", "auto"):
        r = psb.bfs(p, algo, start, final=True, direction=direction, window_bits=10)
        assert r["counts"] == counts and r["final"] == fin, (spec, algo, direction)


def test_legacy_golden_and_segmented(golden):
    """The reference's sliding-tile vectors over the optimized index: every
    full vector of SlidingPuzzleTests/TestFrontierSearch.cpp:19-72 up to 12
    cells (4x3: 319,334,400 indexes), the first 33 depths of 7x2 (:74-76);
    and the reference's DiskBasedOpt* bodies on SlidingTilePuzzleOptimized<5, 2>
    (PuzzleSearchTests.cpp:294-333, segmentBits 19 and 22) give ST5x2."""
    ran = 0
    for v in golden["legacy_sliding"]:
        w, h = v["puzzle"][1:]
        if w * h < 4 or w * h > 14 or (not v["full"] and w * h != 14):
            continue
        p = psb.SlidingTilePuzzleOptimized(w, h)
        start = p.Parse(v["start"])
        depth = 0 if v["full"] else len(v["counts"]) - 1
        for algo in ("two_bit", "three_bit") if w * h <= 12 else ("two_bit",):
            assert psb.bfs(p, algo, start, max_depth=depth)["counts"] == v["counts"], (v["source"], algo)
        ran += 1
    assert ran >= 10
    psb.lib().psb_release_cached_memory(0)
    st5x2 = [x for x in golden["search"] if x["puzzle"] == ["sliding", 5, 2] and x["full"]][0]["counts"]
    p = psb.SlidingTilePuzzleOptimized(5, 2)
    for sb in (19, 22):
        assert psb.bfs_segmented(p, p.Parse("0 1 2 3 4 5 6 7 8 9"), segment_bits=sb)["counts"] == st5x2


def test_7x2_equals_simple_index():
    """7x2 (14 cells): 13 segments of 2^32 indexes (14 GB of two-bit codes)
    against the Simple index's 14! (21.8 GB): two independent index schemes
    give the same per-depth counts, and half of 14! states in all."""
    o = psb.SlidingTilePuzzleOptimized(7, 2)
    a = psb.bfs(o, "two_bit", o.Parse(" ".join(str(i) for i in range(14))))["counts"]
    psb.lib().psb_release_cached_memory(0)
    s = psb.SlidingTilePuzzleSimple(7, 2)
    b = psb.bfs(s, "two_bit", s.Parse(" ".join(str(i) for i in range(14))))["counts"]
    psb.lib().psb_release_cached_memory(0)
    assert a == b and sum(a) == 87178291200 // 2
