"""Bottom-up levels (PSB_DIR_BOTTOM_UP / PSB_DIR_AUTO) against the oracle.

A bottom-up level scans the unvisited states and lets each probe its
neighbours for a frontier state, instead of expanding the frontier.  The
reference only expands top-down (Common/InMemoryThreeBitBFS.cpp,
InMemoryTwoBitBFS.cpp, InMemoryClassicBFS.cpp), so these tests require the
same per-depth counts and the same final arrays bit for bit, with every level
bottom-up, with the switch at several depths, and with the automatic choice."""
import functools
import math

import pytest

import oracle as O
import puzzlesearch_b200 as psb
from _puzzles import make

pytestmark = pytest.mark.gpu

BU_ALGOS = ["two_bit", "three_bit", "classic"]
CASES = [(["pancake", 8, 0], 0), (["pancake", 9, 0], 77), (["pancake", 10, 0], 12345), (["sliding", 3, 3], 0),
         (["sliding", 4, 2], 5), (["sliding", 2, 5], 1234), (["hanoi4", 8, 0], 0), (["hanoi4", 9, 0], 1000)]


@functools.lru_cache(maxsize=None)
def oracle_bfs(spec, algo, init):
    return O.bfs(list(spec), algo, init, final=True)




@pytest.mark.parametrize("case", CASES, ids=lambda c: f"{c[0][0]}{c[0][1]}x{c[0][2]}")
def test_every_level_bottom_up_bit_exact(case):
    spec, init = case
    p = make(spec)
    if spec[0] == "sliding":
        init = O.parse(spec, O.to_string(spec, init))  # any index; only its component is searched
    for algo in BU_ALGOS:
        counts, fin = oracle_bfs(tuple(spec), algo, init)
        r = psb.bfs(p, algo, init, final=True, direction="bottom_up")
        assert r["stats"]["bottom_up_levels"] == r["stats"]["levels"] > 0, (spec, algo)
        assert r["counts"] == counts, (spec, algo)
        assert r["final"] == fin, (spec, algo)


@pytest.mark.parametrize("ratio", [0.05, 0.5, 2.0, 8.0, 64.0])
def test_switch_depths_bit_exact(ratio):
    """The switch to bottom-up at different depths (bottom_up_ratio), with the
    active-window flags of sparse levels in use on both sides of it."""
    for spec, init in [(["pancake", 10, 0], 0), (["hanoi4", 9, 0], 0), (["sliding", 3, 3], 0)]:
        p = make(spec)
        for algo in BU_ALGOS:
            counts, fin = oracle_bfs(tuple(spec), algo, init)
            r = psb.bfs(p, algo, init, final=True, bottom_up_ratio=ratio)
            assert r["counts"] == counts, (spec, algo, ratio)
            assert r["final"] == fin, (spec, algo, ratio)


def test_auto_direction_switches_on_pancake():
    """13-pancake: the automatic choice runs the last dense levels bottom-up;
    counts match the top-down search and sum to 13!."""
    p = psb.PancakeSimple(13)
    auto = psb.bfs(p, "three_bit", 0)
    top = psb.bfs(p, "three_bit", 0, direction="top_down")
    assert auto["counts"] == top["counts"]
    assert sum(auto["counts"]) == math.factorial(13)
    assert 1 <= auto["stats"]["bottom_up_levels"] < auto["stats"]["levels"]
    assert auto["stats"]["children"] < top["stats"]["children"]
    p12 = psb.PancakeSimple(12)
    two = psb.bfs(p12, "two_bit", 0)
    assert two["counts"] == psb.bfs(p12, "two_bit", 0, direction="top_down")["counts"]
    assert two["stats"]["bottom_up_levels"] >= 1


def test_hanoi_symmetry_stays_top_down():
    """Hanoi with symmetry has non-canonical indexes, so it never goes bottom-up."""
    spec = ["hanoi4", 9, 1]
    p = make(spec)
    for algo in BU_ALGOS:
        r = psb.bfs(p, algo, 0, final=True, direction="bottom_up")
        assert r["stats"]["bottom_up_levels"] == 0
        counts, fin = oracle_bfs(tuple(spec), algo, 0)
        assert r["counts"] == counts and r["final"] == fin


def test_partial_last_window_and_max_depth():
    """Index spaces that are not a multiple of the window or of 64 (7! = 5040,
    5x2 = 10!), and max_depth cut-offs."""
    for spec in (["pancake", 7, 0], ["sliding", 5, 2]):
        p = make(spec)
        for algo in BU_ALGOS:
            counts = oracle_bfs(tuple(spec), algo, 0)[0]
            for md in (1, 3, len(counts) - 2):
                r = psb.bfs(p, algo, 0, max_depth=md, direction="bottom_up")
                assert r["counts"] == counts[:md + 1], (spec, algo, md)
