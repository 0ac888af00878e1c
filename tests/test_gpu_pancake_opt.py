"""PancakeOptimized (Puzzles/PancakeOptimized.cpp:26-139) on the GPU: the
pancake moves in the reference's GPU pancake index, (rank / 12!) << 29 |
rank % 12! above 11 pancakes, whose offsets past 12! in each 2^29 block name
no permutation.  Expand equals the oracle's (pinned to the reference class in
tests/test_oracle.py); searches reach the same per-depth counts as
PancakeSimple, and final arrays equal the oracle's in this index."""
import math
import random

import pytest

import oracle as O
import puzzlesearch_b200 as psb

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [12, 13, 14, 16])
def test_expand_matches_oracle(n):
    p = psb.PancakeOptimized(n)
    rng = random.Random(n)
    parents = []
    while len(parents) < 2000:
        x = rng.randrange(p.IndexesCount())
        if (x & ((1 << 29) - 1)) < math.factorial(12):
            parents.append(x)
    want = O.expand(["pancake_opt", n, 0], parents)
    got = p.Expand(parents)
    assert got == want
    for x in parents[:20]:
        assert p.Parse(p.ToString(x)) == x
        assert p.ToString(x) == O.to_string(["pancake_opt", n, 0], x)


@pytest.mark.parametrize("algo", ["two_bit", "three_bit", "classic"])
def test_counts_equal_simple(algo):
    for n in (9, 11, 12):
        a = psb.bfs(psb.PancakeOptimized(n), algo, 0)["counts"]
        assert a == psb.bfs(psb.PancakeSimple(n), algo, 0)["counts"], (n, algo)


def test_final_arrays_small():
    for algo in ("two_bit", "three_bit"):
        counts, fin = O.bfs(["pancake_opt", 8, 0], algo, 0, final=True)
        r = psb.bfs(psb.PancakeOptimized(8), algo, 0, final=True)
        assert r["counts"] == counts and r["final"] == fin


def test_13_pancake_optimized_three_bit():
    """13 x 2^29 = 6,979,321,856 indexes, 13! of them permutations."""
    p = psb.PancakeOptimized(13)
    assert p.IndexesCount() == 13 << 29
    r = psb.bfs(p, "three_bit", 0)
    assert r["counts"] == psb.bfs(psb.PancakeSimple(13), "three_bit", 0)["counts"]
    assert sum(r["counts"]) == math.factorial(13)
    assert psb.bfs_segmented(psb.PancakeOptimized(12), 0, segment_bits=29)["counts"] == \
        psb.bfs(psb.PancakeSimple(12), "three_bit", 0)["counts"]


@pytest.mark.parametrize("n,sym", [(6, 1), (10, 1), (18, 1), (18, 0)])
def test_hanoi_optimized_expand(n, sym):
    """FourPegHanoiOptimized: Expand equals the oracle's (pinned to the
    reference class), on random parents, canonical or not."""
    p = psb.FourPegHanoiOptimized(n, bool(sym))
    rng = random.Random(n)
    parents = [rng.randrange(4 ** n) for _ in range(3000)]
    ops = [rng.randrange(16) if i % 3 else 0 for i in range(3000)]
    assert p.Expand(parents, ops) == O.expand(["hanoi4_opt", n, sym], parents, ops)


def test_hanoi_optimized_searches():
    for algo in ("two_bit", "three_bit", "frontier", "classic"):
        for sym in (0, 1):
            want = O.bfs(["hanoi4_opt", 9, sym], algo)[0]
            assert psb.bfs(psb.FourPegHanoiOptimized(9, bool(sym)), algo, 0)["counts"] == want, (algo, sym)
    r = psb.bfs(psb.FourPegHanoiOptimized(12, True), "two_bit", 0, restored=True)
    assert r["restored"] == O.bfs(["hanoi4", 12, 0], "two_bit")[0]
