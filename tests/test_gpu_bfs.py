"""GPU parity of the in-memory searches (psb_bfs) against the reference's golden
vectors, the reference's own runs (oracle/_ref output committed as fixtures)
and the oracle's final bit arrays.  Integer work: bit-exact.

The reference varies segment sizes and thread counts to test its segmented
drivers (PuzzlesTests/PuzzleSearchTests.cpp:133-333); the equivalent knob here
is the thread-block window size, varied in test_window_sizes_agree."""
import math

import pytest

import oracle as O
import puzzlesearch_b200 as psb
from _puzzles import make

pytestmark = pytest.mark.gpu

ALGOS = ["two_bit", "three_bit", "frontier", "classic"]




def algos_for(p):
    return [a for a in ALGOS if a != "frontier" or p.OperatorsCount() <= 4]


def test_search_vectors(golden):
    """PuzzlesTests/PuzzleSearchTests.cpp vectors through every in-memory algorithm."""
    ran = 0
    for v in golden["search"]:
        p = make(v["puzzle"])
        if p.IndexesCount() > 1 << 34:
            continue
        init = 0 if v["start"] is None else p.Parse(v["start"])
        max_depth = 0 if v["full"] else len(v["counts"]) - 1
        for algo in algos_for(p):
            if not v["full"] and algo in ("frontier", "classic"):
                continue
            got = psb.bfs(p, algo, init, max_depth=max_depth)["counts"]
            assert got == v["counts"], (v["puzzle"], algo, v["source"])
            ran += 1
    assert ran >= 20


def test_legacy_sliding_vectors(golden):
    """SlidingPuzzleTests/TestFrontierSearch.cpp full vectors (up to 12 tiles)."""
    ran = 0
    for v in golden["legacy_sliding"]:
        p = make(v["puzzle"])
        if not v["full"] or p.IndexesCount() > 10 ** 9:
            continue
        init = p.Parse(v["start"])
        for algo in ("two_bit", "three_bit"):
            got = psb.bfs(p, algo, init)["counts"]
            assert got == v["counts"], (v["puzzle"], v["start"], algo, v["source"])
        ran += 1
    assert ran >= 9


def test_sliding_3x4_equals_4x3_golden(golden):
    """The 3x4 board is the transpose of the reference's 4x3 golden
    (SlidingPuzzleTests/TestFrontierSearch.cpp:70-72): same per-depth counts."""
    v = [x for x in golden["legacy_sliding"] if x["puzzle"] == ["sliding", 4, 3]][0]
    p = psb.SlidingTilePuzzleSimple(3, 4)
    r = psb.bfs(p, "two_bit", p.Parse("0 1 2 3 4 5 6 7 8 9 10 11"))
    assert r["counts"] == v["counts"]
    assert sum(r["counts"]) == math.factorial(12) // 2


def test_reference_runs(golden):
    """Per-depth counts of the reference's own InMemory BFS runs."""
    for run in golden["ref_runs"]:
        p = make(run["puzzle"])
        got = psb.bfs(p, run["algo"], p.Parse(run["start"]))["counts"]
        assert got == run["counts"], (run["puzzle"], run["algo"], run["start"])


FINAL_CASES = [(["sliding", 3, 3], 0), (["sliding", 4, 2], 5), (["pancake", 8, 0], 0), (["pancake", 9, 0], 77),
               (["hanoi4", 8, 0], 0), (["hanoi4", 9, 1], 0), (["sliding", 2, 5], 1234)]


@pytest.mark.parametrize("case", FINAL_CASES, ids=lambda c: f"{c[0][0]}{c[0][1]}x{c[0][2]}")
def test_final_arrays_bit_exact(case):
    spec, init = case
    p = make(spec)
    if spec[0] == "sliding":
        init = O.parse(spec, O.to_string(spec, init))  # any index; only its component is searched
    for algo in algos_for(p):
        r = psb.bfs(p, algo, init, final=True)
        counts, fin = O.bfs(spec, algo, init, final=True)
        assert r["counts"] == counts, (spec, algo)
        assert r["final"] == fin, (spec, algo)


def test_window_sizes_agree():
    p = psb.PancakeSimple(10)
    expect = O.bfs(["pancake", 10, 0], "three_bit")[0]
    for wb in (10, 12, 14, 16, 18):
        assert psb.bfs(p, "three_bit", 0, window_bits=wb)["counts"] == expect, wb
        assert psb.bfs(p, "two_bit", 0, window_bits=wb)["counts"] == expect, wb
    h = psb.FourPegHanoiSimple(9)
    expect = O.bfs(["hanoi4", 9, 0], "frontier")[0]
    for wb in (10, 13, 16):
        assert psb.bfs(h, "frontier", 0, window_bits=wb)["counts"] == expect, wb


def test_pancake13_prefix_and_sum(golden):
    """PuzzleSearchTests.cpp:569 prefix (depth 6) and every state reached (13!)."""
    v = [x for x in golden["search"] if x["puzzle"] == ["pancake", 13, 0]][0]
    p = psb.PancakeSimple(13)
    r = psb.bfs(p, "three_bit", 0, max_depth=6)
    assert r["counts"] == v["counts"]
    full = psb.bfs(p, "three_bit", 0)["counts"]
    assert full[:7] == v["counts"]
    assert sum(full) == math.factorial(13)


def test_hanoi18_prefix_and_sum(golden):
    """HanoiTowersTests/HanoiSearchTests.cpp:25-33: first 121 depths of 18-disk
    Hanoi; the full two-bit search reaches all 4^18 states."""
    v = [x for x in golden["legacy_hanoi"] if x["puzzle"] == ["hanoi4", 18, 0]][0]
    p = psb.FourPegHanoiSimple(18)
    r = psb.bfs(p, "two_bit", 0)
    assert r["counts"][:121] == v["counts"]
    assert sum(r["counts"]) == 4 ** 18


def test_hanoi17_prefix(golden):
    v = [x for x in golden["legacy_hanoi"] if x["puzzle"] == ["hanoi4", 17, 0]][0]
    p = psb.FourPegHanoiSimple(17)
    r = psb.bfs(p, "three_bit", 0, max_depth=120)
    assert r["counts"] == v["counts"]


def test_session_reuse_and_starts():
    p = psb.SlidingTilePuzzleSimple(3, 3)
    s = psb.BfsSession(p, "two_bit")
    for start in ("0 1 2 3 4 5 6 7 8", "1 2 3 4 0 5 6 7 8", "8 7 6 5 4 3 2 1 0"):
        idx = p.Parse(start)
        a, _ = s.run(idx)
        b, _ = s.run(idx)
        assert a == b == O.bfs(["sliding", 3, 3], "two_bit", idx)[0]
    s.close()


def test_stats_are_consistent():
    p = psb.PancakeSimple(11)
    r = psb.bfs(p, "three_bit", 0, levels=True, direction="top_down")
    st = r["stats"]
    assert st["expanded"] == math.factorial(11)
    assert st["children"] == 10 * math.factorial(11)
    assert 0 < st["local_children"] <= st["children"]
    assert sum(r["level_children"]) == st["children"]
    assert st["levels"] == len(r["counts"])


@pytest.mark.parametrize("spec,algo", [(["hanoi4", 8, 0], "two_bit"), (["hanoi4", 9, 0], "three_bit"),
                                       (["hanoi4", 10, 0], "two_bit"), (["sliding", 3, 3], "two_bit"),
                                       (["sliding", 3, 3], "three_bit"), (["pancake", 9, 0], "two_bit")])
def test_children_stat_equals_oracle_expand(spec, algo):
    """A top-down search expands every reached state once, so its children
    statistic equals the oracle's Expand count over all reached states
    (4-peg Hanoi: 6*4^n - 6*2^n, since no move joins two empty pegs)."""
    p = {"pancake": lambda: psb.PancakeSimple(spec[1]), "sliding": lambda: psb.SlidingTilePuzzleSimple(*spec[1:]),
         "hanoi4": lambda: psb.FourPegHanoiSimple(spec[1], bool(spec[2]))}[spec[0]]()
    r = psb.bfs(p, algo, 0, levels=True, direction="top_down")
    dist, _ = O.depths(spec, 0)
    reached = [i for i in range(len(dist)) if dist[i] != 255]
    want = sum(len(O.expand(spec, reached[k:k + 4096])[0]) for k in range(0, len(reached), 4096))
    assert r["stats"]["children"] == want
    assert sum(r["level_children"]) == want
    if spec[0] == "hanoi4":
        assert want == 6 * 4 ** spec[1] - 6 * 2 ** spec[1]


@pytest.mark.parametrize("disks", [1, 2, 3, 6, 9, 12])
def test_hanoi_search_restored_counts(disks):
    """HanoiSearch (HanoiTowers/HanoiSearch.cpp): the two-bit search over the
    symmetric space, each canonical state counted by its class size
    (PegsMult), gives the per-depth counts of the full space (the oracle's
    search without symmetry); the canonical counts are the symmetric
    search's own."""
    r = psb.bfs(psb.FourPegHanoiSimple(disks, True), "two_bit", 0, restored=True)
    assert r["counts"] == O.bfs(["hanoi4", disks, 1], "two_bit")[0]
    assert r["restored"] == O.bfs(["hanoi4", disks, 0], "two_bit")[0]
    assert sum(r["restored"]) == 4 ** disks


@pytest.mark.parametrize("disks", [17, 18])
def test_hanoi_search_golden(disks, golden):
    """The reference's HanoiSearchTests (121 depths, maxSteps = 120)."""
    v = [x for x in golden["legacy_hanoi"] if x["puzzle"] == ["hanoi4", disks, 0]][0]
    r = psb.bfs(psb.FourPegHanoiSimple(disks, True), "two_bit", 0, max_depth=120, restored=True)
    assert r["restored"] == v["counts"]


def test_restored_counts_need_symmetric_hanoi():
    with pytest.raises(psb.PsbError) as e:
        psb.bfs(psb.FourPegHanoiSimple(8), "two_bit", 0, restored=True)
    assert e.value.code == -5
    with pytest.raises(psb.PsbError):
        psb.bfs(psb.FourPegHanoiSimple(8, True), "three_bit", 0, restored=True)


@pytest.mark.parametrize("spec", [["pancake", 10, 0], ["sliding", 3, 3], ["hanoi4", 9, 0], ["hanoi4", 8, 1]])
def test_far_mark_modes_agree(spec):
    """Two-bit long-range marks read-first, through the far bitmap for the
    near marks, or for all of them: the same counts and final code array
    as the oracle, top-down and with bottom-up levels."""
    p = {"pancake": lambda: psb.PancakeSimple(spec[1]), "sliding": lambda: psb.SlidingTilePuzzleSimple(*spec[1:]),
         "hanoi4": lambda: psb.FourPegHanoiSimple(spec[1], bool(spec[2]))}[spec[0]]()
    counts, fin = O.bfs(spec, "two_bit", 0, final=True)
    for mode in ("none", "near", "all", "auto"):
        for direction in ("top_down", "auto"):
            r = psb.bfs(p, "two_bit", 0, final=True, far_marks=mode, direction=direction, window_bits=10)
            assert r["counts"] == counts and r["final"] == fin, (mode, direction)


@pytest.mark.parametrize("spec,algo", [(["pancake", 10, 0], "two_bit"), (["pancake", 10, 0], "three_bit"),
                                       (["hanoi4", 9, 0], "two_bit"), (["sliding", 4, 2], "three_bit")])
def test_thread_shapes_agree(spec, algo):
    """128, 256 and 512 threads per block (separate kernel instances) give
    the oracle's counts and final arrays, top-down and with bottom-up levels."""
    p = {"pancake": lambda: psb.PancakeSimple(spec[1]), "sliding": lambda: psb.SlidingTilePuzzleSimple(*spec[1:]),
         "hanoi4": lambda: psb.FourPegHanoiSimple(spec[1], bool(spec[2]))}[spec[0]]()
    counts, fin = O.bfs(spec, algo, 0, final=True)
    for threads in (128, 256, 512):
        for direction in ("top_down", "auto"):
            for wb in (10, 0):
                r = psb.bfs(p, algo, 0, final=True, threads=threads, direction=direction, window_bits=wb)
                assert r["counts"] == counts and r["final"] == fin, (threads, direction, wb)


def test_trivial_puzzles():
    assert psb.bfs(psb.PancakeSimple(2), "three_bit", 0)["counts"] == [1, 1]
    assert psb.bfs(psb.FourPegHanoiSimple(1), "two_bit", 0)["counts"] == [1, 3]
    assert psb.bfs(psb.SlidingTilePuzzleSimple(2, 1), "classic", 0)["counts"] == [1, 1]


def test_pool_reuse_and_release():
    """Back-to-back searches reuse the pooled arrays (same results); releasing
    the pool between searches changes nothing either."""
    p = psb.PancakeSimple(10)
    expect = O.bfs(["pancake", 10, 0], "three_bit")[0]
    for _ in range(3):
        assert psb.bfs(p, "three_bit", 0)["counts"] == expect
    psb.release_cached_memory()
    assert psb.bfs(p, "three_bit", 0)["counts"] == expect
    assert psb.bfs(p, "two_bit", 0)["counts"] == expect
    psb.release_cached_memory(0)
