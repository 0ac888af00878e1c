"""Pins the CPU oracle (oracle/psb_oracle.c) to the reference's golden vectors
and, when oracle/_ref has been built from the reference's sources, to the
reference itself.  CPU only."""
import json
import math
import os
import random
import subprocess

import pytest

import oracle as O

SMALL = 4_000_000  # state-count cap for full BFS runs in the CPU suite


def n_states(spec):
    return O.info(spec)["indexes"]


def start_index(spec, start):
    return 0 if start is None else O.parse(spec, start)


# --- permutation ranking (PuzzlesTests/PermutationMapTest.cpp) ---------------

def test_permutation_compact(golden):
    for case in golden["permutation"]["compact"]:
        assert O.perm_compact(case["perm"]) == case["compact"], case["source"]
        assert O.perm_uncompact(case["compact"]) == case["perm"], case["source"]


def test_permutation_rank(golden):
    for case in golden["permutation"]["rank"]:
        assert O.perm_rank(case["perm"]) == case["rank"], case["source"]
        assert O.perm_unrank(case["rank"], len(case["perm"])) == case["perm"], case["source"]


def test_permutation_roundtrip_random():
    rng = random.Random(1)
    for n in range(1, 17):
        for _ in range(50):
            idx = rng.randrange(math.factorial(n))
            assert O.perm_rank(O.perm_unrank(idx, n)) == idx


# --- expand known-answer tests (PancakeTest, FourPegHanoiTest, SlidingPuzzleTest)

def test_expand_known_answers(golden):
    for kat in golden["expand_kats"]:
        spec = kat["puzzle"]
        parent = 0 if kat["parent"] is None else O.parse(spec, kat["parent"])
        if kat["parent_index"] is not None:
            assert parent == kat["parent_index"], kat["source"]
        if kat["parent"] is not None:
            assert O.to_string(spec, parent) == kat["parent"], kat["source"]
        children, ops = O.expand(spec, [parent])
        got = [O.to_string(spec, c) for c in children]
        exp = kat["children"]
        if kat["prefix_only"] and spec[0] == "sliding":
            # The sliding tests list the children they check; all must be present.
            assert set(exp) <= set(got), kat["source"]
            continue
        # Each test checks the first len(exp) children in order (some list fewer
        # than the puzzle produces, e.g. FourPegHanoiTest.cpp Opt19_Symmetry).
        assert got[:len(exp)] == exp, (kat["test"], kat["source"])
        for o, e in zip(ops, kat["ops"]):
            if e is not None:
                assert o == e, (kat["test"], kat["source"])


def test_expand_matches_reference_batches(golden):
    """Seeded batches run through the reference's Puzzle::Expand (oracle/_ref)."""
    for batch in golden["ref_expand"]:
        children, ops = O.expand(batch["puzzle"], batch["parents"], batch["opbits"])
        assert children == batch["children"], batch["puzzle"]
        assert ops == batch["child_ops"], batch["puzzle"]


# --- BFS golden vectors -------------------------------------------------------

ALGOS = ["two_bit", "three_bit", "frontier", "classic"]


def _algos_for(spec):
    return [a for a in ALGOS if a != "frontier" or O.info(spec)["ops"] <= 4]


def test_search_vectors(golden):
    """PuzzlesTests/PuzzleSearchTests.cpp vectors, every in-memory algorithm."""
    ran = 0
    for v in golden["search"]:
        spec = v["puzzle"]
        if not v["full"] or n_states(spec) > SMALL:
            continue
        init = start_index(spec, v["start"])
        for algo in _algos_for(spec):
            counts, _ = O.bfs(spec, algo, init)
            assert counts == v["counts"], (spec, algo, v["source"])
            ran += 1
    assert ran >= 12


def test_legacy_sliding_vectors(golden):
    """SlidingPuzzleTests/TestFrontierSearch.cpp: other starts and boards."""
    ran = 0
    for v in golden["legacy_sliding"]:
        spec = v["puzzle"]
        if not v["full"] or n_states(spec) > SMALL:
            continue
        counts, _ = O.bfs(spec, "three_bit", O.parse(spec, v["start"]))
        assert counts == v["counts"], (spec, v["start"], v["source"])
        assert len(counts) - 1 == v["radius"]
        ran += 1
    assert ran >= 7


def test_reference_runs(golden):
    """Per-depth counts from the reference's own InMemory BFS (oracle/_ref)."""
    for run in golden["ref_runs"]:
        spec = run["puzzle"]
        counts, _ = O.bfs(spec, run["algo"], O.parse(spec, run["start"]))
        assert counts == run["counts"], (spec, run["algo"], run["start"])


def test_depths_match_reference_runs(golden):
    """orc_depths (the per-state distances a spilled frontier is checked
    against) gives the reference's own per-depth counts."""
    import numpy as np
    ran = 0
    for run in golden["ref_runs"]:
        spec = run["puzzle"]
        if O.info(spec)["indexes"] > 4_000_000 or run["algo"] != "two_bit":
            continue
        d, k = O.depths(spec, O.parse(spec, run["start"]))
        hist = np.bincount(d[d != 255], minlength=k)
        assert hist.tolist() == run["counts"], (spec, run["start"])
        ran += 1
    assert ran >= 10


def test_sum_invariants():
    """Every pancake and Hanoi state is reachable; half of the sliding states are."""
    assert sum(O.bfs(["pancake", 8, 0], "three_bit")[0]) == math.factorial(8)
    assert sum(O.bfs(["hanoi4", 8, 0], "two_bit")[0]) == 4 ** 8
    assert sum(O.bfs(["sliding", 3, 3], "two_bit")[0]) == math.factorial(9) // 2


def test_final_arrays_consistent():
    """Final arrays: the 2-bit array holds every reached state as OLD (code 1);
    three-bit old|cur hold the last two levels."""
    spec = ["pancake", 7, 0]
    counts, fin = O.bfs(spec, "two_bit", 0, final=True)
    N = n_states(spec)
    old = sum(1 for i in range(N) if (fin[(2 * i) >> 6] >> ((2 * i) & 63)) & 1 == 0 and
              (fin[(2 * i + 1) >> 6] >> ((2 * i + 1) & 63)) & 1 == 1)
    assert old == sum(counts) == N
    counts3, fin3 = O.bfs(spec, "three_bit", 0, final=True)
    W = (N + 63) // 64
    popc = [sum(bin(w).count("1") for w in fin3[k * W:(k + 1) * W]) for k in range(3)]
    assert popc == [counts3[-2], counts3[-1], 0]


@pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built (reference sources absent)")
def test_oracle_visits_what_reference_expands():
    """The set of parents the reference expands equals the oracle's reached set."""
    for spec, algo in [(["hanoi4", 6, 1], "two_bit"), (["sliding", 3, 2], "three_bit"), (["pancake", 6, 0], "classic")]:
        start = O.to_string(spec, 0)
        parents = O.ref_bfs_parents(spec, algo, start, 1 << 22)
        counts, fin = O.bfs(spec, "two_bit", 0, final=True)
        reached = [i for i in range(n_states(spec)) if (fin[(2 * i + 1) >> 6] >> ((2 * i + 1) & 63)) & 1]
        assert sorted(parents) == reached
        assert len(parents) == sum(counts)


@pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built (reference sources absent)")
def test_oracle_vs_reference_random_expand():
    rng = random.Random(5)
    for spec in [["sliding", 4, 3], ["sliding", 2, 8], ["pancake", 14, 0], ["hanoi4", 18, 0], ["hanoi4", 12, 1]]:
        N = n_states(spec)
        ops_n = O.info(spec)["ops"]
        parents = [rng.randrange(N) for _ in range(500)]
        opbits = [rng.randrange(1 << ops_n) if i % 2 else 0 for i in range(500)]
        assert O.expand(spec, parents, opbits) == O.ref_expand(spec, parents, opbits), spec


@pytest.mark.skipif(not os.path.exists(os.path.join(O.HERE, "_ref", "psbref_mt")),
                    reason="oracle/_ref not built (reference sources absent)")
def test_mt_fixture_driver_matches_reference():
    """psbref_mt (the reference's puzzle classes under a multi-threaded
    three-bit level loop, which made the 14-pancake and 18-disk fixtures)
    gives the unmodified reference's per-depth counts."""
    ref_dir = os.path.join(O.HERE, "_ref")
    for spec in (["pancake", 10, 0], ["hanoi4", 11, 0], ["hanoi4", 9, 1], ["sliding", 3, 3], ["sliding", 4, 2]):
        kind = {"sliding": 1, "pancake": 2, "hanoi4": 3}[spec[0]]
        args = [str(kind), str(spec[1]), str(spec[2])]
        mt = subprocess.run([os.path.join(ref_dir, "psbref_mt")] + args + ["3"], check=True, capture_output=True,
                            text=True).stdout
        one = subprocess.run([os.path.join(ref_dir, "psbref")] + args + ["2"], check=True, capture_output=True,
                             text=True).stdout
        assert json.loads(mt)["counts"] == json.loads(one)["counts"], spec


def test_large_fixtures(golden):
    """The full-size fixtures: every state reached once, and each vector
    starts with the reference's own golden prefix where one exists."""
    path = os.path.join(os.path.dirname(__file__), "golden", "large_counts.json")
    with open(path) as f:
        large = json.load(f)["searches"]
    assert sorted(large) == ["hanoi18", "pancake13", "pancake14"]
    assert sum(large["pancake13"]["counts"]) == math.factorial(13)
    assert sum(large["hanoi18"]["counts"]) == 4 ** 18
    assert large["pancake13"]["kind"] == "reference InMemoryThreeBitBFS"
    h18 = [v for v in golden["legacy_hanoi"] if v["puzzle"] == ["hanoi4", 18, 0]][0]
    assert large["hanoi18"]["counts"][:len(h18["counts"])] == h18["counts"]
    p13 = [v for v in golden["search"] if v["puzzle"] == ["pancake", 13, 0]][0]
    assert large["pancake13"]["counts"][:len(p13["counts"])] == p13["counts"]
    assert sum(large["pancake14"]["counts"]) == math.factorial(14)
    assert large["pancake14"]["counts"][:2] == [1, 13]  # depth 1: the 13 flips of the identity


# --- codecs (CommonTests/StreamVIntTests.cpp, CompressionTests.cpp) -----------

def test_streamvint_tuples(golden):
    for case in golden["streamvint"]["tuples"]:
        enc = O.svi_encode_tuple(case["values"])
        assert len(enc) == case["bytes"], case["source"]
        dec, n = O.svi_decode_tuple(enc)
        assert dec == case["values"] and n == case["bytes"]


def test_streamvint_tuple_lists(golden):
    for case in golden["streamvint"]["tuple_lists"]:
        vals = case["values"]
        total = sum(len(O.svi_encode_tuple(vals[i:i + 4])) for i in range(0, len(vals), 4))
        assert total == case["bytes"], case["source"]


def test_streamvint_roundtrip():
    vals = [i * i for i in range(65536)]  # StreamVIntTests.cpp:146-160
    enc = O.svi_encode(vals)
    dec, size = O.svi_decode(enc)
    assert dec == vals and size == len(enc)
    assert O.svi_encode([]) == b""


def test_compression_selection(golden):
    c = golden["compression"]
    for key in ("bitmap_stride", "svi_stride"):
        case = c[key]
        vals = [i * case["stride"] for i in range(case["count"])]
        enc = O.fc_encode(vals)
        assert O.fc_is_bitmap(enc) == case["is_bitmap"], case["source"]
        dec, size = O.fc_decode(enc, 1024)
        assert dec == vals and size == len(enc)
    vals = c["bitmap_small"]["values"]
    enc = O.fc_encode_bitmap(vals)
    assert O.fc_decode(enc, 1024)[0] == vals
    for key in ("out_of_order", "same_begin_end"):
        assert O.fc_encode_bitmap(c[key]["values"], with_check=True) == -1, c[key]["source"]
    vals = [i * 7 for i in range(150)] + [700]  # CompressionTests.cpp TestCompression_WithCheck
    enc = O.fc_encode(vals, with_check=True)
    assert not O.fc_is_bitmap(enc)
    assert O.fc_decode(enc, 1024)[0] == vals
    vals = c["large_range"]["values"]
    enc = O.fc_encode(vals)
    assert O.fc_decode(enc, 400)[0] == vals


@pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built (reference sources absent)")
def test_codec_bytes_match_reference():
    rng = random.Random(3)
    for trial in range(40):
        n = rng.choice([1, 3, 8, 129, 200, 1000, 5000])
        span = rng.choice([n, 2 * n, 10 * n, 1 << 20, 1 << 31])
        vals = sorted(rng.sample(range(span), n)) if span >= n else list(range(n))
        for wc in (False, True):
            assert O.fc_encode(vals, wc) == O.ref_fc_encode(vals, wc), (n, span, wc)


def test_opbits_known_answers(golden):
    """OpBitsCompression<2/4/8> (CommonTests/CompressionOpBitsTests.cpp):
    encoded sizes and round trips."""
    assert len(golden["opbits"]) == 9
    for v in golden["opbits"]:
        enc = O.opbits_encode(v["bits"], v["values"])
        assert len(enc) == v["bytes"], v["source"]
        assert O.opbits_decode(v["bits"], enc, len(v["values"])) == v["values"], v["source"]


@pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built (reference sources absent)")
def test_opbits_bytes_match_reference():
    rng = random.Random(11)
    for bits in (2, 4, 8):
        for n in (8, 64, 4096):
            ops = [rng.randrange(1 << bits) for _ in range(n)]
            assert O.opbits_encode(bits, ops) == O.ref_opbits_encode(bits, ops), (bits, n)


@pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built (reference sources absent)")
def test_pancake_optimized_matches_reference():
    """PancakeOptimized (Puzzles/PancakeOptimized.cpp): the oracle's index,
    Expand and BFS equal the reference class's; below 12 pancakes the index is
    PancakeSimple's, above it the 29-bit split of the same rank."""
    rng = random.Random(12)
    for n in (5, 8, 11, 12, 13, 14, 16):
        spec = ["pancake_opt", n, 0]
        N = n_states(spec)
        parents = []
        while len(parents) < 300:
            p = rng.randrange(N)
            if n < 12 or (p & ((1 << 29) - 1)) < math.factorial(12):
                parents.append(p)
        ops = [rng.randrange(1 << (n - 1)) if i % 2 else 0 for i in range(len(parents))]
        assert O.expand(spec, parents, ops) == O.ref_expand(spec, parents, ops), n
        for p in parents[:30]:
            assert O.parse(spec, O.to_string(spec, p)) == p
    for n in (6, 9, 10):
        start = O.to_string(["pancake_opt", n, 0], 0)
        assert O.bfs(["pancake_opt", n, 0], "three_bit")[0] == O.ref_bfs(["pancake_opt", n, 0], "three_bit", start)
    assert n_states(["pancake_opt", 12, 0]) == 1 << 29
    assert n_states(["pancake_opt", 14, 0]) == 13 * 14 << 29


@pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built (reference sources absent)")
def test_hanoi_optimized_matches_reference():
    """FourPegHanoiOptimized (Puzzles/FourPegHanoiOptimized.cpp:164-204):
    FourPegHanoiSimple's index; with symmetry it restores the peg order only
    when a move empties or fills a peg.  The oracle's kind 5 equals the
    reference class on any parent, and on the canonical (reachable) states
    it equals the Simple class."""
    rng = random.Random(24)
    for n, sym in ((5, 0), (10, 1), (18, 0), (18, 1), (24, 1)):
        parents = [rng.randrange(4 ** n) for _ in range(400)]
        ops = [rng.randrange(16) if i % 2 else 0 for i in range(400)]
        assert O.expand(["hanoi4_opt", n, sym], parents, ops) == O.ref_expand(["hanoi4_opt", n, sym], parents, ops)
    import numpy as np
    d, _ = O.depths(["hanoi4", 8, 1], 0)
    reached = [int(x) for x in np.nonzero(d != 255)[0]]
    assert O.expand(["hanoi4_opt", 8, 1], reached) == O.expand(["hanoi4", 8, 1], reached)
    for n, sym in ((8, 0), (9, 1)):
        start = O.to_string(["hanoi4", n, sym], 0)
        assert O.ref_bfs(["hanoi4_opt", n, sym], "three_bit", start) == O.bfs(["hanoi4_opt", n, sym], "three_bit")[0]


SLIDING_OPT_SHAPES = [(2, 2), (3, 2), (4, 2), (5, 2), (6, 2), (7, 2), (8, 2), (3, 3), (4, 3), (5, 3), (4, 4)]


@pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built (reference sources absent)")
def test_sliding_optimized_index_matches_reference():
    """SlidingTilePuzzleOptimized's index (Puzzles/SlidingTilePuzzleOptimized.cpp:
    99-236): the oracle's Parse, ToString and IndexesCount equal the reference
    class's own on random solvable boards of every shape the reference
    instantiates (the reference's Expand runs on a GPU and is not built into
    the oracle; the expand is pinned by the Opt3x2 / Opt4x4 known answers and
    by search counts)."""
    rng = random.Random(31)
    for w, h in SLIDING_OPT_SHAPES:
        spec = ["sliding_opt", w, h]
        assert O.info(spec)["indexes"] == O.ref_indexes_count(spec), spec
        checked = 0
        while checked < 60:
            perm = list(range(w * h))
            rng.shuffle(perm)
            state = " ".join(map(str, perm))
            try:
                index = O.parse(spec, state)
            except ValueError:
                continue  # the other parity class: the reference's Parse exits on it
            assert index == O.ref_parse(spec, state), (spec, state)
            assert O.to_string(spec, index) == state == O.ref_to_string(spec, index), (spec, state)
            checked += 1


def test_sliding_optimized_searches_equal_simple(golden):
    """Search counts are index-independent: the optimized index gives the
    golden ST vectors (PuzzleSearchTests.cpp:294-333 run DiskBasedOpt* on
    SlidingTilePuzzleOptimized<5, 2> and expect ST5x2), and left / right
    moves are the index -+ 1 of the blank digit."""
    ran = 0
    for v in golden["search"]:
        spec = v["puzzle"]
        if spec[0] != "sliding" or not v["full"] or n_states(spec) > SMALL:
            continue
        ospec = ["sliding_opt", spec[1], spec[2]]
        init = O.parse(ospec, v["start"])
        for algo in ("two_bit", "three_bit", "frontier", "classic"):
            assert O.bfs(ospec, algo, init)[0] == v["counts"], (ospec, algo, v["source"])
            ran += 1
    assert ran >= 8
    rng = random.Random(5)
    spec = ["sliding_opt", 4, 3]
    parents = []
    while len(parents) < 300:
        i = rng.randrange(O.info(spec)["indexes"])
        if (i & 15) < 12:
            parents.append(i)
    ch, ops = O.expand(spec, parents)
    simple = ["sliding", 4, 3]
    sch, sops = O.expand(simple, [O.parse(simple, O.to_string(spec, p)) for p in parents])
    assert [O.to_string(spec, c) for c in ch] == [O.to_string(simple, c) for c in sch] and ops == sops
