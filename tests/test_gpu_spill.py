"""Frontier spill (psb_bfs_opts.spill): every depth's states, encoded on the
GPU segment by segment into the reference's compressed segment stream
(Common/CompressedFrontier.cpp:103-140; for frontier search the stream with
each state's operator bits, CompressedFrontierWriter, :56-70) and handed over
from pinned host memory.  Each stream must equal, byte for byte, the oracle's segment stream
of that depth's states in that segment (the oracle's distances come from
orc_depths, pinned to the reference's per-depth counts in test_oracle.py)."""
import math

import numpy as np
import pytest

import oracle as O
import puzzlesearch_b200 as psb
from _puzzles import make

pytestmark = pytest.mark.gpu




def run_spill(spec, algo, start=0, segment_bits=0, **kw):
    got = []

    def sink(depth, segment, data, states):
        got.append((depth, segment, data, states))
        return False

    res = psb.bfs(make(spec), algo, start, spill=sink, segment_bits=segment_bits, **kw)
    return res, got


def expected_streams(dist, depth, segment_bits, nibbles=None):
    """{segment: stream} of the states at `depth`, by the oracle: the segment
    stream, or for frontier search (nibbles = each state's operator bits) the
    stream with operator bits."""
    states = np.nonzero(dist == depth)[0].astype(np.uint64)
    seg = states >> np.uint64(segment_bits)
    out = {}
    for g in np.unique(seg):
        sel = states[seg == g]
        offs = (sel - (g << np.uint64(segment_bits))).astype(np.uint32)
        out[int(g)] = (O.segment_stream(offs) if nibbles is None
                       else O.frontier_stream(offs, nibbles[sel.astype(np.int64)]))
    return out


def check(spec, algo, start, segment_bits, res, got):
    dist, n_depths = O.depths(spec, start)
    nib = O.frontier_nibbles(spec, dist) if algo == "frontier" else None
    assert len(res["counts"]) == n_depths
    sb = segment_bits or 32
    # depths ascending, segments ascending within a depth, every depth present
    order = [(d, g) for d, g, _, _ in got]
    assert order == sorted(order)
    assert sorted({d for d, _, _, _ in got}) == list(range(n_depths))
    for d in range(n_depths):
        mine = {g: (data, states) for dd, g, data, states in got if dd == d}
        want = expected_streams(dist, d, sb, nib)
        assert set(mine) == set(want), (spec, algo, d)
        assert sum(st for _, st in mine.values()) == res["counts"][d]
        for g, stream in want.items():
            assert mine[g][0] == stream, (spec, algo, d, g)
    st = res["stats"]
    assert st["spill_segments"] == len(got)
    assert st["spill_bytes"] == sum(len(x[2]) for x in got)


CASES = [
    (["pancake", 8, 0], "two_bit", 0, 0),
    (["pancake", 8, 0], "three_bit", 0, 10),
    (["pancake", 8, 0], "classic", 0, 12),
    (["pancake", 5, 0], "frontier", 0, 6),
    (["sliding", 3, 3], "two_bit", "1 2 0 3 4 5 6 7 8", 14),
    (["sliding", 3, 3], "frontier", 0, 16),
    (["sliding", 4, 2], "three_bit", 0, 8),
    (["hanoi4", 8, 0], "two_bit", 0, 11),
    (["hanoi4", 8, 1], "three_bit", 0, 9),
    (["hanoi4", 7, 0], "frontier", 0, 7),
    (["hanoi4", 8, 1], "classic", 0, 0),
]


@pytest.mark.parametrize("case", CASES, ids=lambda c: f"{c[0][0]}{c[0][1]}-{c[1]}-sb{c[3]}")
def test_spilled_streams_equal_oracle(case):
    spec, algo, start, sb = case
    if isinstance(start, str):
        start = O.parse(spec, start)
    res, got = run_spill(spec, algo, start, sb)
    assert res["counts"] == O.bfs(spec, algo, start)[0]
    check(spec, algo, start, sb, res, got)


@pytest.mark.parametrize("algo", ["two_bit", "three_bit", "classic"])
@pytest.mark.parametrize("direction", ["bottom_up", "auto", "top_down"])
def test_spill_with_bottom_up_levels(algo, direction):
    """The frontier handed over is the same whichever direction each level
    ran: bottom-up levels keep the arrays in the same state between levels."""
    spec = ["pancake", 10, 0]
    start = 123_456
    res, got = run_spill(spec, algo, start, 20, direction=direction)
    if direction != "top_down":
        assert res["stats"]["bottom_up_levels"] > 0
    check(spec, algo, start, 20, res, got)


@pytest.mark.parametrize("algo", ["two_bit", "three_bit", "classic", "frontier"])
def test_spill_with_max_depth(algo):
    """Every depth the counts report is spilled, the last one too (three-bit
    and classic searches hold it in cur / open without expanding it)."""
    spec = ["hanoi4", 9, 0]
    res, got = run_spill(spec, algo, 0, 12, max_depth=7)
    assert len(res["counts"]) == 8
    assert sorted({d for d, _, _, _ in got}) == list(range(8))
    dist, _ = O.depths(spec, 0)
    nib = O.frontier_nibbles(spec, dist) if algo == "frontier" else None
    for d in range(8):
        want = expected_streams(dist, d, 12, nib)
        mine = {g: data for dd, g, data, _ in got if dd == d}
        assert mine == want


def test_spill_callback_stops_search():
    def sink(depth, segment, data, states):
        return depth == 3

    with pytest.raises(psb.PsbError) as e:
        psb.bfs(psb.PancakeSimple(9), "three_bit", 0, spill=sink)
    assert e.value.code == -8

    def failing(depth, segment, data, states):
        if depth == 2:
            raise KeyError("sink full")

    with pytest.raises(KeyError):  # the callback's own exception, once the search has stopped
        psb.bfs(psb.PancakeSimple(9), "two_bit", 0, spill=failing)
    assert psb.bfs(psb.PancakeSimple(9), "two_bit", 0)["counts"][:3] == [1, 8, 56]


def test_bad_segment_bits():
    with pytest.raises(psb.PsbError) as e:
        psb.bfs(psb.PancakeSimple(7), "two_bit", 0, spill=lambda *a: False, segment_bits=5)
    assert e.value.code == -1


def test_spilled_frontier_decodes_on_gpu():
    """Round trip through psb_frontier_index / psb_frontier_decode: the
    decoded depth sets partition the state space."""
    torch = pytest.importorskip("torch")
    spec = ["pancake", 9, 0]
    res, got = run_spill(spec, "two_bit", 0, 16)
    n = math.factorial(9)
    words = (n + 63) // 64
    seen = torch.zeros(words, dtype=torch.int64, device="cuda")
    for d in range(len(res["counts"])):
        level = torch.zeros(words, dtype=torch.int64, device="cuda")
        for dd, g, data, states in got:
            if dd != d:
                continue
            blocks, nb = psb.frontier_index(data)
            dev = torch.frombuffer(bytearray(data), dtype=torch.uint8).cuda()
            torch.cuda.synchronize()
            first = g << 16
            psb.frontier_decode(dev.data_ptr(), blocks, nb, level.data_ptr(), first, min(1 << 16, n - first))
        cnt = int(np.unpackbits(level.cpu().numpy().view(np.uint8)).sum())
        assert cnt == res["counts"][d]
        assert not bool((level & seen).any())
        seen |= level
    assert int(np.unpackbits(seen.cpu().numpy().view(np.uint8)).sum()) == n


def test_spill_full_size_13_pancake():
    """13-pancake three-bit (6,227,020,800 states: two 2^32-state segments),
    spilled at full size: the streams' offsets add up to every depth's count,
    the counts are unchanged and the spill is the only extra work."""
    spec = ["pancake", 13, 0]
    totals = {}

    def sink(depth, segment, data, states):
        assert segment < 2
        totals[depth] = totals.get(depth, 0) + states
        return False

    p = psb.PancakeSimple(13)
    res = psb.bfs(p, "three_bit", 0, spill=sink)
    plain = psb.bfs(p, "three_bit", 0)
    assert res["counts"] == plain["counts"]
    assert [totals[d] for d in range(len(res["counts"]))] == res["counts"]
    assert sum(res["counts"]) == math.factorial(13)
    assert res["counts"][:7] == [1, 12, 132, 1451, 14556, 130096, 1030505]


def test_spill_resources_reused_across_searches():
    """The spill's buffers stay cached between searches: a session run twice,
    and a search after one that a callback stopped part-way (its copies in
    flight are dropped), hand over the same streams."""
    spec = ["hanoi4", 9, 0]
    _, first = run_spill(spec, "two_bit", 0, 10)
    sess = psb.BfsSession(make(spec), "two_bit")
    runs = []
    for _ in range(2):
        got = []
        sess.run(0, spill=lambda d, g, data, st: got.append((d, g, data, st)) and False, segment_bits=10)
        runs.append(got)
    sess.close()
    assert runs[0] == first and runs[1] == first
    with pytest.raises(psb.PsbError):
        psb.bfs(make(spec), "two_bit", 0, spill=lambda d, g, data, st: d == 5, segment_bits=10)
    _, again = run_spill(spec, "two_bit", 0, 10)
    assert again == first
    psb.release_cached_memory()
    _, fresh = run_spill(spec, "two_bit", 0, 10)
    assert fresh == first
