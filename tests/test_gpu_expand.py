"""GPU parity of the batched Expand kernels (psb_expand) against the oracle,
the reference's own Expand batches and its known-answer tests.
Integer work: every child index and operator must match bit for bit."""
import math
import random
import zlib

import pytest

import oracle as O
import puzzlesearch_b200 as psb
from _puzzles import make

pytestmark = pytest.mark.gpu




ALL_SPECS = ([["pancake", n, 0] for n in range(2, 17)] +
             [["sliding", w, h] for w in range(1, 9) for h in range(1, 9) if 2 <= w * h <= 16] +
             [["hanoi4", n, s] for n in (1, 2, 5, 7, 10, 12, 18, 21, 31) for s in (0, 1)])


def test_known_answers(golden):
    """PuzzlesTests/{PancakeTest,FourPegHanoiTest,SlidingPuzzleTest}.cpp on the GPU."""
    for kat in golden["expand_kats"]:
        p = make(kat["puzzle"])
        parent = 0 if kat["parent"] is None else p.Parse(kat["parent"])
        children, ops = p.Expand([parent], [0])
        got = [p.ToString(c) for c in children]
        if kat["puzzle"][0] == "sliding":
            assert set(kat["children"]) <= set(got), kat["source"]
            continue
        assert got[:len(kat["children"])] == kat["children"], (kat["test"], kat["source"])
        for o, e in zip(ops, kat["ops"]):
            if e is not None:
                assert o == e, (kat["test"], kat["source"])


def test_reference_expand_batches(golden):
    """Seeded batches run through the reference's own Puzzle::Expand."""
    for batch in golden["ref_expand"]:
        p = make(batch["puzzle"])
        children, ops = p.Expand(batch["parents"], batch["opbits"])
        assert children == batch["children"], batch["puzzle"]
        assert ops == batch["child_ops"], batch["puzzle"]


@pytest.mark.parametrize("spec", ALL_SPECS, ids=lambda s: f"{s[0]}{s[1]}x{s[2]}")
def test_random_batches_match_oracle(spec):
    p = make(spec)
    rng = random.Random(zlib.crc32(repr(spec).encode()))
    N = p.IndexesCount()
    ops_n = p.OperatorsCount()
    n = 3000
    parents = [rng.randrange(N) for _ in range(n)] + [0, N - 1]
    opbits = [rng.randrange(1 << ops_n) if i % 4 == 3 else 0 for i in range(len(parents))]
    assert p.Expand(parents, [0] * len(parents)) == O.expand(spec, parents)
    assert p.Expand(parents, opbits) == O.expand(spec, parents, opbits)


def test_fixed_slots_and_padding():
    """Without compaction each parent gets BranchingFactor() slots; unused ones
    are INVALID_INDEX with operator 15 (PuzzlesTests/SlidingPuzzleTest.cpp:43-60)."""
    p = psb.SlidingTilePuzzleSimple(3, 2)
    ch, ops = p.Expand([p.Parse("0 1 2 3 4 5")], compact=False)
    assert len(ch) == 4
    valid = [(c, o) for c, o in zip(ch, ops) if c != psb.INVALID_INDEX]
    assert sorted(p.ToString(c) for c, _ in valid) == sorted(["3 1 2 0 4 5", "1 0 2 3 4 5"])
    assert [o for c, o in zip(ch, ops) if c == psb.INVALID_INDEX] == [15, 15]
    h = psb.FourPegHanoiSimple(5)
    ch, ops = h.Expand([0], compact=False)
    assert len(ch) == 6 and ch.count(psb.INVALID_INDEX) == 3


def test_large_batch_spans_chunks():
    """More parents than one 2M-parent chunk (Puzzle::MAX_INDEXES_BUFFER)."""
    spec = ["pancake", 12, 0]
    p = make(spec)
    rng = random.Random(4)
    parents = [rng.randrange(p.IndexesCount()) for _ in range(2 * 1024 * 1024 + 1000)]
    got = p.Expand(parents)
    # compare a prefix and the tail across the chunk boundary with the oracle
    head = parents[:20000]
    tail = parents[-20000:]
    eh = O.expand(spec, head)
    et = O.expand(spec, tail)
    br = 11
    assert got[0][:len(eh[0])] == eh[0]
    assert got[0][-len(et[0]):] == et[0] and got[1][-len(et[1]):] == et[1]
    assert len(got[0]) == len(parents) * br


def test_device_pointers():
    torch = pytest.importorskip("torch")
    spec = ["hanoi4", 12, 1]
    p = make(spec)
    rng = random.Random(8)
    parents = [rng.randrange(p.IndexesCount()) for _ in range(5000)]
    d_par = torch.tensor(parents, dtype=torch.int64, device="cuda")
    d_out = torch.empty(len(parents) * 6, dtype=torch.int64, device="cuda")
    d_ops = torch.empty(len(parents) * 6, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()  # the library runs on its own non-blocking stream
    n = p.expand_device(d_par.data_ptr(), 0, len(parents), d_out.data_ptr(), d_ops.data_ptr())
    assert n == len(parents) * 6
    out = [v & (2 ** 64 - 1) for v in d_out.cpu().tolist()]
    ops = d_ops.cpu().tolist()
    got = ([c for c in out if c != psb.INVALID_INDEX], [o for c, o in zip(out, ops) if c != psb.INVALID_INDEX])
    assert got == O.expand(spec, parents)


def test_rejects_out_of_range_parent():
    p = psb.PancakeSimple(6)
    with pytest.raises(psb.PsbError):
        p.Expand([math.factorial(6)])
