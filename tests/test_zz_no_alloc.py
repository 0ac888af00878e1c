"""psb_bfs_noalloc: the search for callers that cannot allocate device memory.

Some callers may not call cudaMalloc: all device memory belongs to another
allocator (a framework's caching allocator, a pool sized at start-up) or
arrives from one pre-reserved arena.  They pass the bit arrays in, and the
entry point keeps its few bytes of scratch in a static device array shared
by all calls.  This test calls it through the C ABI, twice in a row per case,
and checks its per-depth counts (and, for the two-bit search, the final code
array) against psb_bfs bit for bit.  It sits in its own file so that pytest
collects it last."""
import ctypes

import pytest

import puzzlesearch_b200 as psb

pytestmark = pytest.mark.gpu

CASES = [(lambda: psb.PancakeSimple(10), "three_bit"),
         (lambda: psb.SlidingTilePuzzleSimple(3, 3), "two_bit"),
         (lambda: psb.FourPegHanoiSimple(9), "frontier"),
         (lambda: psb.PancakeSimple(8), "classic"),
         (lambda: psb.FourPegHanoiSimple(12, True), "two_bit"),
         (lambda: psb.PancakeSimple(13), "three_bit")]


def noalloc(puzzle, algo, d, initial=0, max_depth=0):
    cap = 1 << 16
    counts = (ctypes.c_uint64 * cap)()
    nd = ctypes.c_uint32()
    rc = psb.lib().psb_bfs_noalloc(puzzle.handle, psb._algo(algo), initial,
                                   ctypes.cast(d.data_ptr(), psb.u64p), d.numel(), max_depth, None,
                                   counts, cap, ctypes.byref(nd))
    psb._check(rc)
    return list(counts[:nd.value])


@pytest.mark.parametrize("case", range(len(CASES)))
def test_matches_psb_bfs_twice(case):
    torch = pytest.importorskip("torch")
    make, algo = CASES[case]
    puzzle = make()
    ref = psb.bfs(puzzle, algo, 0, final=(algo == "two_bit"))
    words = puzzle.footprint(algo) // 8 + 1
    d = torch.empty(words, dtype=torch.int64, device="cuda")  # the caller allocates
    d.fill_(-1)  # garbage in: the entry point must clear what it needs
    torch.cuda.synchronize()
    for _ in range(2):
        got = noalloc(puzzle, algo, d)
        assert got == ref["counts"]
        if algo == "two_bit":
            w2 = len(ref["final"])
            final = [v & (2 ** 64 - 1) for v in d[:w2].cpu().tolist()]
            assert final == ref["final"]


def test_max_depth_and_other_start():
    torch = pytest.importorskip("torch")
    p = psb.PancakeSimple(11)
    d = torch.empty(p.footprint("two_bit") // 8 + 1, dtype=torch.int64, device="cuda")
    torch.cuda.synchronize()
    start = p.Parse("3 1 4 0 5 9 2 6 8 7 10")
    for _ in range(2):
        assert noalloc(p, "two_bit", d, start, max_depth=5) == psb.bfs(p, "two_bit", start, max_depth=5)["counts"]


def test_rejects_what_does_not_fit():
    torch = pytest.importorskip("torch")
    p = psb.PancakeSimple(9)
    small = torch.empty(16, dtype=torch.int64, device="cuda")
    with pytest.raises(psb.PsbError) as e:
        noalloc(p, "three_bit", small)
    assert e.value.code == -4
    # More windows than the static scratch holds: rejected before any device access.
    huge = psb.FourPegHanoiSimple(26)
    cap = 1 << 4
    counts = (ctypes.c_uint64 * cap)()
    nd = ctypes.c_uint32()
    rc = psb.lib().psb_bfs_noalloc(huge.handle, psb.TWO_BIT, 0, ctypes.cast(small.data_ptr(), psb.u64p),
                                   2 ** 62, 0, None, counts, cap, ctypes.byref(nd))
    assert rc == -4


def test_rejects_unaligned_arrays():
    """A sub-tensor one word in is 8-byte aligned only: rejected on the host
    before the device is touched, and the next aligned call still works."""
    torch = pytest.importorskip("torch")
    p = psb.PancakeSimple(9)
    d = torch.empty(p.footprint("three_bit") // 8 + 64, dtype=torch.int64, device="cuda")
    torch.cuda.synchronize()
    with pytest.raises(psb.PsbError) as e:
        noalloc(p, "three_bit", d[1:])
    assert e.value.code == -1
    assert noalloc(p, "three_bit", d) == psb.bfs(p, "three_bit", 0)["counts"]
