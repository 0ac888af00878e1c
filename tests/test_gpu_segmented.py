"""The segmented (out-of-core) search, psb_bfs_segmented: the reference's
DiskBasedOptThreeBitBFS scheme (Common/DiskBasedOptThreeBitBFS.cpp:12-252)
with host memory for its segment files.  Only one segment's bit arrays are
on the device at a time; its per-depth counts must equal the in-memory
searches' and the reference's golden vectors, whatever the segment size
(the reference's own disk-based tests vary segmentBits the same way,
PuzzlesTests/PuzzleSearchTests.cpp:133-333)."""
import math

import pytest

import oracle as O
import puzzlesearch_b200 as psb
from _puzzles import make

pytestmark = pytest.mark.gpu




@pytest.mark.parametrize("spec,bits", [(["sliding", 5, 2], 19), (["sliding", 5, 2], 15), (["sliding", 5, 2], 22),
                                       (["pancake", 9, 0], 12), (["pancake", 10, 0], 16), (["hanoi4", 10, 0], 14),
                                       (["hanoi4", 9, 1], 10), (["sliding", 3, 3], 32)])
def test_counts_equal_in_memory(spec, bits):
    p = make(spec)
    r = psb.bfs_segmented(p, 0, segment_bits=bits)
    assert r["counts"] == O.bfs(spec, "three_bit", 0)[0]
    n = p.IndexesCount()
    assert r["stats"]["segments"] == (n + (1 << bits) - 1) >> bits
    if r["stats"]["segments"] > 1:
        assert r["stats"]["cross_children"] > 0


def test_other_starts_and_max_depth():
    p = psb.SlidingTilePuzzleSimple(4, 3)
    for start in ("1 2 0 3 4 5 6 7 8 9 10 11", "11 10 9 8 7 6 5 4 3 2 1 0"):
        idx = p.Parse(start)
        full = psb.bfs(p, "two_bit", idx)["counts"]
        assert psb.bfs_segmented(p, idx, segment_bits=22)["counts"] == full
        assert psb.bfs_segmented(p, idx, segment_bits=24, max_depth=9)["counts"] == full[:10]


def test_reduced_memory_12_pancake():
    """12-pancake (479,001,600 states) in segments of 2^26 states: the device
    holds 3 x 8 MB of bit arrays instead of the in-memory search's 3 x 60 MB,
    and the counts equal the in-memory search's."""
    p = psb.PancakeSimple(12)
    r = psb.bfs_segmented(p, 0, segment_bits=26)
    assert r["counts"] == psb.bfs(p, "three_bit", 0)["counts"]
    assert sum(r["counts"]) == math.factorial(12)
    assert r["stats"]["segments"] == 8
    assert r["stats"]["cross_children"] > 0


def test_small_chunks_and_bad_arguments():
    p = psb.PancakeSimple(8)
    assert psb.bfs_segmented(p, 0, segment_bits=10, chunk_states=64)["counts"] == O.bfs(["pancake", 8, 0], "two_bit")[0]
    with pytest.raises(psb.PsbError) as e:
        psb.bfs_segmented(p, 0, segment_bits=9)
    assert e.value.code == -1


@pytest.mark.parametrize("fpp", [0, 1, 5])
def test_segment_files(tmp_path, fpp):
    """StoreOptions: the layers and cross-segment children go to files in two
    directories (filesPerPath 0, 1 and the reference's default 5); the counts
    equal the in-memory search's, and no file is left afterwards."""
    import os
    p = psb.SlidingTilePuzzleSimple(4, 3)
    dirs = [str(tmp_path / "disk0"), str(tmp_path / "disk1")]
    r = psb.bfs_segmented(p, 0, segment_bits=24, directories=dirs, files_per_path=fpp)
    assert r["counts"] == psb.bfs(p, "two_bit", 0)["counts"]
    assert r["stats"]["peak_disk_bytes"] > 0
    assert r["stats"]["peak_host_bytes"] < r["stats"]["peak_disk_bytes"]
    assert all(os.listdir(d) == [] for d in dirs)


def test_segment_files_unwritable(tmp_path):
    f = tmp_path / "plain"
    f.write_text("x")
    with pytest.raises(psb.PsbError) as e:
        psb.bfs_segmented(psb.PancakeSimple(8), 0, segment_bits=10, directories=[str(f)])
    assert e.value.code == -9
