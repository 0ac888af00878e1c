"""Full-size parity on the large configurations: per-depth counts of every
depth equal the reference's own CPU code's (tests/golden/large_counts.json,
made by tests/golden/make_large_fixtures.py):
  * 13-pancake three-bit and two-bit (6,227,020,800 states, 16 depths);
  * 14-pancake two-bit (87,178,291,200 states, 17 depths), with every
    depth's frontier spilled as the reference's segment streams;
  * 18-disk 4-peg Hanoi two-bit (68,719,476,736 states, 226 depths), and
    the same counts from the symmetric search (HanoiSearch) restored by
    class size."""
import json
import math
import os

import pytest

import puzzlesearch_b200 as psb

pytestmark = pytest.mark.gpu

PATH = os.path.join(os.path.dirname(__file__), "golden", "large_counts.json")


def fixture(name):
    with open(PATH) as f:
        return json.load(f)["searches"][name]["counts"]


def test_pancake13_three_bit():
    want = fixture("pancake13")
    r = psb.bfs(psb.PancakeSimple(13), "three_bit", 0)
    assert r["counts"] == want
    assert sum(want) == math.factorial(13)


def test_pancake13_two_bit_shapes():
    """The default two-bit search (far marks NEAR, 128 threads per block at
    this size), the 256-thread shape with the far bitmap for every long-range
    mark, and read-first far marks."""
    want = fixture("pancake13")
    p = psb.PancakeSimple(13)
    r = psb.bfs(p, "two_bit", 0)
    assert r["counts"] == want and r["stats"]["threads"] == 128
    r = psb.bfs(p, "two_bit", 0, threads=256, far_marks="all")
    assert r["counts"] == want and r["stats"]["threads"] == 256
    r = psb.bfs(p, "two_bit", 0, far_marks="none")
    assert r["counts"] == want
    psb.lib().psb_release_cached_memory(0)


def test_pancake14_two_bit_with_spill():
    want = fixture("pancake14")
    per_depth = {}

    def sink(depth, segment, data, states):
        per_depth[depth] = per_depth.get(depth, 0) + states
        return False

    r = psb.bfs(psb.PancakeSimple(14), "two_bit", 0, spill=sink)
    assert r["counts"] == want
    assert [per_depth[d] for d in range(len(want))] == want
    psb.lib().psb_release_cached_memory(0)


def test_hanoi18_two_bit_and_symmetric():
    want = fixture("hanoi18")
    assert psb.bfs(psb.FourPegHanoiSimple(18), "two_bit", 0)["counts"] == want
    psb.lib().psb_release_cached_memory(0)
    r = psb.bfs(psb.FourPegHanoiSimple(18, True), "two_bit", 0, restored=True)
    assert r["restored"] == want
    psb.lib().psb_release_cached_memory(0)
