"""The batch engine (psb_engine_*): many two-bit searches stepped together in
one persistent launch per level.  Every instance's per-depth counts must equal
the single-instance path (psb_bfs, two-bit) and the reference's own runs."""
import random

import pytest

import oracle as O
import puzzlesearch_b200 as psb

pytestmark = pytest.mark.gpu

TYPES = [("sliding", 2, 3), ("sliding", 2, 4), ("sliding", 3, 3), ("sliding", 2, 5), ("sliding", 4, 3),
         ("pancake", 7, 0), ("pancake", 8, 0), ("pancake", 9, 0), ("pancake", 10, 0), ("pancake", 11, 0),
         ("pancake", 12, 0), ("hanoi4", 8, 0), ("hanoi4", 10, 1), ("hanoi4", 12, 0)]


def make(kind, a, b):
    return {"sliding": lambda: psb.SlidingTilePuzzleSimple(a, b), "pancake": lambda: psb.PancakeSimple(a),
            "hanoi4": lambda: psb.FourPegHanoiSimple(a, bool(b))}[kind]()


def random_start(rng, kind, a, b, puzzle):
    if kind == "sliding":  # a uniformly random state of the start state's component
        while True:
            p = list(range(a * b))
            rng.shuffle(p)
            inv = sum(1 for i in range(len(p)) for j in range(i + 1, len(p)) if p[i] > p[j])
            z = p.index(0)
            if inv % 2 == (z // a + z % a) % 2:
                return puzzle.Parse(" ".join(map(str, p)))
    return rng.randrange(puzzle.IndexesCount())


def run_engine(eng, items):
    pending = dict(items)
    results = {}
    for tag, (p, start) in items.items():
        assert eng.add(p, start, tag)
    for _ in range(200):
        eng.step(8)
        results.update(eng.poll())
        if len(results) == len(items):
            break
    return results


def test_mixed_batch_matches_single_instance():
    rng = random.Random(2026)
    eng = psb.Engine(max_instances=256, pool_bytes=2 << 30)
    items = {}
    for tag in range(120):
        kind, a, b = TYPES[tag % len(TYPES)]
        if (kind, a) == ("sliding", 4) and tag > 60:
            continue
        p = make(kind, a, b)
        items[tag] = (p, random_start(rng, kind, a, b, p))
    got = run_engine(eng, items)
    assert set(got) == set(items)
    for tag, (p, start) in items.items():
        assert got[tag] == psb.bfs(p, "two_bit", start)["counts"], (tag, p.Name(), start)
    eng.close()


def test_reference_runs_through_engine(golden):
    eng = psb.Engine(max_instances=128, pool_bytes=1 << 30)
    items = {}
    for i, run in enumerate(golden["ref_runs"]):
        kind, a, b = run["puzzle"]
        p = make(kind, a, b)
        try:
            ok = eng.add(p, p.Parse(run["start"]), 10_000 + i)
        except psb.PsbError:
            continue  # a shape the engine does not compile in
        assert ok
        items[10_000 + i] = run["counts"]
    done = {}
    for _ in range(100):
        eng.step(8)
        done.update(eng.poll())
        if len(done) == len(items):
            break
    assert len(items) >= 30
    for tag, counts in items.items():
        assert done[tag] == counts


def test_continuous_admission_and_capacity():
    """Searches admitted while others are mid-flight give the same counts, and
    admission stops at the pool limit (HBM-footprint admission)."""
    p11 = psb.PancakeSimple(11)
    foot = psb.Engine.footprint(p11)
    eng = psb.Engine(max_instances=8, pool_bytes=3 * foot + 4096)
    assert eng.add(p11, 0, 1)
    assert eng.add(p11, 5, 2)
    assert eng.add(p11, 77, 3)
    assert not eng.add(p11, 9, 4)  # pool full
    eng.step(5)
    res = eng.poll()
    assert res == {}
    eng.step(20)
    res.update(eng.poll())
    assert set(res) == {1, 2, 3}
    assert eng.add(p11, 9, 4)  # space freed by poll
    h = psb.FourPegHanoiSimple(9)
    assert eng.add(h, 0, 5)
    while len(res) < 5:
        eng.step(10)
        res.update(eng.poll())
    for tag, (p, s) in {1: (p11, 0), 2: (p11, 5), 3: (p11, 77), 4: (p11, 9), 5: (h, 0)}.items():
        assert res[tag] == psb.bfs(p, "two_bit", s)["counts"]
    eng.close()


def test_without_graph_same_result():
    rng = random.Random(5)
    items = {}
    for tag in range(20):
        kind, a, b = TYPES[tag % 11]
        p = make(kind, a, b)
        items[tag] = (p, random_start(rng, kind, a, b, p))
    a = run_engine(psb.Engine(max_instances=32, pool_bytes=1 << 30, use_graph=True), items)
    b = run_engine(psb.Engine(max_instances=32, pool_bytes=1 << 30, use_graph=False), items)
    assert a == b and len(a) == 20


def test_directions_agree_with_single_instance():
    """Instances with bottom-up levels (the default) and with every level
    top-down give the same counts as psb_bfs, including Hanoi with symmetry,
    which never goes bottom-up."""
    rng = random.Random(77)
    items = {}
    for tag in range(28):
        kind, a, b = TYPES[tag % len(TYPES)]
        if (kind, a) == ("sliding", 4):
            continue
        p = make(kind, a, b)
        items[tag] = (p, random_start(rng, kind, a, b, p))
    auto = run_engine(psb.Engine(max_instances=64, pool_bytes=2 << 30), items)
    top = run_engine(psb.Engine(max_instances=64, pool_bytes=2 << 30, direction="top_down"), items)
    assert auto == top and set(auto) == set(items)
    for tag, (p, start) in items.items():
        assert auto[tag] == psb.bfs(p, "two_bit", start, direction="top_down")["counts"], (tag, p.Name())
