"""The solve server (psb_server_*): continuous batching.  Requests that arrive
while others are on the GPU are admitted as slots and pool space free up, and
every result (per-depth counts, eccentricity) must be exactly what the same
search gives alone (psb_bfs, two-bit).  Integer results: exact."""
import random
import time

import pytest

import puzzlesearch_b200 as psb

pytestmark = pytest.mark.gpu

TYPES = [("sliding", 2, 4), ("sliding", 3, 3), ("sliding", 2, 5), ("sliding", 3, 4),
         ("pancake", 8, 0), ("pancake", 9, 0), ("pancake", 10, 0), ("pancake", 11, 0), ("pancake", 12, 0),
         ("hanoi4", 8, 0), ("hanoi4", 10, 0), ("hanoi4", 12, 0), ("hanoi4", 14, 0)]


def make(kind, a, b):
    return {"sliding": lambda: psb.SlidingTilePuzzleSimple(a, b), "pancake": lambda: psb.PancakeSimple(a),
            "hanoi4": lambda: psb.FourPegHanoiSimple(a, bool(b))}[kind]()


def start(rng, kind, a, b, p):
    if kind != "sliding":
        return rng.randrange(p.IndexesCount())
    while True:
        perm = list(range(a * b))
        rng.shuffle(perm)
        inv = sum(1 for i in range(len(perm)) for j in range(i + 1, len(perm)) if perm[i] > perm[j])
        z = perm.index(0)
        if inv % 2 == (z // a + z % a) % 2:
            return p.Parse(" ".join(map(str, perm)))


def test_results_alone_equal_results_in_the_mix():
    rng = random.Random(77)
    puzzles = {t: make(*t) for t in TYPES}
    srv = psb.Server(max_instances=64, pool_bytes=4 << 30)
    reqs = {}
    for i in range(40):
        t = TYPES[rng.randrange(len(TYPES))]
        s = start(rng, *t, puzzles[t])
        reqs[srv.submit(puzzles[t], s)] = (t, s)
        time.sleep(rng.random() * 0.01)  # later requests arrive while earlier ones run
    done = {}
    deadline = time.time() + 300
    while len(done) < len(reqs) and time.time() < deadline:
        done.update(srv.poll())
        time.sleep(0.005)
    info = srv.info()
    srv.stop()
    assert len(done) == len(reqs), info
    for ticket, (t, s) in reqs.items():
        status, counts, latency = done[ticket]
        assert status == 0
        assert counts == psb.bfs(puzzles[t], "two_bit", s)["counts"], (t, s)
        assert latency > 0
    assert info["steps"] > 0


def test_unsupported_request_fails_alone():
    """Without a large lane the engine rejects a puzzle it has no kernels
    for; with one, the large lane takes it and reports that its arrays do
    not fit the device (4x4: 16! states).  The other request completes."""
    for lane, code in ((None, -5), (0, -3)):
        srv = psb.Server(max_instances=8, pool_bytes=1 << 30, large_states=lane)
        ok = srv.submit(psb.PancakeSimple(9), 0)
        bad = srv.submit(psb.SlidingTilePuzzleSimple(4, 4), 0)  # 16 cells: not compiled into the engine
        done = {}
        deadline = time.time() + 60
        while len(done) < 2 and time.time() < deadline:
            done.update(srv.poll())
            time.sleep(0.005)
        srv.stop()
        assert done[bad][0] == code
        assert done[ok][0] == 0 and done[ok][1] == psb.bfs(psb.PancakeSimple(9), "two_bit", 0)["counts"]


def test_admission_waits_for_pool_space():
    """A pool with room for one 12-pancake array at a time still completes all
    requests: the rest wait in the queue until space frees up."""
    p = psb.PancakeSimple(11)
    foot = psb.Engine.footprint(p)
    srv = psb.Server(max_instances=16, pool_bytes=foot + 4096)
    tickets = [srv.submit(p, s) for s in (0, 1, 2, 3)]
    done = {}
    deadline = time.time() + 120
    while len(done) < 4 and time.time() < deadline:
        done.update(srv.poll())
        time.sleep(0.005)
    srv.stop()
    assert [done[t][1] for t in tickets] == [psb.bfs(p, "two_bit", s)["counts"] for s in (0, 1, 2, 3)]


def test_request_larger_than_the_pool_fails_at_once():
    """A request whose footprint exceeds the whole pool completes at once with
    PSB_ERR_NOMEM; the requests submitted before and after it all complete
    with their correct counts, and the server stays responsive."""
    small = psb.PancakeSimple(9)
    big = psb.PancakeSimple(12)  # 120 MB of codes: never fits a 16 MB pool
    foot = psb.Engine.footprint(small)
    srv = psb.Server(max_instances=8, pool_bytes=16 << 20, large_states=None)  # every request in the batch lane
    assert psb.Engine.footprint(big) > 16 << 20 > 2 * foot
    before = [srv.submit(small, s) for s in (0, 5)]
    bad = srv.submit(big, 0)
    after = [srv.submit(small, s) for s in (7, 11, 13)]
    done = {}
    deadline = time.time() + 60
    while len(done) < 6 and time.time() < deadline:
        done.update(srv.poll())
        time.sleep(0.005)
    info = srv.info()
    srv.stop()
    assert len(done) == 6, info
    assert done[bad][0] == -3
    for t, s in zip(before + after, (0, 5, 7, 11, 13)):
        assert done[t][0] == 0 and done[t][1] == psb.bfs(small, "two_bit", s)["counts"]


def test_small_requests_pass_a_waiting_large_one():
    """While a large request waits for pool space, smaller ones that fit are
    admitted around it; the large one still completes once space frees up."""
    small, large = psb.PancakeSimple(8), psb.PancakeSimple(10)
    fl, fs = psb.Engine.footprint(large), psb.Engine.footprint(small)
    srv = psb.Server(max_instances=16, pool_bytes=fl + 2 * fs + 4096)
    first = srv.submit(large, 0)      # takes most of the pool
    waiting = srv.submit(large, 1)    # must wait for the first to finish
    smalls = [srv.submit(small, s) for s in range(6)]
    done = {}
    deadline = time.time() + 120
    while len(done) < 8 and time.time() < deadline:
        done.update(srv.poll())
        time.sleep(0.002)
    srv.stop()
    assert len(done) == 8
    assert done[first][1] == psb.bfs(large, "two_bit", 0)["counts"]
    assert done[waiting][1] == psb.bfs(large, "two_bit", 1)["counts"]
    for s, t in enumerate(smalls):
        assert done[t][0] == 0 and done[t][1] == psb.bfs(small, "two_bit", s)["counts"]


def test_large_lane_and_batch_lane_together():
    """Requests above large_states run one at a time as single searches on
    their own stream while the others batch in the engine; every result
    equals the search alone, whichever lane ran it."""
    rng = random.Random(9)
    small = [psb.PancakeSimple(8), psb.SlidingTilePuzzleSimple(3, 3), psb.FourPegHanoiSimple(8)]
    large = [psb.PancakeSimple(10), psb.FourPegHanoiSimple(11)]
    srv = psb.Server(max_instances=32, pool_bytes=1 << 30, large_states=1 << 20)
    reqs = {}
    for i in range(30):
        p = (large if i % 5 == 0 else small)[rng.randrange(2 if i % 5 == 0 else 3)]
        st = 0 if p.Name().startswith("Sliding") else rng.randrange(p.IndexesCount())
        reqs[srv.submit(p, st)] = (p, st)
    done = {}
    deadline = time.time() + 120
    while len(done) < len(reqs) and time.time() < deadline:
        done.update(srv.poll())
        time.sleep(0.002)
    info = srv.info()
    srv.stop()
    assert len(done) == len(reqs), info
    for t, (p, st) in reqs.items():
        assert done[t][0] == 0 and done[t][1] == psb.bfs(p, "two_bit", st)["counts"]
