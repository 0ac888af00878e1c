"""The C++ adapter (include/psb200.hpp) used the way the reference's own tests
use its classes: PuzzleSearchTests-style searches and Pancake/Hanoi Expand
known-answer tests, through tests/cpp/psb200_driver.cpp."""
import os
import subprocess

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVER = os.path.join(REPO, "tests", "cpp", "psb200_driver")


def build_driver():
    src = os.path.join(REPO, "tests", "cpp", "psb200_driver.cpp")
    if os.path.exists(DRIVER) and os.path.getmtime(DRIVER) >= max(
            os.path.getmtime(src), os.path.getmtime(os.path.join(REPO, "include", "psb200.hpp"))):
        return DRIVER
    subprocess.check_call(["g++", "-std=c++17", "-O2", "-I" + os.path.join(REPO, "include"), src, "-o", DRIVER,
                           "-L" + os.path.join(REPO, "puzzlesearch_b200"), "-lpsb200",
                           "-Wl,-rpath,$ORIGIN/../../puzzlesearch_b200"])
    return DRIVER


def run(lines, cwd=None):
    out = subprocess.run([build_driver()], input="\n".join(lines) + "\n", capture_output=True, text=True,
                         timeout=600, check=True, cwd=cwd).stdout
    return out.strip().split("\n")


def test_driver_compiles():
    assert os.path.exists(build_driver())


@pytest.mark.gpu
def test_search_vectors_through_adapter(golden):
    cases = []
    for v in golden["search"]:
        kind, a, b = v["puzzle"]
        if not v["full"] or (kind == "sliding" and a * b > 10):
            continue
        algos = ["classic", "two_bit", "three_bit"] + (["frontier"] if kind != "pancake" else [])
        for algo in algos:
            cases.append((f"bfs {kind} {a} {b} {algo} {v['start'] or ''}".rstrip(), v["counts"]))
    got = run([c for c, _ in cases])
    assert len(got) == len(cases)
    for (cmd, exp), line in zip(cases, got):
        assert [int(x) for x in line.split()] == exp, cmd


@pytest.mark.gpu
def test_expand_known_answers_through_adapter(golden):
    kats = [k for k in golden["expand_kats"] if k["puzzle"][0] != "sliding"]
    cmds = [f"expand {k['puzzle'][0]} {k['puzzle'][1]} {k['puzzle'][2]} {k['parent'] or ''}".rstrip() for k in kats]
    got = run(cmds)
    for k, line in zip(kats, got):
        items = [x.split("|") for x in line.split(";")]
        states = [s for s, _ in items]
        assert states[:len(k["children"])] == k["children"], k["test"]
        for (s, op), e in zip(items, k["ops"]):
            if e is not None:
                assert int(op) == e, k["test"]


@pytest.mark.gpu
def test_error_path_through_adapter():
    got = run(["bfs pancake 6 0 frontier"])
    assert got[0].startswith("ERROR -5")


@pytest.mark.gpu
def test_reference_gpu_class_bodies_through_adapter(golden):
    """The reference's GPU test bodies (PuzzlesTests/PuzzleSearchTests.cpp:85-131)
    construct SlidingTilePuzzleGpu(w, h) and run every in-memory search on it;
    FourPegHanoiGPU(n, symmetry) takes the Simple class's index space as well.
    Through the adapter they give the reference's golden vectors."""
    cases = []
    for v in golden["search"]:
        kind, a, b = v["puzzle"]
        if not v["full"] or kind == "pancake" or (kind == "sliding" and a * b > 8):
            continue
        gpu_kind = {"sliding": "sliding_gpu", "hanoi4": "hanoi4_gpu"}[kind]
        for algo in ("classic", "two_bit", "three_bit", "frontier"):
            cases.append((f"bfs {gpu_kind} {a} {b} {algo} {v['start'] or ''}".rstrip(), v["counts"]))
    assert len(cases) >= 12
    got = run([c for c, _ in cases])
    for (cmd, exp), line in zip(cases, got):
        assert [int(x) for x in line.split()] == exp, cmd


def test_caller_defined_puzzle():
    """Puzzle is abstract as in the reference: a caller's own subclass runs
    through ExpandBuffer (every state's two children delivered), and the
    in-memory searches, which need a device expander, reject it with
    PSB_ERR_UNSUPPORTED instead of running it on the host."""
    line = run(["custom 5000"])[0]
    children, rest = line.split(" ", 1)
    assert int(children) == 10000
    assert rest.startswith("ERROR -5")


@pytest.mark.gpu
def test_gpu_class_limits_and_names():
    got = run(["bfs hanoi4_gpu 25 0 two_bit", "expand sliding_gpu 3 2 1 0 2 3 4 5"])
    assert got[0].startswith("ERROR -1")
    assert got[1] == run(["expand sliding 3 2 1 0 2 3 4 5"])[0]


@pytest.mark.gpu
def test_hanoi_search_through_adapter(golden):
    """HanoiSearch<size> as the reference's HanoiSearchTests call it
    (HanoiTowers<17>::ToString(0), maxSteps = 120), and a full search whose
    counts equal the oracle's search without symmetry."""
    import oracle as O
    v = [x for x in golden["legacy_hanoi"] if x["puzzle"] == ["hanoi4", 17, 0]][0]
    got = run(["hanoisearch 17 120", "hanoisearch 11 0"])
    assert [int(x) for x in got[0].split()] == v["counts"]
    assert [int(x) for x in got[1].split()] == O.bfs(["hanoi4", 11, 0], "two_bit")[0]


@pytest.mark.gpu
def test_disk_based_bodies_through_adapter(golden, tmp_path):
    """The reference's disk-based test bodies (PuzzlesTests/PuzzleSearchTests.cpp:
    133-333): PuzzleOptions with segmentBits 15..22 and threads 1 or 4, on
    SlidingTilePuzzleGpu(5, 2), the Simple class and
    SlidingTilePuzzleOptimized<5, 2>, give ST5x2.  Their default StoreOptions
    put the segment files in the working directory; none is left behind."""
    v = [x for x in golden["search"] if x["puzzle"] == ["sliding", 5, 2]][0]
    cmds = []
    for kind in ("sliding_gpu", "sliding", "sliding_opt"):
        for algo in ("Classic", "TwoBit", "ThreeBit", "FrontierSearch", "OptFrontierSearch", "OptThreeBit"):
            for bits, threads in ((22, 1), (19, 1), (19, 4), (15, 1)):
                if kind == "sliding_opt" and bits == 15:
                    continue
                cmds.append(f"disk {kind} 5 2 {algo} {bits} {threads} 0 1 2 3 4 5 6 7 8 9")
    got = run(cmds, cwd=str(tmp_path))
    for cmd, line in zip(cmds, got):
        assert [int(x) for x in line.split()] == v["counts"], cmd
    assert os.listdir(tmp_path) == []
