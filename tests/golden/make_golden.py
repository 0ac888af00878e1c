#!/usr/bin/env python3
"""Generates tests/golden/reference_vectors.json.

Two sources, both from the reference project (lightln2/PuzzleSearch):

1. Golden vectors and known-answer tests written in the reference's own test
   files.  They are read as text and pulled out with regular expressions,
   then stored with the file:line they came from.
2. Per-depth counts and Expand batches produced by running the reference's own CPU
   path.  It is built from its sources into oracle/_ref/ by oracle/build_ref.sh.

Usage:  python tests/golden/make_golden.py [--reference DIR] [--skip-ref-runs]

It must run where the reference sources are available.  The JSON it writes is
committed, so tests never need the reference at run time.
"""
import argparse
import ctypes
import json
import os
import random
import re
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))


def lineno(text, pos):
    return text.count("\n", 0, pos) + 1


def ints(s):
    return [int(x) for x in s.split()]


def search_vectors(ref):
    """PuzzlesTests/PuzzleSearchTests.cpp: per-depth count vectors."""
    path = "PuzzlesTests/PuzzleSearchTests.cpp"
    text = open(os.path.join(ref, path)).read()
    out = []
    consts = {}
    for m in re.finditer(r'static std::string (ST\dx\d) = "([0-9 ]+)";', text):
        consts[m.group(1)] = (ints(m.group(2)), lineno(text, m.start()))
    for name, (vec, ln) in consts.items():
        w, h = int(name[2]), int(name[4])
        out.append({"puzzle": ["sliding", w, h], "start": " ".join(str(i) for i in range(w * h)),
                    "counts": vec, "full": True, "source": f"{path}:{ln}"})
    # Hanoi / pancake vectors: the TEST body holds the puzzle, maxSteps and the string.
    for m in re.finditer(r"TEST\((\w+), (\w+)\) \{(.*?)\n\}", text, re.S):
        body = m.group(3)
        e = re.search(r'EXPECT_EQ\(ToString\(result\), "([0-9 ]+)"\)', body)
        if not e:
            continue
        vec = ints(e.group(1))
        ln = lineno(text, m.start() + len(m.group(0)) - len(body) - 2 + e.start())
        ms = re.search(r"maxSteps = (\d+)", body)
        hp = re.search(r"FourPegHanoi\w*? puzzle\((\d+)(?:, (true|false))?\)", body)
        pp = re.search(r"Pancake\w*? puzzle\((\d+)", body)
        if hp:
            spec = ["hanoi4", int(hp.group(1)), 1 if hp.group(2) == "true" else 0]
        elif pp:
            spec = ["pancake", int(pp.group(1)), 0]
        else:
            continue
        item = {"puzzle": spec, "start": None, "counts": vec, "full": ms is None,
                "source": f"{path}:{ln}", "test": f"{m.group(1)}.{m.group(2)}"}
        if not any(o["puzzle"] == spec and o["counts"] == vec for o in out):
            out.append(item)
    return out


def legacy_sliding_vectors(ref):
    """SlidingPuzzleTests/TestFrontierSearch.cpp: TestSearch<w, h>(radius, "counts", opts)."""
    path = "SlidingPuzzleTests/TestFrontierSearch.cpp"
    text = open(os.path.join(ref, path)).read()
    out = []
    for m in re.finditer(r"TEST\(TestFrontierSearch, (\w+)\) \{(.*?)\n\}", text, re.S):
        body = m.group(2)
        t = re.search(r'TestSearch<(\d+), (\d+)>\((\d+),\s*"([0-9 ]+)"', body, re.S)
        if not t:
            continue
        w, h = int(t.group(1)), int(t.group(2))
        iv = re.search(r'InitialValue = "([0-9 ]+)"', body)
        md = re.search(r"MaxDepth = (\d+)", body)
        start = " ".join(iv.group(1).split()) if iv else " ".join(str(i) for i in range(w * h))
        ln = lineno(text, m.start())
        out.append({"puzzle": ["sliding", w, h], "start": start, "counts": ints(t.group(4)),
                    "full": md is None, "radius": int(t.group(3)), "source": f"{path}:{ln}",
                    "test": m.group(1)})
    return out


def hanoi_legacy_vectors(ref):
    """HanoiTowersTests/HanoiSearchTests.cpp: full (symmetry-restored) prefixes."""
    path = "HanoiTowersTests/HanoiSearchTests.cpp"
    text = open(os.path.join(ref, path)).read()
    out = []
    for m in re.finditer(r"TEST\(HanoiSearchTests, Search(\d+)\) \{(.*?)\n\}", text, re.S):
        body = m.group(2)
        e = re.search(r'expected = "([0-9 ]+)"', body)
        ms = re.search(r"maxSteps = (\d+)", body)
        if not e:
            continue
        out.append({"puzzle": ["hanoi4", int(m.group(1)), 0], "start": None, "counts": ints(e.group(1)),
                    "full": False, "max_steps": int(ms.group(1)) if ms else None,
                    "source": f"{path}:{lineno(text, m.start())}", "test": f"Search{m.group(1)}"})
    return out


def expand_kats(ref):
    """Known-answer Expand tests: parent state -> ordered children states + ops."""
    out = []
    files = {"PuzzlesTests/PancakeTest.cpp": "pancake", "PuzzlesTests/FourPegHanoiTest.cpp": "hanoi4",
             "PuzzlesTests/SlidingPuzzleTest.cpp": "sliding"}
    for path, kind in files.items():
        text = open(os.path.join(ref, path)).read()
        for m in re.finditer(r"TEST\((\w+), (\w+)\) \{(.*?)\n\}", text, re.S):
            body = m.group(3)
            ctor = re.search(r"(\w+) puz\(([^)]*)\);", body)
            tctor = re.search(r"(\w+)<(\d+), (\d+)> puz;", body)  # SlidingTilePuzzleOptimized<w, h>
            if not ctor and not tctor:
                continue
            if tctor:
                cls, args = tctor.group(1), [tctor.group(2), tctor.group(3)]
            else:
                cls, args = ctor.group(1), [a.strip() for a in ctor.group(2).split(",") if a.strip()]
            if tctor:
                spec = ["sliding_opt", int(args[0]), int(args[1])]
            elif kind == "pancake":
                spec = ["pancake", int(args[0]), 0]
            elif kind == "hanoi4":
                spec = ["hanoi4", int(args[0]), 1 if len(args) > 1 and args[1] == "true" else 0]
            else:
                spec = ["sliding", int(args[0]), int(args[1])]
            # parent state
            ps = re.search(r'(?:puz\.Parse\(|stateStr = )"([0-9 ]+)"', body)
            if ps:
                parent = ps.group(1)
            elif re.search(r"auto index = 0;", body):
                parent = None  # index 0
            else:
                continue
            kids = {int(k): s for s, k in re.findall(r'EXPECT_EQ\("([0-9 ]+)", puz\.ToString\(children\[(\d+)\]\)\)', body)}
            ops = {int(k): int(v) for v, k in re.findall(r"EXPECT_EQ\((\d+), ops\[(\d+)\]\)", body)}
            invalid = [int(k) for k in re.findall(r"EXPECT_EQ\(puz\.INVALID_INDEX, children\[(\d+)\]\)", body)]
            pidx = re.search(r"EXPECT_EQ\(index, (\d+)\);", body)
            if not kids:
                continue
            # GPU classes emit fixed slots padded with INVALID_INDEX: keep only valid slots, in order.
            order = sorted(kids)
            item = {"class": cls, "puzzle": spec, "parent": parent,
                    "parent_index": int(pidx.group(1)) if pidx else None,
                    "children": [kids[k] for k in order],
                    "ops": [ops.get(k) for k in order],
                    "complete": not invalid and cls.endswith(("Simple",)) is False or True,
                    "source": f"{path}:{lineno(text, m.start())}", "test": f"{m.group(1)}.{m.group(2)}"}
            # Only the Simple classes promise the Simple index; for other classes the
            # states (strings) are what the test pins, and the index is not compared.
            item["index_pinned"] = cls.endswith("Simple")
            # The sliding Simple4x4 / Simple3x2 tests only list some children.
            item["prefix_only"] = kind == "sliding" or (kind == "pancake" and cls != "PancakeSimple" and spec[1] == 15)
            out.append(item)
    return out


def permutation_kats(ref):
    path = "PuzzlesTests/PermutationMapTest.cpp"
    text = open(os.path.join(ref, path)).read()
    compact = [{"perm": ints(a), "compact": ints(b), "source": f"{path}:{lineno(text, m.start())}"}
               for m in re.finditer(r'TestCompact\("([0-9 ]+)", "([0-9 ]+)"\);', text)
               for a, b in [m.groups()]]
    rank = []
    for m in re.finditer(r'TestRank\("([0-9 ]+)", ([^;]+)\);', text):
        expr = m.group(2).replace("ui64", "")
        val = eval(expr, {"__builtins__": {}})
        rank.append({"perm": ints(m.group(1)), "rank": val, "source": f"{path}:{lineno(text, m.start())}"})
    return {"compact": compact, "rank": rank}


def streamvint_kats(ref):
    path = "CommonTests/StreamVIntTests.cpp"
    text = open(os.path.join(ref, path)).read()
    tuples = []
    for m in re.finditer(r"TestTuple\(\{([^}]*)\}, (\d+)\);", text):
        vals = [int(x.strip(), 0) for x in m.group(1).split(",")]
        tuples.append({"values": vals, "bytes": int(m.group(2)), "source": f"{path}:{lineno(text, m.start())}"})
    lists = []
    for m in re.finditer(r"TestIndexesTuples\(\s*\{(.*?)\},\s*(\d+)\);", text, re.S):
        vals = [int(x.strip(), 0) for x in m.group(1).split(",") if x.strip()]
        lists.append({"values": vals, "bytes": int(m.group(2)), "source": f"{path}:{lineno(text, m.start())}"})
    bounds = []
    for m in re.finditer(r"TestBoundsTuple\(\{([^}]*)\}\);", text):
        bounds.append({"values": [int(x) for x in m.group(1).split(",")], "source": f"{path}:{lineno(text, m.start())}"})
    return {"tuples": tuples, "tuple_lists": lists, "bounds_tuples": bounds}


def compression_kats(ref):
    path = "CommonTests/CompressionTests.cpp"
    text = open(os.path.join(ref, path)).read()
    m = re.search(r'std::string str = "([0-9 ]+)";', text)
    large = [int(x) & 0xFFFFFFFF for x in m.group(1).split()]
    return {"large_range": {"values": large, "source": f"{path}:{lineno(text, m.start())}"},
            "bitmap_stride": {"stride": 7, "count": 150, "is_bitmap": True, "source": f"{path}:{lineno(text, text.index('TestCompression_Map'))}"},
            "svi_stride": {"stride": 11, "count": 150, "is_bitmap": False, "source": f"{path}:{lineno(text, text.index('TestCompression_StreamVInt'))}"},
            "bitmap_small": {"values": [7, 8, 32, 39, 177, 999, 1000, 1001, 1002, 1005], "source": f"{path}:{lineno(text, text.index('TestBitmapCompression'))}"},
            "out_of_order": {"values": [100, 10000, 2500, 2, 20000], "result": -1, "source": f"{path}:{lineno(text, text.index('OutOfOrder'))}"},
            "same_begin_end": {"values": [100, 10000, 2500, 2, 100], "result": -1, "source": f"{path}:{lineno(text, text.index('SameBeginningEnd'))}"}}


def opbits_kats(ref):
    """CommonTests/CompressionOpBitsTests.cpp: OpBitsCompression<BITS> round
    trips with their encoded sizes."""
    path = "CommonTests/CompressionOpBitsTests.cpp"
    text = open(os.path.join(ref, path)).read()
    out = []
    for m in re.finditer(r"TestOpBits<(\d)>\(\{([^}]*)\}, (\d+)\);", text):
        out.append({"bits": int(m.group(1)), "values": [int(x) for x in m.group(2).split(",")],
                    "bytes": int(m.group(3)), "source": f"{path}:{lineno(text, m.start())}"})
    return out


def bitarray_kat(ref):
    path = "CommonTests/TestBoolArray.cpp"
    text = open(os.path.join(ref, path)).read()
    m = re.search(r"res == (\d+)ui64", text)
    return {"size": 1 << 32, "stride": 13, "index_sum": int(m.group(1)), "source": f"{path}:{lineno(text, m.start())}"}


# ---------------------------------------------------------------------------
# Runs of the reference's own CPU path (oracle/_ref).
# ---------------------------------------------------------------------------
KIND = {"sliding": 1, "pancake": 2, "hanoi4": 3}
ALGO = {"two_bit": 1, "three_bit": 2, "frontier": 3, "classic": 4}


def load_ref():
    path = os.path.join(REPO, "oracle", "_ref", "libpsbref.so")
    if not os.path.exists(path):
        subprocess.check_call(["bash", os.path.join(REPO, "oracle", "build_ref.sh")])
    lib = ctypes.CDLL(path)
    lib.ref_bfs.argtypes = [ctypes.c_int] * 4 + [ctypes.c_char_p, ctypes.POINTER(ctypes.c_uint64), ctypes.c_int, ctypes.c_int]
    lib.ref_to_string.argtypes = [ctypes.c_int] * 3 + [ctypes.c_uint64, ctypes.c_char_p, ctypes.c_int]
    lib.ref_parse.argtypes = [ctypes.c_int] * 3 + [ctypes.c_char_p, ctypes.POINTER(ctypes.c_uint64)]
    lib.ref_expand.restype = ctypes.c_int64
    lib.ref_expand.argtypes = [ctypes.c_int] * 3 + [ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint32),
                                                    ctypes.c_uint64, ctypes.POINTER(ctypes.c_uint64),
                                                    ctypes.POINTER(ctypes.c_uint32), ctypes.c_uint64]
    return lib


def ref_bfs(lib, spec, algo, start):
    kind, a, b = KIND[spec[0]], spec[1], spec[2]
    if start is None:
        buf = ctypes.create_string_buffer(512)
        lib.ref_to_string(kind, a, b, 0, buf, 512)
        start = buf.value.decode()
    counts = (ctypes.c_uint64 * 4096)()
    n = lib.ref_bfs(kind, a, b, ALGO[algo], start.encode(), counts, 4096, 1)
    assert n > 0, (spec, algo, n)
    return start, list(counts[:n])


def sliding_solvable_start(rng, w, h):
    """A uniformly random permutation in the same reachable class as the solved
    state.  Parity rule for the blank-tile puzzle with the blank counted as tile 0:
    the permutation parity must equal the parity of the blank's taxicab distance from
    cell 0.  The result is confirmed by the reference BFS, whose reached-state count
    is N/2 for every start in that class."""
    n = w * h
    while True:
        p = list(range(n))
        rng.shuffle(p)
        inv = sum(1 for i in range(n) for j in range(i + 1, n) if p[i] > p[j])
        b = p.index(0)
        if inv % 2 == (b // w + b % w) % 2:
            return " ".join(map(str, p))


def ref_runs(lib):
    rng = random.Random(20261203)
    runs = []
    cases = [
        (["sliding", 2, 2], ["two_bit", "three_bit", "frontier", "classic"], [None]),
        (["sliding", 3, 2], ["two_bit", "three_bit", "frontier", "classic"], [None, "1 0 2 3 4 5"]),
        (["sliding", 4, 2], ["two_bit", "three_bit", "frontier", "classic"], [None]),
        (["sliding", 3, 3], ["two_bit", "three_bit", "frontier", "classic"], [None, "1 2 3 4 0 5 6 7 8"]),
        (["sliding", 5, 2], ["two_bit", "three_bit"], [None]),
        (["pancake", 2, 0], ["two_bit", "three_bit", "classic"], [None]),
        (["pancake", 5, 0], ["two_bit", "three_bit", "classic"], [None]),
        (["pancake", 7, 0], ["two_bit", "three_bit", "classic"], [None, "5 1 3 6 0 2 4"]),
        (["pancake", 8, 0], ["two_bit", "three_bit"], [None]),
        (["pancake", 9, 0], ["two_bit", "three_bit"], [None]),
        (["pancake", 10, 0], ["three_bit"], [None]),
        (["hanoi4", 1, 0], ["two_bit", "three_bit", "frontier", "classic"], [None]),
        (["hanoi4", 5, 0], ["two_bit", "three_bit", "frontier", "classic"], [None]),
        (["hanoi4", 7, 1], ["two_bit", "three_bit", "frontier", "classic"], [None]),
        (["hanoi4", 8, 0], ["two_bit", "three_bit", "frontier", "classic"], [None]),
        (["hanoi4", 10, 1], ["two_bit", "three_bit", "frontier"], [None]),
        (["hanoi4", 11, 0], ["three_bit"], [None]),
    ]
    for spec, algos, starts in cases:
        for start in starts:
            for algo in algos:
                s, counts = ref_bfs(lib, spec, algo, start)
                runs.append({"puzzle": spec, "algo": algo, "start": s, "counts": counts,
                             "source": "oracle/_ref (reference InMemory BFS)"})
    # Seeded random solvable starts, the shape of the batched workload (small boards).
    for (w, h) in [(2, 3), (3, 2), (2, 4), (3, 3), (2, 5)]:
        for _ in range(3):
            s = sliding_solvable_start(rng, w, h)
            s, counts = ref_bfs(lib, ["sliding", w, h], "three_bit", s)
            assert sum(counts) * 2 == __import__("math").factorial(w * h)
            runs.append({"puzzle": ["sliding", w, h], "algo": "three_bit", "start": s, "counts": counts,
                         "source": "oracle/_ref (reference InMemory BFS), seeded random start"})
    for n in [7, 8, 9]:
        for _ in range(2):
            p = list(range(n))
            rng.shuffle(p)
            s, counts = ref_bfs(lib, ["pancake", n, 0], "two_bit", " ".join(map(str, p)))
            runs.append({"puzzle": ["pancake", n, 0], "algo": "two_bit", "start": s, "counts": counts,
                         "source": "oracle/_ref (reference InMemory BFS), seeded random start"})
    return runs


def ref_expand_batches(lib):
    """Reference Expand on seeded batches of parents with seeded operator bits."""
    rng = random.Random(7)
    out = []
    specs = [["sliding", 3, 2], ["sliding", 4, 4], ["sliding", 3, 4], ["pancake", 5, 0], ["pancake", 13, 0],
             ["pancake", 16, 0], ["hanoi4", 7, 0], ["hanoi4", 7, 1], ["hanoi4", 18, 0], ["hanoi4", 21, 1]]
    for spec in specs:
        kind, a, b = KIND[spec[0]], spec[1], spec[2]
        if spec[0] == "hanoi4":
            N, ops_n = 4 ** a, 4
        else:
            n = a * b if spec[0] == "sliding" else a
            N = __import__("math").factorial(n)
            ops_n = 4 if spec[0] == "sliding" else n - 1
        cnt = 64
        parents = [rng.randrange(N) for _ in range(cnt)]
        opbits = [rng.randrange(1 << ops_n) if i % 3 == 2 else 0 for i in range(cnt)]
        P = (ctypes.c_uint64 * cnt)(*parents)
        O = (ctypes.c_uint32 * cnt)(*opbits)
        cap = cnt * 16
        C = (ctypes.c_uint64 * cap)()
        CO = (ctypes.c_uint32 * cap)()
        n_out = lib.ref_expand(kind, a, b, P, O, cnt, C, CO, cap)
        assert n_out >= 0
        out.append({"puzzle": spec, "parents": parents, "opbits": opbits, "children": list(C[:n_out]),
                    "child_ops": list(CO[:n_out]), "source": "oracle/_ref (reference Puzzle::Expand)"})
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("PSB_REFERENCE"), required=not os.environ.get("PSB_REFERENCE"),
                    help="the reference project's source tree (or set PSB_REFERENCE)")
    ap.add_argument("--skip-ref-runs", action="store_true")
    args = ap.parse_args()
    ref = args.reference
    data = {
        "comment": "Golden vectors of lightln2/PuzzleSearch, extracted by tests/golden/make_golden.py",
        "search": search_vectors(ref),
        "legacy_sliding": legacy_sliding_vectors(ref),
        "legacy_hanoi": hanoi_legacy_vectors(ref),
        "expand_kats": expand_kats(ref),
        "permutation": permutation_kats(ref),
        "streamvint": streamvint_kats(ref),
        "compression": compression_kats(ref),
        "bitarray": bitarray_kat(ref),
        "opbits": opbits_kats(ref),
    }
    path = os.path.join(HERE, "reference_vectors.json")
    if args.skip_ref_runs and os.path.exists(path):  # keep the runs already recorded
        old = json.load(open(path))
        for key in ("ref_runs", "ref_expand"):
            if key in old:
                data[key] = old[key]
    if not args.skip_ref_runs:
        lib = load_ref()
        data["ref_runs"] = ref_runs(lib)
        data["ref_expand"] = ref_expand_batches(lib)
    with open(path, "w") as f:
        json.dump(data, f, indent=1)
    print(f"wrote {path}: " + ", ".join(f"{k}={len(v) if isinstance(v, list) else 'obj'}" for k, v in data.items()))


if __name__ == "__main__":
    sys.exit(main())
