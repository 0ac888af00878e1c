#!/usr/bin/env python3
"""Generates tests/golden/large_counts.json: full per-depth counts of the
large searches, produced by the reference's own CPU code.

    python tests/golden/make_large_fixtures.py [--threads T] [--only NAME ...]
    python tests/golden/make_large_fixtures.py --record NAME OUTPUT_FILE SECONDS

Each entry is the complete per-depth count vector of one search, with the
program that made it, its wall time and the host it ran on:

* 13-pancake (13! states): the reference's unmodified single-threaded
  InMemoryThreeBitBFS (oracle/_ref/psbref, hours on one core).
* 18-disk 4-peg Hanoi (4^18 states) and 14-pancake (14! states): the
  reference's own *Simple puzzle classes and ExpandBuffer driven by a
  multi-threaded restatement of InMemoryThreeBitBFS's level loop
  (oracle/_ref/psbref_mt, oracle/ref_mt_bfs.cpp).  The single-threaded
  reference needs 7-9 hours and 26-33 GB for each of these.  psbref_mt's
  counts equal the unmodified reference's on every search the tests compare
  (tests/test_oracle.py), and the 18-disk vector's first 121 depths equal the
  reference's own golden prefix (HanoiTowersTests/HanoiSearchTests.cpp:25-33).

Both programs are built from the reference's sources by oracle/build_ref.sh.
The runs are long: start this in the background, or run the programs
yourself and add each finished run's JSON line with --record.  Searches run
one after the other (18-disk Hanoi needs 26 GB of host memory, 14-pancake
33 GB).  Results already in the JSON are kept unless --only names them.
"""
import argparse
import json
import os
import platform
import subprocess
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
OUT = os.path.join(HERE, "large_counts.json")
REF = os.path.join(REPO, "oracle", "_ref")

# name: (puzzle spec, algorithm, program, CLI arguments)
SEARCHES = {
    "pancake13": (["pancake", 13, 0], "three_bit", "psbref", ["2", "13", "0", "2"]),
    "hanoi18": (["hanoi4", 18, 0], "three_bit", "psbref_mt", ["3", "18", "0", "{threads}"]),
    "pancake14": (["pancake", 14, 0], "three_bit", "psbref_mt", ["2", "14", "0", "{threads}"]),
}


def entry(name, result, threads, seconds):
    spec, algo, prog, argv = SEARCHES[name]
    args = [a.format(threads=threads) for a in argv]
    return {"puzzle": spec, "algo": algo, "start": 0, "counts": result["counts"], "states": result["states"],
            "program": f"oracle/_ref/{prog} " + " ".join(args),
            "kind": "reference InMemoryThreeBitBFS" if prog == "psbref"
                    else "reference puzzle classes and ExpandBuffer, multi-threaded three-bit level loop",
            "threads": 1 if prog == "psbref" else threads, "seconds": round(seconds, 1),
            "host": f"{platform.machine()}, {os.cpu_count()} CPUs"}


def run(name, threads):
    spec, algo, prog, argv = SEARCHES[name]
    cmd = [os.path.join(REF, prog)] + [a.format(threads=threads) for a in argv]
    t0 = time.time()
    out = subprocess.run(cmd, check=True, capture_output=True, text=True).stdout
    return entry(name, json.loads(out.strip().splitlines()[-1]), threads, time.time() - t0)


def load():
    if os.path.exists(OUT):
        return json.load(open(OUT))
    return {"comment": "Full per-depth counts of large searches from the reference's CPU code; "
                       "made by tests/golden/make_large_fixtures.py", "searches": {}}


def save(data):
    with open(OUT, "w") as f:
        json.dump(data, f, indent=1)
        f.write("\n")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--threads", type=int, default=max(1, (os.cpu_count() or 2) - 2))
    ap.add_argument("--only", nargs="*", default=None, choices=sorted(SEARCHES))
    ap.add_argument("--record", nargs=3, metavar=("NAME", "OUTPUT_FILE", "SECONDS"),
                    help="add a finished run: the program's JSON output line and its wall seconds")
    args = ap.parse_args()
    data = load()
    if args.record:
        name, path, secs = args.record
        result = json.loads(open(path).read().strip().splitlines()[-1])
        data["searches"][name] = entry(name, result, result.get("threads", args.threads), float(secs))
        save(data)
        return 0
    for name in args.only or list(SEARCHES):
        if args.only is None and name in data["searches"]:
            continue
        print(f"running {name} ...", file=sys.stderr, flush=True)
        data["searches"][name] = run(name, args.threads)
        save(data)
    return 0


if __name__ == "__main__":
    sys.exit(main())
