#!/usr/bin/env python3
"""Benchmark: full in-memory BFS of the 14-pancake puzzle (two-bit codes,
frontier spill) on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload NAME]

One step is one complete BFS from the identity (14! = 87,178,291,200 states,
17 depths, a 21.8 GB two-bit array resident in HBM), with every depth's
frontier encoded on the GPU into the reference's compressed segment stream
and handed over from pinned host memory (the large-instance configuration:
14-pancake and 18-disk 4-peg Hanoi two-bit with frontier compression).  The
metric is BFS states per second: states reached divided by device time.
`value` times psb_bfs_session_run with the arrays already allocated.  `e2e`
times the public C-ABI call psb_bfs, which allocates from the pool, runs,
copies every spilled segment and the per-depth counts to the host.

Multi-GPU: the path does not shard across GPUs inside one search (the
reference has no multi-GPU path), so --gpus N runs N independent replicas,
one process per GPU under torchrun.  value = total states / max-over-ranks time.

--impl reference times the reference's own CPU path: InMemoryTwoBitBFS built
from its sources into oracle/_ref.  The reference's in-memory search is
single-threaded, so every step runs one search per host core at once, on a
bounded sample (the full 10-pancake search) so the run ends in minutes; the
single-threaded 14-pancake search takes many hours.
"""
import argparse
import ctypes
import json
import math
import os
import re
import statistics
import subprocess
import sys
import threading
import time

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

WORKLOADS = {
    # name: (kind, a, b, algo, description); the two large instances spill every depth by default
    "pancake14-2bit": ("pancake", 14, 0, "two_bit", "14-pancake in-memory two-bit BFS, full solve from the identity"),
    "hanoi18-2bit": ("hanoi4", 18, 0, "two_bit", "18-disk 4-peg Hanoi in-memory two-bit BFS, full solve from all disks on peg 0"),
    "pancake13-3bit": ("pancake", 13, 0, "three_bit", "13-pancake in-memory three-bit BFS, full solve from the identity"),
    "sliding3x4-2bit": ("sliding", 3, 4, "two_bit", "3x4 sliding-tile in-memory two-bit BFS, full solve from the solved state"),
    # smaller cases of the same kernels, sized for ncu captures (arrays above L2, a few GB at most)
    "hanoi15-2bit": ("hanoi4", 15, 0, "two_bit", "15-disk 4-peg Hanoi in-memory two-bit BFS (profiling case)"),
    "pancake12-3bit": ("pancake", 12, 0, "three_bit", "12-pancake in-memory three-bit BFS (profiling case)"),
    "pancake13-2bit": ("pancake", 13, 0, "two_bit", "13-pancake in-memory two-bit BFS (profiling case)"),
    # the other two in-memory algorithms
    "hanoi16-frontier": ("hanoi4", 16, 0, "frontier", "16-disk 4-peg Hanoi in-memory frontier search, full solve"),
    "pancake12-classic": ("pancake", 12, 0, "classic", "12-pancake in-memory classic BFS, full solve from the identity"),
    "sliding4x3-frontier": ("sliding", 4, 3, "frontier", "4x3 sliding-tile in-memory frontier search, full solve"),
}
SPILL_BY_DEFAULT = {"pancake14-2bit", "hanoi18-2bit"}
# DRAM traffic (dram__bytes_read.sum + dram__bytes_write.sum) of the level
# kernels over one full search, from a one-pass ncu capture of the same search
# without spill (the level launches are the same with it); ncu cannot run
# inside the bench.  Used for roofline.traffic when the run has the same
# launches (same level count, window and shape defaults).
LEVEL_TRAFFIC = {
    "pancake14-2bit": {"bytes": 11978881712384, "launches": 17, "window_bits": 16, "threads": 128,
                       "profile": "profiles/level_kernel_pancake14_2bit_traffic.md"},
}
REF_SAMPLE = ("pancake", 11, 0, "two_bit")      # cpu_baseline: one reference InMemoryTwoBitBFS, one core
REF_ARM_SAMPLE = ("pancake", 10, 0, "two_bit")  # --impl reference: one search per host core per step


def load_peaks():
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """Samples nvidia-smi clocks and throttle reasons while the timed region runs."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup(n_gpus, backend="nccl"):
    """One process per GPU (torchrun): returns (rank, world, local_rank, torch.distributed or None)."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world != n_gpus:
        raise SystemExit(f"--gpus {n_gpus} but WORLD_SIZE={world}")
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
        pg = dist
    return rank, world, local, pg


def max_over_ranks(x, dist, device="cuda"):
    """The largest x over all ranks (the timing rule: a multi-GPU time is the slowest rank's)."""
    if not dist:
        return x
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(world, steps, units_per_step, seconds):
    """Whole-job throughput: every rank processes units_per_step per step (replicas, weak scaling)."""
    return world * steps * units_per_step / seconds


def _ref_cmd(sample):
    kind, a, b, algo = sample
    kinds = {"sliding": 1, "pancake": 2, "hanoi4": 3}
    algos = {"two_bit": 1, "three_bit": 2, "frontier": 3, "classic": 4}
    return [os.path.join(REPO, "oracle", "_ref", "psbref"), str(kinds[kind]), str(a), str(b), str(algos[algo])]


def cpu_reference_sample(sample=REF_SAMPLE):
    """Runs the reference's InMemory BFS (oracle/_ref/psbref) on the sample; returns (states, seconds, kind)."""
    kind, a, b, algo = sample
    cmd = _ref_cmd(sample)
    if os.path.exists(cmd[0]):
        out = subprocess.run(cmd, capture_output=True, text=True, check=True).stdout
        d = json.loads(out.strip().splitlines()[-1])
        return d["states"], d["seconds"], "reference"
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import oracle as O
    t0 = time.perf_counter()
    counts, _ = O.bfs([kind, a, b], algo, 0)
    return sum(counts), time.perf_counter() - t0, "port"


def reference_step(procs, sample=REF_ARM_SAMPLE):
    """One step of the reference arm: `procs` copies of the reference's
    single-threaded search at once, one per host core.  Returns (states, wall seconds)."""
    cmd = _ref_cmd(sample)
    t0 = time.perf_counter()
    running = [subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
               for _ in range(procs)]
    states = 0
    for p in running:
        out, _ = p.communicate()
        if p.returncode != 0:
            raise RuntimeError(f"reference search failed: {' '.join(cmd)}")
        states += json.loads(out.strip().splitlines()[-1])["states"]
    return states, time.perf_counter() - t0


def host_cores():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def run_reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    kind, a, b, algo = REF_ARM_SAMPLE
    wl = WORKLOADS[args.workload]
    if not os.path.exists(_ref_cmd(REF_ARM_SAMPLE)[0]):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/psbref was not built (the reference's "
                          "sources were absent when the repository was built)"}), flush=True)
        return 0
    procs = host_cores()
    for _ in range(args.warmup):
        reference_step(procs)
    secs, states = 0.0, 0
    for _ in range(args.steps):
        s, t = reference_step(procs)
        states += s
        secs += t
    value = states / secs
    sample = (f"reference InMemoryTwoBitBFS on {a}-pancake (full search, {math.factorial(a):,} states), "
              f"{procs} single-threaded searches at once, one per host core, per step")
    line = {
        "impl": "reference", "metric": f"BFS states/sec ({wl[4]})", "value": value, "unit": "states/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * secs / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": "synthetic",
        "config": {"workload": args.workload, "sample": sample, "same_config": False,
                   "why_not_same_config": "the reference's single-threaded in-memory search of the full workload "
                                          "takes hours; the sample runs the same algorithm on a smaller instance of "
                                          "the same puzzle, whose arrays fit the host caches (a faster rate per "
                                          "state than the full instance would reach)"},
        "cpu_baseline": {"value": value, "unit": "states/s", "cores": procs, "kind": "reference", "sample": sample},
        "e2e": {"value": value, "unit": "states/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


BATCH_TYPES = [("sliding", 2, 3), ("sliding", 2, 4), ("sliding", 3, 3), ("sliding", 2, 5),
               ("pancake", 7, 0), ("pancake", 8, 0), ("pancake", 9, 0), ("pancake", 10, 0), ("pancake", 11, 0)]


def _make(psb, kind, a, b):
    return {"pancake": lambda: psb.PancakeSimple(a), "sliding": lambda: psb.SlidingTilePuzzleSimple(a, b),
            "hanoi4": lambda: psb.FourPegHanoiSimple(a, bool(b))}[kind]()


def solvable_start(rng, kind, a, b, puzzle):
    """Uniformly random start in the start state's component: any permutation
    for pancake; for the sliding tile, permutation parity must equal the
    parity of the blank's taxicab distance from cell 0."""
    if kind != "sliding":
        return rng.randrange(puzzle.IndexesCount())
    while True:
        p = list(range(a * b))
        rng.shuffle(p)
        inv = sum(1 for i in range(len(p)) for j in range(i + 1, len(p)) if p[i] > p[j])
        z = p.index(0)
        if inv % 2 == (z // a + z % a) % 2:
            return puzzle.Parse(" ".join(map(str, p)))


def batch_bench(args):
    """Batched solves: 4096 independent two-bit searches drawn from a seed,
    uniform over sliding 2x3/2x4/3x3/2x5 and pancake 7..11, from random
    solvable starts; batched engine vs one search per launch, counts equal."""
    import random

    import puzzlesearch_b200 as psb
    rng = random.Random(4096)
    puzzles = {t: _make(psb, *t) for t in BATCH_TYPES}
    items = []
    for i in range(args.instances):
        t = BATCH_TYPES[rng.randrange(len(BATCH_TYPES))]
        items.append((i, t, solvable_start(rng, *t, puzzles[t])))
    total_states = sum(puzzles[t].IndexesCount() // (2 if t[0] == "sliding" else 1) for _, t, _ in items)
    direction = "top_down" if args.direction == "top_down" else "auto"
    blocks_per_sm, wb_offset, tuning = 0, 0, None
    if args.autotune:  # launch shape picked on a separate calibration batch (another seed)
        from puzzlesearch_b200 import autotune
        crng = random.Random(77)
        calib = []
        for _ in range(min(1024, args.instances)):
            t = BATCH_TYPES[crng.randrange(len(BATCH_TYPES))]
            calib.append((puzzles[t], solvable_start(crng, *t, puzzles[t])))
        (blocks_per_sm, wb_offset), timings = autotune.tune_engine(calib, pool_bytes=24 << 30, direction=direction)
        tuning = {"blocks_per_sm": blocks_per_sm, "window_bits_offset": wb_offset,
                  "calibration_instances": len(calib),
                  "seconds": {f"{k[0]} blocks/SM, window offset {k[1]}": round(v, 4) for k, v in timings.items()}}

    def run_batched():
        eng = psb.Engine(max_instances=args.instances, max_depths=128, pool_bytes=24 << 30,
                         blocks_per_sm=blocks_per_sm, direction=direction, window_bits_offset=wb_offset)
        t0 = time.perf_counter()
        for i, t, st in items:
            assert eng.add(puzzles[t], st, i)
        res = {}
        while len(res) < len(items):
            eng.step(8)
            res.update(eng.poll())
        dt = time.perf_counter() - t0
        levels = eng.info()["levels_run"]
        eng.close()
        return res, dt, levels

    sessions = {t: psb.BfsSession(puzzles[t], "two_bit") for t in BATCH_TYPES}

    def run_plain():
        t0 = time.perf_counter()
        res = {i: sessions[t].run(st)[0] for i, t, st in items}
        return res, time.perf_counter() - t0

    for _ in range(max(1, args.warmup - 2)):
        run_batched()
        run_plain()
    b_res, b_dt, levels = run_batched()
    p_res, p_dt = run_plain()
    assert b_res == p_res, "batched counts differ from the single-instance path"
    line = {"metric": f"batched solves/s ({len(items)} two-bit searches, sliding 2x3/2x4/3x3/2x5 + pancake 7..11)",
            "value": len(items) / b_dt, "unit": "solves/s", "n_gpus": 1, "steps": 1, "warmup": args.warmup,
            "higher_is_better": True, "dtype": "u64", "data": "seeded random solvable starts",
            "config": {"workload": "batch4096", "instances": len(items), "states": total_states,
                       "engine_levels": levels, "direction": direction,
                       "blocks_per_sm": blocks_per_sm or 2, "window_bits_offset": wb_offset,
                       "autotune": tuning},
            "batched": {"seconds": b_dt, "solves_per_s": len(items) / b_dt, "states_per_s": total_states / b_dt},
            "plain_one_per_launch": {"seconds": p_dt, "solves_per_s": len(items) / p_dt,
                                     "states_per_s": total_states / p_dt},
            "speedup_vs_plain": p_dt / b_dt, "counts_equal": True}
    print(json.dumps(line), flush=True)
    return 0


SERVE_TYPES = [("sliding", 2, 4), ("sliding", 3, 3), ("sliding", 2, 5), ("sliding", 3, 4)] + \
              [("pancake", n, 0) for n in range(8, 13)] + [("hanoi4", n, 0) for n in range(8, 15)]


def serve_bench(args):
    """Served solves: seeded Poisson request streams (rates 10..2000 req/s),
    request type uniform over sliding 2x4/3x3/2x5/3x4, pancake 8..12 and Hanoi
    8..14 disks, random solvable starts.  The server (continuous batching,
    admission by HBM footprint) against plain sequential solves of the same
    stream (one search at a time, FIFO), both on this GPU.  Latency = arrival
    to completion."""
    import random

    import puzzlesearch_b200 as psb
    puzzles = {t: _make(psb, *t) for t in SERVE_TYPES}
    sessions = {t: psb.BfsSession(puzzles[t], "two_bit") for t in SERVE_TYPES}
    for t in SERVE_TYPES:  # warm-up: load every kernel once
        sessions[t].run(0)
    rows = []
    for rate in args.rates:
        rng = random.Random(int(rate))
        n_req = int(max(30, min(args.max_requests, rate * args.window)))
        arrivals, reqs, t = [], [], 0.0
        for _ in range(n_req):
            t += rng.expovariate(rate)
            ty = SERVE_TYPES[rng.randrange(len(SERVE_TYPES))]
            arrivals.append(t)
            reqs.append((ty, solvable_start(rng, *ty, puzzles[ty])))
        # plain: the same arrival times, one search at a time in arrival
        # order (FIFO); a request waits until it has arrived and the GPU is free
        plain_counts, plain_lat = [], []
        t_start = time.perf_counter()
        for a, (ty, st) in zip(arrivals, reqs):
            while time.perf_counter() - t_start < a:
                time.sleep(0.0002)
            c, _ = sessions[ty].run(st)
            plain_lat.append(time.perf_counter() - t_start - a)
            plain_counts.append(c)
        plain_span = time.perf_counter() - t_start - arrivals[0]
        # served: submit at the arrival times, continuous batching on the GPU
        srv = psb.Server(max_instances=1024, max_depths=256, pool_bytes=args.pool_gb << 30,
                         levels_per_step=args.levels_per_step)
        # warm-up, as the plain arm's sessions were: one request of each type
        # (loads the kernels, sizes the large lane's search arrays)
        warm = [srv.submit(puzzles[t], 0) for t in SERVE_TYPES]
        got = {}
        while len(got) < len(warm):
            got.update(srv.poll())
            time.sleep(0.001)
        t_start = time.perf_counter()
        tickets = {}
        done = {}
        for i, (a, (ty, st)) in enumerate(zip(arrivals, reqs)):
            while time.perf_counter() - t_start < a:
                done.update(srv.poll())
                time.sleep(0.0005)
            tickets[srv.submit(puzzles[ty], st)] = i
        while len(done) < n_req:
            done.update(srv.poll())
            time.sleep(0.001)
        t_end = time.perf_counter()
        srv.stop()
        lat = sorted(done[k][2] for k in tickets)
        for k, i in tickets.items():
            assert done[k][0] == 0 and done[k][1] == plain_counts[i], "served result differs from the plain solve"
        pl = sorted(plain_lat)
        q = lambda v, f: v[min(len(v) - 1, int(f * len(v)))]
        rows.append({"rate": rate, "requests": n_req,
                     "served": {"solves_per_s": n_req / (t_end - t_start - arrivals[0]),
                                "p50_s": q(lat, 0.5), "p99_s": q(lat, 0.99)},
                     "plain": {"solves_per_s": n_req / plain_span, "p50_s": q(pl, 0.5), "p99_s": q(pl, 0.99)},
                     "mean_eccentricity": sum(len(done[k][1]) - 1 for k in tickets) / n_req})
        print(json.dumps({"progress": rows[-1]}), file=sys.stderr, flush=True)
    line = {"metric": "served solves/s and p50/p99 latency (Poisson request streams, continuous batching)",
            "value": max(r["served"]["solves_per_s"] for r in rows), "unit": "solves/s", "n_gpus": 1,
            "higher_is_better": True, "dtype": "u64", "data": "seeded Poisson streams, random solvable starts",
            "config": {"workload": "serve", "types": len(SERVE_TYPES), "pool_gb": args.pool_gb,
                       "levels_per_step": args.levels_per_step},
            "rates": rows, "results_equal_plain": True}
    print(json.dumps(line), flush=True)
    return 0


def profile_once(args):
    """One search with per-level device times (the command ncu wraps)."""
    import puzzlesearch_b200 as psb

    kind, a, b, algo, desc = WORKLOADS[args.workload]
    puzzle = {"pancake": lambda: psb.PancakeSimple(a), "sliding": lambda: psb.SlidingTilePuzzleSimple(a, b),
              "hanoi4": lambda: psb.FourPegHanoiSimple(a, bool(b))}[kind]()
    sink = psb.SPILL_FN(lambda *_: 0) if args.spill else None
    r = psb.bfs(puzzle, algo, 0, max_depth=args.max_depth, window_bits=args.window_bits, levels=True,
                direction=args.direction, bottom_up_ratio=args.bottom_up_ratio, spill=sink,
                segment_bits=args.segment_bits, far_marks=args.far_marks, threads=args.threads)
    out = {"workload": args.workload, "counts": r["counts"], "level_ms": [round(x, 3) for x in r["level_ms"]],
           "level_children": r["level_children"], "stats": r["stats"]}
    print(json.dumps(out), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="pancake14-2bit", choices=sorted(WORKLOADS) + ["batch4096", "serve"])
    ap.add_argument("--window-bits", type=int, default=0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--direction", default="auto", choices=["auto", "top_down", "bottom_up"],
                    help="level direction (PSB_DIR_*): auto switches to bottom-up on the last dense levels")
    ap.add_argument("--bottom-up-ratio", type=float, default=0.0,
                    help="auto: a level runs bottom-up when unvisited < ratio x frontier (0 = library default)")
    ap.add_argument("--spill", action="store_true",
                    help="encode every depth's frontier on the GPU (segment streams) and hand it over in pinned"
                         " host memory during the timed searches (default for pancake14-2bit and hanoi18-2bit)")
    ap.add_argument("--no-spill", action="store_true", help="no frontier spill, whatever the workload")
    ap.add_argument("--threads", type=int, default=0, choices=[0, 128, 256, 512],
                    help="threads per block of the top-down two-bit / three-bit level kernels (0 = 128 for two-bit"
                         " pancake and Hanoi searches of 2^32 states or more, else 256)")
    ap.add_argument("--far-marks", default="auto", choices=["auto", "none", "near", "all"],
                    help="two-bit long-range marks (PSB_FAR_*); --autotune picks it for two-bit workloads")
    ap.add_argument("--e2e-calls", type=int, default=5,
                    help="timed calls of the public entry point for `e2e` (at most --steps)")
    ap.add_argument("--segment-bits", type=int, default=0, help="with --spill: 2^bits states per segment (0 = 32)")
    ap.add_argument("--autotune", action="store_true",
                    help="pick the level window (single searches) or the engine's blocks per SM (batch4096) by"
                         " timing the candidates first")
    ap.add_argument("--profile-once", action="store_true",
                    help="run ONE search (no warm-up, no e2e, no CPU baseline) and print per-level times; for ncu")
    ap.add_argument("--max-depth", type=int, default=0, help="with --profile-once: stop after this depth")
    ap.add_argument("--instances", type=int, default=4096, help="--workload batch4096: number of searches")
    ap.add_argument("--rates", type=float, nargs="+", default=[10, 30, 100, 300, 1000, 2000],
                    help="--workload serve: request rates (req/s)")
    ap.add_argument("--window", type=float, default=3.0, help="--workload serve: seconds of arrivals per rate")
    ap.add_argument("--max-requests", type=int, default=400, help="--workload serve: requests per rate at most")
    ap.add_argument("--pool-gb", type=int, default=32, help="--workload serve: engine pool (HBM admission limit)")
    ap.add_argument("--levels-per-step", type=int, default=4,
                    help="--workload serve: engine levels per step while no request waits")
    args = ap.parse_args()
    args.spill = (args.spill or args.workload in SPILL_BY_DEFAULT) and not args.no_spill
    if args.profile_once:
        return profile_once(args)
    if args.workload == "batch4096":
        return batch_bench(args)
    if args.workload == "serve":
        return serve_bench(args)
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference_arm(args)

    import torch

    import puzzlesearch_b200 as psb

    rank, world, local, dist = dist_setup(args.gpus)
    torch.cuda.set_device(local)
    kind, a, b, algo, desc = WORKLOADS[args.workload]
    puzzle = {"pancake": lambda: psb.PancakeSimple(a), "sliding": lambda: psb.SlidingTilePuzzleSimple(a, b),
              "hanoi4": lambda: psb.FourPegHanoiSimple(a, bool(b))}[kind]()
    N = puzzle.IndexesCount()
    tuning = None
    if args.autotune and not args.window_bits:
        from puzzlesearch_b200 import autotune
        args.window_bits, timings = autotune.tune_window_bits(puzzle, algo, 0, direction=args.direction)
        tuning = {"window_bits": args.window_bits, "search_ms": {str(k): round(v, 2) for k, v in timings.items()}}
        if algo == "two_bit":
            args.far_marks, ft = autotune.tune_far_marks(puzzle, 0, window_bits=args.window_bits)
            tuning.update({"far_marks": args.far_marks, "far_marks_ms": {k: round(v, 2) for k, v in ft.items()}})
        if algo in ("two_bit", "three_bit"):
            args.threads, tt = autotune.tune_threads(puzzle, algo, 0, window_bits=args.window_bits,
                                                     far_marks=args.far_marks)
            tuning.update({"threads": args.threads, "threads_ms": {str(k): round(v, 2) for k, v in tt.items()}})
    stream = torch.cuda.Stream()
    # Session on torch's stream so the CUDA events below bracket exactly the searches.
    opts = psb._opts(0, args.window_bits, local, stream.cuda_stream, direction=args.direction,
                     far_marks=args.far_marks, threads=args.threads)
    h = ctypes.c_void_p()
    psb._check(psb.lib().psb_bfs_session_create(puzzle.handle, psb._algo(algo), ctypes.byref(opts), ctypes.byref(h)))
    cap = 1 << 16
    counts = (ctypes.c_uint64 * cap)()
    nd = ctypes.c_uint32()
    # Frontier spill sink: the streams arrive in the library's pinned host
    # buffer; this caller only tallies them (a real caller stores them).
    spilled = {"bytes": 0, "segments": 0, "states": 0}

    def _sink(_user, depth, segment, data, n, states):
        spilled["bytes"] += n
        spilled["segments"] += 1
        spilled["states"] += states
        return 0

    spill_fn = psb.SPILL_FN(_sink) if args.spill else None

    def run_once():
        st = psb.BfsStats()
        st.struct_size = ctypes.sizeof(psb.BfsStats)
        o = psb._opts(0, 0, local, stream.cuda_stream, direction=args.direction,
                      bottom_up_ratio=args.bottom_up_ratio, spill=spill_fn, segment_bits=args.segment_bits,
                      far_marks=args.far_marks, threads=args.threads)
        psb._check(psb.lib().psb_bfs_session_run(h, 0, ctypes.byref(o), counts, cap, ctypes.byref(nd), ctypes.byref(st)))
        return list(counts[:nd.value]), st

    for _ in range(args.warmup):
        ref_counts, _ = run_once()
    assert sum(ref_counts) in (N, N // 2), "search did not reach the whole component"

    def barrier():
        if dist:
            dist.barrier()

    stats = []
    torch.cuda.synchronize()
    barrier()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        start.record(stream)
        for _ in range(args.steps):
            c, st = run_once()
            assert c == ref_counts
            stats.append(st)
        end.record(stream)
        torch.cuda.synchronize()
    barrier()
    elapsed_ms = max_over_ranks(start.elapsed_time(end), dist)
    states_per_step = sum(ref_counts)
    value = job_rate(world, args.steps, states_per_step, elapsed_ms / 1000.0)

    # e2e: the public C-ABI entry point, host in/out, allocation included.
    # An untimed warm-up call first: the first call grows the library's
    # memory pool.  Fewer calls than device steps keep the run short.
    e2e_calls = max(1, min(args.steps, args.e2e_calls))
    for _ in range(1):
        psb.bfs(puzzle, algo, 0, device=local, direction=args.direction, bottom_up_ratio=args.bottom_up_ratio,
                spill=spill_fn, segment_bits=args.segment_bits, window_bits=args.window_bits,
                far_marks=args.far_marks, threads=args.threads)
    torch.cuda.synchronize()
    barrier()
    t0 = time.perf_counter()
    levels = 0
    calls = []
    for _ in range(e2e_calls):
        tc = time.perf_counter()
        r = psb.bfs(puzzle, algo, 0, device=local, direction=args.direction, bottom_up_ratio=args.bottom_up_ratio,
                    spill=spill_fn, segment_bits=args.segment_bits, window_bits=args.window_bits,
                far_marks=args.far_marks, threads=args.threads)
        calls.append(time.perf_counter() - tc)
        assert r["counts"] == ref_counts
        levels = r["stats"]["levels"]
    torch.cuda.synchronize()
    e2e_s = max_over_ranks(time.perf_counter() - t0, dist)
    e2e_value = job_rate(world, e2e_calls, states_per_step, e2e_s)

    psb.lib().psb_bfs_session_destroy(h)
    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return 0

    # Roofline of the dominant kernel (the fused level kernel), algorithmic bytes:
    # per level N/8 bytes of frontier swept + 8 bytes per generated child
    # (three-bit); two-bit sweeps 2N/8 read + 2N/8 write per level.
    st = stats[-1]
    if algo == "three_bit":
        sweep_bytes = N / 8
    elif algo == "two_bit":
        sweep_bytes = 2 * (2 * N / 8)
    else:
        sweep_bytes = N / 8
    alg_bytes = st.levels * sweep_bytes + 8.0 * st.children
    expand_ms = sum(s.expand_ms for s in stats) / len(stats)
    achieved = alg_bytes / (expand_ms / 1000.0) / 1e9
    peak, peak_kind = load_peaks()
    traffic = None
    tr = LEVEL_TRAFFIC.get(args.workload)
    if tr and st.levels == tr["launches"] and st.window_bits == tr["window_bits"] and st.threads == tr["threads"]:
        traffic = {"per_launch": tr["bytes"] / tr["launches"], "per_search": tr["bytes"],
                   "vs_algorithmic": tr["bytes"] / alg_bytes,
                   # the captured bytes over this run's level time: the DRAM throughput the kernels sustain
                   "dram_gbs": tr["bytes"] / (expand_ms / 1000.0) / 1e9,
                   "dram_frac": tr["bytes"] / (expand_ms / 1000.0) / 1e9 / peak,
                   "source": "ncu one-pass capture, dram__bytes_read.sum + dram__bytes_write.sum over the search's"
                             " level launches (" + tr["profile"] + ")"}
    # level kernels + one finalize per level (three-bit, classic) or one
    # CUR -> OLD pass per bottom-up level (two-bit)
    launches_per_step = st.levels + st.other_launches + st.spill_launches

    if args.spill:
        desc += "; every depth's frontier encoded on the GPU and spilled to pinned host memory"
    line = {
        "metric": f"BFS states/sec ({desc})", "value": value, "unit": "states/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": elapsed_ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64",
        "data": "synthetic (the puzzle's full state space from its standard start state)",
        "config": {"workload": args.workload, "states": states_per_step, "depths": len(ref_counts),
                   "index_space": N, "device_bytes": st.device_bytes, "window_bits": st.window_bits,
                   "l2": "inputs larger than L2 (bit arrays of %d MB resident in HBM)" % (st.device_bytes >> 20),
                   "parallelism": f"replicas x{world}" if world > 1 else "1 GPU"},
        "e2e": {"value": e2e_value, "unit": "states/s", "calls": e2e_calls, "h2d_bytes_per_step": 8,
                "d2h_bytes_per_step": 64 * levels + 8 * len(ref_counts),
                "call_s": [round(c, 4) for c in calls]},
        "gpu_launches": launches_per_step * args.steps,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic["per_launch"] if traffic else None,
                     "note": f"level kernel (top-down and bottom-up launches), {peak_kind} peak; algorithmic bytes"
                             f" per level = {'N/8' if algo != 'two_bit' else '2 x 2N/8'} sweep + 8 B per child"
                             " generated or probe issued; traffic (bytes per launch) from the capture named in"
                             " traffic_detail, null where no capture covers this workload",
                     "traffic_detail": traffic},
        "kernel_ms_per_step": {"level": expand_ms, "finalize": sum(s.finalize_ms for s in stats) / len(stats)},
        "children_per_step": st.children, "local_child_fraction": st.local_children / max(st.children, 1),
        "direction": {"mode": args.direction, "bottom_up_levels": st.bottom_up_levels, "levels": st.levels},
        "clocks": clk.summary(),
    }
    if tuning:
        line["config"]["autotune"] = tuning
    if args.spill:
        line["spill"] = {"segment_bits": args.segment_bits or 32, "bytes_per_step": st.spill_bytes,
                         "segments_per_step": st.spill_segments,
                         "ms_per_step": sum(s.spill_ms for s in stats) / len(stats),
                         "encode_ms_per_step": sum(s.spill_encode_ms for s in stats) / len(stats),
                         "copy_ms_per_step": sum(s.spill_copy_ms for s in stats) / len(stats),
                         "copy_gbs": st.spill_bytes / max(st.spill_copy_ms, 1e-9) / 1e6,
                         "bytes_per_state": st.spill_bytes / states_per_step,
                         "d2h_bytes_per_step": st.spill_bytes}
        line["e2e"]["d2h_bytes_per_step"] += st.spill_bytes
    if not args.no_cpu_baseline and world == 1:
        s, secs, ck = cpu_reference_sample()
        kind_s, a_s, _, algo_s = REF_SAMPLE
        line["cpu_baseline"] = {"value": s / secs, "unit": "states/s", "cores": 1, "kind": ck,
                                "sample": f"reference InMemory{'TwoBit' if algo_s == 'two_bit' else 'ThreeBit'}BFS"
                                          f" on {a_s}-pancake (full search, {math.factorial(a_s):,} states),"
                                          " single-threaded as in the reference"}
    print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
