"""Autotuner for the launch shapes and strategies that are picked by
measurement rather than by rule: the batch engine's persistent grid (blocks
per SM) and its instances' window size; the window of a single search's
level kernel (states per thread-block window, the unit of work the kernel
sweeps and marks in shared memory) and its threads per block; and where a
two-bit search's long-range marks go (PSB_FAR_*).

Each candidate runs the same workload on this device.  The tuner checks that
every candidate gives the same results, and returns the fastest one with all
timings.  Results can be kept in a JSON file, keyed by device name and
workload, so that later runs on the same GPU model reuse them.
"""
import json
import os
import time

from . import Engine, bfs, device_name, lib

__all__ = ["tune", "tune_engine", "tune_window_bits", "tune_far_marks", "tune_threads", "Cache"]


def tune(candidates, measure):
    """measure(candidate) -> (seconds, result).  Returns (best, {candidate:
    seconds}).  Every candidate must produce the same result."""
    timings, reference = {}, None
    for c in candidates:
        seconds, result = measure(c)
        if reference is None:
            reference = result
        elif result != reference:
            raise AssertionError(f"autotune: candidate {c!r} changed the result")
        timings[c] = seconds
    best = min(timings, key=timings.get)
    return best, timings


class Cache:
    """Tuning results in a JSON file: {device: {workload: best}}."""

    def __init__(self, path):
        self.path = path
        self.data = {}
        if path and os.path.exists(path):
            with open(path) as f:
                self.data = json.load(f)

    def get(self, device, key):
        return self.data.get(device, {}).get(key)

    def put(self, device, key, value):
        self.data.setdefault(device, {})[key] = value
        if self.path:
            tmp = self.path + ".tmp"
            with open(tmp, "w") as f:
                json.dump(self.data, f, indent=1, sort_keys=True)
            os.replace(tmp, self.path)


def _run_engine(items, shape, levels_per_step, pool_bytes, direction):
    blocks_per_sm, window_bits_offset = shape if isinstance(shape, tuple) else (shape, 0)
    eng = Engine(max_instances=len(items), pool_bytes=pool_bytes, blocks_per_sm=blocks_per_sm,
                 direction=direction, window_bits_offset=window_bits_offset)
    try:
        t0 = time.perf_counter()
        for tag, (puzzle, start) in enumerate(items):
            if not eng.add(puzzle, start, tag):
                raise RuntimeError("autotune: calibration batch does not fit the engine pool")
        done = {}
        while len(done) < len(items):
            eng.step(levels_per_step)
            done.update(eng.poll())
        return time.perf_counter() - t0, [done[t] for t in range(len(items))]
    finally:
        eng.close()


ENGINE_SHAPES = tuple((b, w) for b in (1, 2, 3, 4) for w in (-2, -1, 0, 1))


def tune_engine(items, candidates=ENGINE_SHAPES, levels_per_step=8, pool_bytes=8 << 30, direction="auto",
                cache=None, key=None):
    """The batch engine's launch shape, timed on a calibration batch `items`
    = [(puzzle, start index)] (admission, all steps and the result
    read-back): persistent blocks per SM x the instances' window size (as an
    offset from the engine's rule of 2^(log2 states - 6) states; windows are
    also the engine's work items and flag units).  A candidate is a
    (blocks_per_sm, window_bits_offset) pair, or a plain blocks-per-SM count.
    Returns (best, {candidate: seconds})."""
    dev = device_name()
    if cache and key and cache.get(dev, key) is not None:
        hit = cache.get(dev, key)
        return (tuple(hit) if isinstance(hit, list) else hit), {}
    _run_engine(items[: max(1, len(items) // 8)], candidates[0], levels_per_step, pool_bytes, direction)  # warm-up
    best, timings = tune(candidates, lambda c: _run_engine(items, c, levels_per_step, pool_bytes, direction))
    if cache and key:
        cache.put(dev, key, best)
    return best, timings


def tune_window_bits(puzzle, algo, initial=0, candidates=None, direction="auto", cache=None, key=None):
    """Window bits for one search's level kernel, timed as the device time of
    the whole search (CUDA events in the library).  Candidates default to the
    automatic choice and its neighbours.  Returns (best, {bits: ms})."""
    dev = device_name()
    if cache and key and cache.get(dev, key) is not None:
        return cache.get(dev, key), {}
    if candidates is None:
        auto = bfs(puzzle, algo, initial, max_depth=1, direction=direction)["stats"]["window_bits"]
        candidates = sorted({max(10, min(18, auto + d)) for d in (-2, -1, 0, 1, 2)})
    bfs(puzzle, algo, initial, window_bits=candidates[0], direction=direction)  # warm-up (pool growth)

    def measure(wb):
        r = bfs(puzzle, algo, initial, window_bits=wb, direction=direction)
        return r["stats"]["total_ms"], r["counts"]

    best, timings = tune(candidates, measure)
    if cache and key:
        cache.put(dev, key, best)
    return best, timings


def tune_far_marks(puzzle, initial=0, candidates=("none", "near", "all"), window_bits=0, cache=None, key=None):
    """Where a two-bit search's long-range marks go (PSB_FAR_*: read the
    target's code first, or a far bitmap folded after each level, for the
    near marks only or for all of them), timed as the device time of the
    whole search.  Returns (best, {mode: ms})."""
    dev = device_name()
    if cache and key and cache.get(dev, key) is not None:
        return cache.get(dev, key), {}
    bfs(puzzle, "two_bit", initial, window_bits=window_bits, far_marks=candidates[-1])  # warm-up (pool growth)

    def measure(mode):
        r = bfs(puzzle, "two_bit", initial, window_bits=window_bits, far_marks=mode)
        return r["stats"]["total_ms"], r["counts"]

    best, timings = tune(candidates, measure)
    if cache and key:
        cache.put(dev, key, best)
    return best, timings


def tune_threads(puzzle, algo, initial=0, candidates=(128, 256, 512), window_bits=0, far_marks="auto",
                 cache=None, key=None):
    """Threads per block of a single search's top-down level kernel (two-bit
    and three-bit: shape variants compiled as separate kernel instances),
    timed as the device time of the whole search.  Returns (best, {threads: ms})."""
    dev = device_name()
    if cache and key and cache.get(dev, key) is not None:
        return cache.get(dev, key), {}
    bfs(puzzle, algo, initial, window_bits=window_bits, far_marks=far_marks)  # warm-up (pool growth)

    def measure(threads):
        r = bfs(puzzle, algo, initial, window_bits=window_bits, far_marks=far_marks, threads=threads)
        return r["stats"]["total_ms"], r["counts"]

    best, timings = tune(candidates, measure)
    if cache and key:
        cache.put(dev, key, best)
    return best, timings
