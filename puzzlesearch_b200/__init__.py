"""puzzlesearch_b200 -- Python binding of the C ABI in include/psb200.h.

It mirrors the reference's Puzzle API (Common/Puzzle.h:16-48) and its
in-memory entry points (Common/InMemoryBFS.h:5-11) under the same names:

    from puzzlesearch_b200 import PancakeSimple, InMemoryThreeBitBFS
    puzzle = PancakeSimple(13)
    counts = InMemoryThreeBitBFS(puzzle, puzzle.ToString(0))

All search work runs on the GPU through libpsb200.so (sm_100a).  There is no
CPU fallback: if the library or a CUDA device is missing, calls raise
PsbError.
"""
import ctypes
import os

__all__ = [
    "PsbError", "lib", "SlidingTilePuzzleSimple", "SlidingTilePuzzleOptimized", "PancakeSimple", "PancakeOptimized", "FourPegHanoiOptimized", "FourPegHanoiSimple",
    "InMemoryTwoBitBFS", "InMemoryThreeBitBFS", "InMemoryFrontierSearch", "InMemoryClassicBFS",
    "bfs", "bfs_segmented", "BfsSession", "Store", "TWO_BIT", "THREE_BIT", "FRONTIER", "CLASSIC", "INVALID_INDEX",
]

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("PSB_LIB") or os.path.join(HERE, "libpsb200.so")

SLIDING, PANCAKE, HANOI4, PANCAKE_OPT, HANOI4_OPT, SLIDING_OPT = 1, 2, 3, 4, 5, 6
TWO_BIT, THREE_BIT, FRONTIER, CLASSIC = 1, 2, 3, 4
ALGOS = {"two_bit": TWO_BIT, "three_bit": THREE_BIT, "frontier": FRONTIER, "classic": CLASSIC}
INVALID_INDEX = (1 << 64) - 1
EXPAND_HOST_POINTERS, EXPAND_COMPACT, EXPAND_USE_OPBITS = 1, 2, 4

u64p = ctypes.POINTER(ctypes.c_uint64)
u32p = ctypes.POINTER(ctypes.c_uint32)


class PsbError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"psb error {code}: {msg}")
        self.code = code


# psb_spill_fn(user, depth, segment, stream, bytes, states)
SPILL_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint32,
                            ctypes.POINTER(ctypes.c_uint8), ctypes.c_uint64, ctypes.c_uint64)


class BfsOpts(ctypes.Structure):
    _fields_ = [("struct_size", ctypes.c_uint32), ("max_depth", ctypes.c_uint32),
                ("window_bits", ctypes.c_int32), ("device", ctypes.c_int32),
                ("stream", ctypes.c_void_p), ("final_words", u64p), ("final_cap", ctypes.c_uint64),
                ("level_ms", ctypes.POINTER(ctypes.c_float)), ("level_children", u64p),
                ("direction", ctypes.c_int32), ("bottom_up_ratio", ctypes.c_float),
                ("spill", SPILL_FN), ("spill_user", ctypes.c_void_p), ("segment_bits", ctypes.c_int32),
                ("far_marks", ctypes.c_int32), ("threads", ctypes.c_int32), ("restored_counts", u64p)]


class BfsStats(ctypes.Structure):
    _fields_ = [("struct_size", ctypes.c_uint32), ("levels", ctypes.c_uint32),
                ("window_bits", ctypes.c_uint32), ("threads", ctypes.c_uint32),
                ("total_ms", ctypes.c_double), ("expand_ms", ctypes.c_double),
                ("finalize_ms", ctypes.c_double), ("expanded", ctypes.c_uint64),
                ("children", ctypes.c_uint64), ("local_children", ctypes.c_uint64),
                ("expand_launches", ctypes.c_uint64), ("device_bytes", ctypes.c_uint64),
                ("bottom_up_levels", ctypes.c_uint64), ("spill_ms", ctypes.c_double),
                ("spill_bytes", ctypes.c_uint64), ("spill_segments", ctypes.c_uint64),
                ("spill_launches", ctypes.c_uint64), ("spill_encode_ms", ctypes.c_double),
                ("spill_copy_ms", ctypes.c_double), ("other_launches", ctypes.c_uint64)]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_ if name != "struct_size"}


class EngineOpts(ctypes.Structure):
    _fields_ = [("struct_size", ctypes.c_uint32), ("max_instances", ctypes.c_uint32),
                ("max_depths", ctypes.c_uint32), ("device", ctypes.c_int32), ("pool_bytes", ctypes.c_uint64),
                ("blocks_per_sm", ctypes.c_int32), ("use_graph", ctypes.c_int32), ("direction", ctypes.c_int32),
                ("window_bits_offset", ctypes.c_int32)]


class ServerOpts(ctypes.Structure):
    _fields_ = [("struct_size", ctypes.c_uint32), ("levels_per_step", ctypes.c_uint32), ("engine", EngineOpts),
                ("large_states", ctypes.c_uint64)]


class SegmentedOpts(ctypes.Structure):
    _fields_ = [("struct_size", ctypes.c_uint32), ("max_depth", ctypes.c_uint32), ("segment_bits", ctypes.c_int32),
                ("device", ctypes.c_int32), ("chunk_states", ctypes.c_uint64),
                ("directories", ctypes.POINTER(ctypes.c_char_p)), ("n_directories", ctypes.c_int32),
                ("files_per_path", ctypes.c_int32)]


class SegmentedStats(ctypes.Structure):
    _fields_ = [("struct_size", ctypes.c_uint32), ("pad", ctypes.c_uint32), ("segments", ctypes.c_uint64),
                ("device_bytes", ctypes.c_uint64), ("peak_host_bytes", ctypes.c_uint64),
                ("h2d_bytes", ctypes.c_uint64), ("d2h_bytes", ctypes.c_uint64), ("cross_children", ctypes.c_uint64),
                ("total_ms", ctypes.c_double), ("peak_disk_bytes", ctypes.c_uint64)]


class CodecBlock(ctypes.Structure):
    """psb_codec_block: one block of a compressed frontier stream."""
    _fields_ = [("offset", ctypes.c_uint64), ("count", ctypes.c_uint32), ("bytes", ctypes.c_uint32),
                ("first", ctypes.c_uint32), ("is_bitmap", ctypes.c_uint32)]


_lib = None


def lib():
    """Loads libpsb200.so; raises PsbError when it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise PsbError(-5, f"{LIB_PATH} is missing: build it with python -m puzzlesearch_b200.build")
        L = ctypes.CDLL(LIB_PATH)
        P = ctypes.c_void_p
        L.psb_version.restype = ctypes.c_char_p
        L.psb_last_error.argtypes = [ctypes.c_char_p, ctypes.c_int]
        L.psb_device_count.argtypes = [ctypes.POINTER(ctypes.c_int)]
        L.psb_device_name.argtypes = [ctypes.c_int, ctypes.c_char_p, ctypes.c_int]
        L.psb_puzzle_create.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(P)]
        L.psb_puzzle_destroy.argtypes = [P]
        L.psb_puzzle_info.argtypes = [P, u64p, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                      ctypes.POINTER(ctypes.c_int)]
        L.psb_puzzle_name.argtypes = [P, ctypes.c_char_p, ctypes.c_int]
        L.psb_parse.argtypes = [P, ctypes.c_char_p, u64p]
        L.psb_to_string.argtypes = [P, ctypes.c_uint64, ctypes.c_char_p, ctypes.c_int]
        L.psb_expand.argtypes = [P, u64p, u32p, ctypes.c_uint64, u64p, u32p, ctypes.c_uint64, u64p,
                                 ctypes.c_uint32, ctypes.c_void_p]
        L.psb_final_words.argtypes = [P, ctypes.c_int, u64p]
        L.psb_bfs.argtypes = [P, ctypes.c_int, ctypes.c_uint64, ctypes.POINTER(BfsOpts), u64p, ctypes.c_uint32,
                              u32p, ctypes.POINTER(BfsStats)]
        L.psb_bfs_footprint.argtypes = [P, ctypes.c_int, u64p]
        L.psb_bfs_session_create.argtypes = [P, ctypes.c_int, ctypes.POINTER(BfsOpts), ctypes.POINTER(P)]
        L.psb_bfs_session_run.argtypes = [P, ctypes.c_uint64, ctypes.POINTER(BfsOpts), u64p, ctypes.c_uint32,
                                          u32p, ctypes.POINTER(BfsStats)]
        L.psb_bfs_session_destroy.argtypes = [P]
        L.psb_release_cached_memory.argtypes = [ctypes.c_int]
        vp = ctypes.c_void_p
        L.psb_bits_set_stride.argtypes = [vp, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64, vp]
        L.psb_bits_scan.argtypes = [vp, vp, ctypes.c_uint64, ctypes.c_int, u64p, u64p, vp]
        L.psb_bits_and_not_count.argtypes = [vp, vp, ctypes.c_uint64, u64p, vp]
        L.psb_bits_or.argtypes = [vp, vp, ctypes.c_uint64, vp]
        L.psb_frontier_encode.argtypes = [u64p, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_void_p, ctypes.c_uint64,
                                          u64p, ctypes.POINTER(CodecBlock), ctypes.c_uint32, u32p, ctypes.c_void_p]
        L.psb_frontier_index.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.POINTER(CodecBlock),
                                         ctypes.c_uint32, u32p]
        L.psb_frontier_decode.argtypes = [ctypes.c_void_p, ctypes.POINTER(CodecBlock), ctypes.c_uint32, u64p,
                                          ctypes.c_uint64, ctypes.c_uint64, ctypes.c_void_p]
        L.psb_opbits_encode.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p,
                                        ctypes.c_void_p]
        L.psb_opbits_decode.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p,
                                        ctypes.c_void_p]
        L.psb_bfs_segmented.argtypes = [P, ctypes.c_uint64, ctypes.POINTER(SegmentedOpts), u64p, ctypes.c_uint32,
                                        u32p, ctypes.POINTER(SegmentedStats)]
        cpp = ctypes.POINTER(ctypes.c_char_p)
        L.psb_store_create.argtypes = [ctypes.c_int, ctypes.c_char_p, cpp, ctypes.c_int, ctypes.c_int,
                                       ctypes.POINTER(P)]
        L.psb_store_destroy.argtypes = [P]
        L.psb_store_write.argtypes = [P, ctypes.c_int, ctypes.c_void_p, ctypes.c_uint64]
        L.psb_store_read.argtypes = [P, ctypes.c_int, ctypes.c_void_p, ctypes.c_uint64, u64p]
        L.psb_store_rewind.argtypes = [P, ctypes.c_int]
        L.psb_store_length.argtypes = [P, ctypes.c_int, u64p]
        L.psb_store_delete.argtypes = [P, ctypes.c_int]
        L.psb_engine_create.argtypes = [ctypes.POINTER(EngineOpts), ctypes.POINTER(P)]
        L.psb_engine_destroy.argtypes = [P]
        L.psb_engine_footprint.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, u64p]
        L.psb_engine_add.argtypes = [P, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_uint64, ctypes.c_uint64,
                                     u32p]
        L.psb_engine_step.argtypes = [P, ctypes.c_uint32]
        L.psb_engine_poll.argtypes = [P, u64p, u32p, u64p, ctypes.c_uint32, u32p]
        L.psb_engine_info.argtypes = [P, u32p, u64p, u64p]
        L.psb_server_start.argtypes = [ctypes.POINTER(ServerOpts), ctypes.POINTER(P)]
        L.psb_server_submit.argtypes = [P, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_uint64, u64p]
        L.psb_server_poll.argtypes = [P, u64p, ctypes.POINTER(ctypes.c_int), u32p, u64p,
                                      ctypes.POINTER(ctypes.c_double), ctypes.c_uint32, u32p]
        L.psb_server_info.argtypes = [P, u32p, u32p, u64p, u64p]
        L.psb_server_stop.argtypes = [P]
        L.psb_bfs_noalloc.argtypes = [P, ctypes.c_int, ctypes.c_uint64, u64p, ctypes.c_uint64, ctypes.c_uint32,
                                      ctypes.c_void_p, u64p, ctypes.c_uint32, u32p]
        _lib = L
    return _lib


def _check(rc):
    if rc < 0:
        buf = ctypes.create_string_buffer(512)
        lib().psb_last_error(buf, 512)
        raise PsbError(rc, buf.value.decode(errors="replace"))
    return rc


def device_name(device=-1):
    """psb_device_name: e.g. "NVIDIA B200 (sm_100, 148 SMs)"."""
    buf = ctypes.create_string_buffer(256)
    _check(lib().psb_device_name(device, buf, 256))
    return buf.value.decode()


def device_count():
    c = ctypes.c_int()
    _check(lib().psb_device_count(ctypes.byref(c)))
    return c.value


class Puzzle:
    """Common/Puzzle.h:16-48, backed by a psb_puzzle handle."""
    MAX_INDEXES_BUFFER = 2 * 1024 * 1024   # Common/Puzzle.h:18
    INVALID_INDEX = INVALID_INDEX           # Common/Puzzle.h:19

    def __init__(self, kind, a, b=0):
        h = ctypes.c_void_p()
        _check(lib().psb_puzzle_create(kind, a, b, ctypes.byref(h)))
        self._h = h
        self.kind, self.a, self.b = kind, a, b
        n = ctypes.c_uint64()
        ops, br, odd = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        _check(lib().psb_puzzle_info(h, ctypes.byref(n), ctypes.byref(ops), ctypes.byref(br), ctypes.byref(odd)))
        self._info = (n.value, ops.value, br.value, bool(odd.value))

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and _lib is not None:
            _lib.psb_puzzle_destroy(h)
            self._h = None

    @property
    def handle(self):
        return self._h

    def Name(self):
        buf = ctypes.create_string_buffer(256)
        _check(lib().psb_puzzle_name(self._h, buf, 256))
        return buf.value.decode()

    def IndexesCount(self):
        return self._info[0]

    def OperatorsCount(self):
        return self._info[1]

    def BranchingFactor(self):
        return self._info[2]

    def HasOddLengthCycles(self):
        return self._info[3]

    def Parse(self, state):
        out = ctypes.c_uint64()
        _check(lib().psb_parse(self._h, state.encode(), ctypes.byref(out)))
        return out.value

    def ToString(self, index):
        buf = ctypes.create_string_buffer(512)
        _check(lib().psb_to_string(self._h, index, buf, 512))
        return buf.value.decode()

    def Expand(self, indexes, usedOperatorBits=None, compact=True):
        """Puzzle::Expand: returns (expandedIndexes, expandedOperators).

        compact=True drops INVALID_INDEX slots (what ExpandBuffer does,
        Common/Puzzle.h:95-101); compact=False returns BranchingFactor() slots
        per parent like the reference's GPU puzzles."""
        n = len(indexes)
        br = self.BranchingFactor()
        P = (ctypes.c_uint64 * max(n, 1))(*indexes)
        flags = EXPAND_HOST_POINTERS | (EXPAND_COMPACT if compact else 0)
        O = None
        if usedOperatorBits is not None:
            O = (ctypes.c_uint32 * max(n, 1))(*usedOperatorBits)
            flags |= EXPAND_USE_OPBITS
        cap = max(n * br, 1)
        C = (ctypes.c_uint64 * cap)()
        CO = (ctypes.c_uint32 * cap)()
        n_out = ctypes.c_uint64()
        _check(lib().psb_expand(self._h, P, O, n, C, CO, cap, ctypes.byref(n_out), flags, None))
        k = n_out.value
        return list(C[:k]), list(CO[:k])

    def expand_device(self, parents_ptr, opbits_ptr, n, children_ptr, ops_ptr, stream=None):
        """Expand with device pointers (ints); BranchingFactor() slots per parent."""
        n_out = ctypes.c_uint64()
        flags = EXPAND_USE_OPBITS if opbits_ptr else 0
        _check(lib().psb_expand(self._h, ctypes.cast(parents_ptr, u64p), ctypes.cast(opbits_ptr or 0, u32p), n,
                                ctypes.cast(children_ptr, u64p), ctypes.cast(ops_ptr, u32p),
                                n * self.BranchingFactor(), ctypes.byref(n_out), flags, stream))
        return n_out.value

    def footprint(self, algo):
        b = ctypes.c_uint64()
        _check(lib().psb_bfs_footprint(self._h, _algo(algo), ctypes.byref(b)))
        return b.value

    def final_words(self, algo):
        w = ctypes.c_uint64()
        _check(lib().psb_final_words(self._h, _algo(algo), ctypes.byref(w)))
        return w.value


class SlidingTilePuzzleSimple(Puzzle):
    """Puzzles/SlidingTilePuzzleSimple.h: index = permutation rank over width*height cells."""

    def __init__(self, width, height):
        super().__init__(SLIDING, width, height)


class SlidingTilePuzzleOptimized(Puzzle):
    """Puzzles/SlidingTilePuzzleOptimized.h (the reference's class template
    SlidingTilePuzzleOptimized<width, height>): the tiles' left-smaller digits
    2..11 in mixed radix times 16 plus the blank, digits 12..14 as nibbles
    above bit 32; 16 * (cells-1)!/2 indexes up to 13 cells."""

    def __init__(self, width, height):
        super().__init__(SLIDING_OPT, width, height)


class PancakeSimple(Puzzle):
    """Puzzles/PancakeSimple.h: operator k reverses the last k+2 values."""

    def __init__(self, size):
        super().__init__(PANCAKE, size, 0)


class PancakeOptimized(Puzzle):
    """Puzzles/PancakeOptimized.h: the pancake moves in the reference's GPU
    pancake index ((rank / 12!) << 29 | rank % 12! above 11 pancakes)."""

    def __init__(self, size, inverseIndex=False):
        super().__init__(PANCAKE_OPT, size, 1 if inverseIndex else 0)


class FourPegHanoiSimple(Puzzle):
    """Puzzles/FourPegHanoiSimple.h: 2 bits per disk; optional peg symmetry."""

    def __init__(self, size, useSymmetry=False):
        super().__init__(HANOI4, size, 1 if useSymmetry else 0)


class FourPegHanoiOptimized(Puzzle):
    """Puzzles/FourPegHanoiOptimized.h: FourPegHanoiSimple's index; with
    symmetry the peg order is restored only when a move empties or fills a peg."""

    def __init__(self, size, useSymmetry=False):
        super().__init__(HANOI4_OPT, size, 1 if useSymmetry else 0)


def _algo(algo):
    return ALGOS[algo] if isinstance(algo, str) else int(algo)


DIRECTIONS = {"auto": 0, "top_down": 1, "bottom_up": 2}


class _Spill:
    """Wraps spill(depth, segment, stream_bytes, states) -> stop (truthy ends
    the search with PSB_ERR_ABORTED) as a psb_spill_fn.  The stream is copied
    out of the pinned staging buffer before spill is called.  An exception
    cannot cross the C ABI: it stops the search and is raised again by
    run() once the library has returned."""

    def __init__(self, spill):
        self.error = None

        def fn(_user, depth, segment, data, n, states):
            try:
                return 1 if spill(depth, segment, ctypes.string_at(data, n), states) else 0
            except Exception as e:
                self.error = e
                return 1

        self.fn = SPILL_FN(fn)

    def run(self, call):
        rc = call()
        if rc < 0 and self.error is not None:
            raise self.error
        _check(rc)


def _spill_fn(spill):
    """(SPILL_FN or None, runner) for a spill argument: a SPILL_FN passes
    through as is (it sees the pinned buffer itself)."""
    if spill is None or isinstance(spill, SPILL_FN):
        return spill, _check_call
    w = _Spill(spill)
    return w.fn, w.run


def _check_call(call):
    _check(call())


FAR_MARKS = {"auto": 0, "none": 1, "near": 2, "all": 3}


def _opts(max_depth=0, window_bits=0, device=-1, stream=None, final=None, level_ms=None, level_children=None,
          direction="auto", bottom_up_ratio=0.0, spill=None, segment_bits=0, far_marks="auto", threads=0):
    o = BfsOpts()
    o.threads = threads
    o.far_marks = FAR_MARKS[far_marks] if isinstance(far_marks, str) else int(far_marks)
    if spill is not None:
        o.spill = spill  # a SPILL_FN the caller keeps alive for the call
        o.segment_bits = segment_bits
    o.struct_size = ctypes.sizeof(BfsOpts)
    o.direction = DIRECTIONS[direction] if isinstance(direction, str) else int(direction)
    o.bottom_up_ratio = bottom_up_ratio
    o.max_depth = max_depth
    o.window_bits = window_bits
    o.device = device
    o.stream = stream
    if final is not None:
        o.final_words = ctypes.cast(final, u64p)
        o.final_cap = len(final)
    if level_ms is not None:
        o.level_ms = level_ms
    if level_children is not None:
        o.level_children = level_children
    return o


def bfs(puzzle, algo, initial=0, max_depth=0, window_bits=0, final=False, levels=False, device=-1,
        direction="auto", bottom_up_ratio=0.0, spill=None, segment_bits=0, restored=False, far_marks="auto",
        threads=0):
    """Runs psb_bfs.  Returns a dict with counts, stats and optionally the final
    arrays (list of 64-bit words in the reference's layout) and per-level data.
    direction: "auto", "top_down" or "bottom_up" (PSB_DIR_*).
    spill: optional callable(depth, segment, stream_bytes, states) receiving
    every depth's frontier as compressed segment streams (2^segment_bits
    states per segment, 0 = 2^32); a truthy return stops the search.  A
    SPILL_FN is passed through as is (it sees the pinned buffer itself).
    far_marks: two-bit long-range marks, "auto", "none", "near" or "all" (PSB_FAR_*).
    threads: threads per block of the top-down two-bit / three-bit level kernels (128, 256, 512; 0 = 128 for
        two-bit pancake and Hanoi searches of 2^32 states or more, else 256).
    restored: 4-peg Hanoi with symmetry, two-bit: also return "restored", the
    per-depth counts weighted by each canonical state's class size
    (HanoiSearch's result)."""
    if isinstance(initial, str):
        initial = puzzle.Parse(initial)
    cap = 1 << 16
    counts = (ctypes.c_uint64 * cap)()
    nd = ctypes.c_uint32()
    fin = None
    if final:
        fin = (ctypes.c_uint64 * puzzle.final_words(algo))()
    lm = (ctypes.c_float * cap)() if levels else None
    lc = (ctypes.c_uint64 * cap)() if levels else None
    fn, runner = _spill_fn(spill)
    o = _opts(max_depth, window_bits, device, None, fin, lm, lc, direction, bottom_up_ratio, fn, segment_bits,
              far_marks, threads)
    rc = (ctypes.c_uint64 * cap)() if restored else None
    if restored:
        o.restored_counts = ctypes.cast(rc, u64p)
    st = BfsStats()
    st.struct_size = ctypes.sizeof(BfsStats)
    runner(lambda: lib().psb_bfs(puzzle.handle, _algo(algo), initial, ctypes.byref(o), counts, cap,
                                 ctypes.byref(nd), ctypes.byref(st)))
    out = {"counts": list(counts[:nd.value]), "stats": st.as_dict()}
    if final:
        out["final"] = list(fin)
    if levels:
        out["level_ms"] = list(lm[:nd.value])
        out["level_children"] = list(lc[:nd.value])
    if restored:
        out["restored"] = list(rc[:nd.value])
    return out


def bfs_segmented(puzzle, initial=0, segment_bits=0, max_depth=0, chunk_states=0, device=-1, directories=(),
                  files_per_path=-1):
    """psb_bfs_segmented: the out-of-core three-layer search (one segment's
    bit arrays on the device at a time).  directories / files_per_path: the
    reference's StoreOptions (segment files there; none = host memory).
    Returns {"counts", "stats"}."""
    if isinstance(initial, str):
        initial = puzzle.Parse(initial)
    cap = 1 << 16
    counts = (ctypes.c_uint64 * cap)()
    nd = ctypes.c_uint32()
    dirs = (ctypes.c_char_p * max(1, len(directories)))(*[os.fsencode(d) for d in directories])
    o = SegmentedOpts(ctypes.sizeof(SegmentedOpts), max_depth, segment_bits, device, chunk_states,
                      ctypes.cast(dirs, ctypes.POINTER(ctypes.c_char_p)), len(directories), files_per_path)
    st = SegmentedStats()
    st.struct_size = ctypes.sizeof(SegmentedStats)
    _check(lib().psb_bfs_segmented(puzzle.handle, initial, ctypes.byref(o), counts, cap, ctypes.byref(nd),
                                   ctypes.byref(st)))
    return {"counts": list(counts[:nd.value]),
            "stats": {k: getattr(st, k) for k, _ in SegmentedStats._fields_ if k not in ("struct_size", "pad")}}


class Store:
    """psb_store: the reference's Store (Common/Store.h:13-178) -- numbered
    segments, each a list of chunks read back in write order; files in
    `directories` (StoreOptions), or host memory without any."""

    def __init__(self, max_segments, name, directories=(), files_per_path=5):
        dirs = (ctypes.c_char_p * max(1, len(directories)))(*[os.fsencode(d) for d in directories])
        h = ctypes.c_void_p()
        _check(lib().psb_store_create(max_segments, name.encode(), dirs, len(directories), files_per_path,
                                      ctypes.byref(h)))
        self._h = h

    def close(self):
        if self._h:
            h, self._h = self._h, None
            _check(lib().psb_store_destroy(h))

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def Write(self, segment, data):
        buf = (ctypes.c_uint8 * max(1, len(data))).from_buffer_copy(bytes(data) or b"\0")
        _check(lib().psb_store_write(self._h, segment, buf, len(data)))

    def Read(self, segment, cap=1 << 24):
        """The next chunk of the segment (b"" after the last one)."""
        buf = (ctypes.c_uint8 * cap)()
        got = ctypes.c_uint64()
        _check(lib().psb_store_read(self._h, segment, buf, cap, ctypes.byref(got)))
        return bytes(buf[:got.value])

    def Rewind(self, segment):
        _check(lib().psb_store_rewind(self._h, segment))

    def Length(self, segment=-1):
        n = ctypes.c_uint64()
        _check(lib().psb_store_length(self._h, segment, ctypes.byref(n)))
        return n.value

    def Delete(self, segment=-1):
        _check(lib().psb_store_delete(self._h, segment))


class BfsSession:
    """psb_bfs_session: device arrays allocated once, reused by run()."""

    def __init__(self, puzzle, algo, window_bits=0, device=-1, direction="auto"):
        self.puzzle = puzzle
        self.algo = _algo(algo)
        self.direction = direction
        h = ctypes.c_void_p()
        o = _opts(0, window_bits, device, direction=direction)
        _check(lib().psb_bfs_session_create(puzzle.handle, self.algo, ctypes.byref(o), ctypes.byref(h)))
        self._h = h
        self._cap = 1 << 16
        self._counts = (ctypes.c_uint64 * self._cap)()

    def run(self, initial=0, max_depth=0, bottom_up_ratio=0.0, spill=None, segment_bits=0):
        nd = ctypes.c_uint32()
        st = BfsStats()
        st.struct_size = ctypes.sizeof(BfsStats)
        fn, runner = _spill_fn(spill)
        o = _opts(max_depth, direction=self.direction, bottom_up_ratio=bottom_up_ratio, spill=fn,
                  segment_bits=segment_bits)
        runner(lambda: lib().psb_bfs_session_run(self._h, initial, ctypes.byref(o), self._counts, self._cap,
                                                 ctypes.byref(nd), ctypes.byref(st)))
        return list(self._counts[:nd.value]), st.as_dict()

    def close(self):
        if getattr(self, "_h", None):
            lib().psb_bfs_session_destroy(self._h)
            self._h = None

    def __del__(self):
        if _lib is not None:
            self.close()


class Engine:
    """psb_engine: many two-bit searches advanced level by level together
    (batched solves, and continuous batching for serving)."""

    def __init__(self, max_instances=4096, max_depths=128, pool_bytes=8 << 30, blocks_per_sm=0, use_graph=True,
                 device=-1, direction="auto", window_bits_offset=0):
        o = EngineOpts()
        o.window_bits_offset = window_bits_offset
        o.direction = DIRECTIONS[direction] if isinstance(direction, str) else int(direction)
        o.struct_size = ctypes.sizeof(EngineOpts)
        o.max_instances = max_instances
        o.max_depths = max_depths
        o.device = device
        o.pool_bytes = pool_bytes
        o.blocks_per_sm = blocks_per_sm
        o.use_graph = 1 if use_graph else 0
        h = ctypes.c_void_p()
        _check(lib().psb_engine_create(ctypes.byref(o), ctypes.byref(h)))
        self._h = h
        self.max_depths = max_depths
        self.max_instances = max_instances

    @staticmethod
    def footprint(puzzle):
        b = ctypes.c_uint64()
        _check(lib().psb_engine_footprint(puzzle.kind, puzzle.a, puzzle.b, ctypes.byref(b)))
        return b.value

    def add(self, puzzle, initial, tag):
        """Admits a search; returns False when the engine is full (no slot or pool space)."""
        slot = ctypes.c_uint32()
        rc = lib().psb_engine_add(self._h, puzzle.kind, puzzle.a, puzzle.b, initial, tag, ctypes.byref(slot))
        if rc == -4:
            return False
        _check(rc)
        return True

    def step(self, levels=1):
        _check(lib().psb_engine_step(self._h, levels))

    def poll(self, cap=None):
        """Finished searches as {tag: per-depth counts}."""
        cap = cap or self.max_instances
        tags = (ctypes.c_uint64 * cap)()
        nd = (ctypes.c_uint32 * cap)()
        counts = (ctypes.c_uint64 * (cap * self.max_depths))()
        n = ctypes.c_uint32()
        _check(lib().psb_engine_poll(self._h, tags, nd, counts, cap, ctypes.byref(n)))
        out = {}
        for i in range(n.value):
            row = i * self.max_depths
            out[tags[i]] = list(counts[row:row + nd[i]])
        return out

    def info(self):
        a, f, l = ctypes.c_uint32(), ctypes.c_uint64(), ctypes.c_uint64()
        _check(lib().psb_engine_info(self._h, ctypes.byref(a), ctypes.byref(f), ctypes.byref(l)))
        return {"active": a.value, "largest_free_bytes": f.value, "levels_run": l.value}

    def close(self):
        if getattr(self, "_h", None):
            lib().psb_engine_destroy(self._h)
            self._h = None

    def __del__(self):
        if _lib is not None:
            self.close()


class Server:
    """psb_server: a solve server with continuous batching on one GPU."""

    def __init__(self, max_instances=1024, max_depths=256, pool_bytes=16 << 30, levels_per_step=1, device=-1,
                 blocks_per_sm=0, window_bits_offset=0, large_states=0):
        """large_states: requests with more states run in the large lane (0 =
        the library's default, None = no large lane)."""
        o = ServerOpts()
        o.struct_size = ctypes.sizeof(ServerOpts)
        o.large_states = (1 << 64) - 1 if large_states is None else large_states
        o.levels_per_step = levels_per_step
        e = o.engine
        e.struct_size = ctypes.sizeof(EngineOpts)
        e.blocks_per_sm = blocks_per_sm
        e.window_bits_offset = window_bits_offset
        e.max_instances = max_instances
        e.max_depths = max_depths
        e.device = device
        e.pool_bytes = pool_bytes
        e.use_graph = 1
        h = ctypes.c_void_p()
        _check(lib().psb_server_start(ctypes.byref(o), ctypes.byref(h)))
        self._h = h
        self.max_depths = max_depths

    def submit(self, puzzle, initial):
        t = ctypes.c_uint64()
        _check(lib().psb_server_submit(self._h, puzzle.kind, puzzle.a, puzzle.b, initial, ctypes.byref(t)))
        return t.value

    def poll(self, cap=1024):
        """Completed requests: {ticket: (status, counts, latency_s)}; eccentricity = len(counts) - 1."""
        tickets = (ctypes.c_uint64 * cap)()
        status = (ctypes.c_int * cap)()
        nd = (ctypes.c_uint32 * cap)()
        counts = (ctypes.c_uint64 * (cap * self.max_depths))()
        lat = (ctypes.c_double * cap)()
        n = ctypes.c_uint32()
        _check(lib().psb_server_poll(self._h, tickets, status, nd, counts, lat, cap, ctypes.byref(n)))
        out = {}
        for i in range(n.value):
            row = i * self.max_depths
            out[tickets[i]] = (status[i], list(counts[row:row + nd[i]]), lat[i])
        return out

    def info(self):
        q, r, c, st = ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_uint64(), ctypes.c_uint64()
        rc = lib().psb_server_info(self._h, ctypes.byref(q), ctypes.byref(r), ctypes.byref(c), ctypes.byref(st))
        return {"queued": q.value, "running": r.value, "completed": c.value, "steps": st.value, "status": rc}

    def stop(self):
        if getattr(self, "_h", None):
            lib().psb_server_stop(self._h)
            self._h = None

    def __del__(self):
        if _lib is not None:
            self.stop()


def release_cached_memory(device=-1):
    """psb_release_cached_memory: return the search arrays' reserved pool memory to the driver."""
    _check(lib().psb_release_cached_memory(device))


def bits_set_stride(d_words, n_bits, first, stride, stream=None):
    """psb_bits_set_stride: BitArray::Set(first + k*stride) on a device bit array (pointer)."""
    _check(lib().psb_bits_set_stride(d_words, n_bits, first, stride, stream))


def bits_scan(d_words, n_bits, clear=False, d_exclude=None, stream=None):
    """psb_bits_scan: (count, sum of indexes mod 2^64) of the set bits; optionally clears them."""
    c, t = ctypes.c_uint64(), ctypes.c_uint64()
    _check(lib().psb_bits_scan(d_words, d_exclude, n_bits, 1 if clear else 0, ctypes.byref(c), ctypes.byref(t), stream))
    return c.value, t.value


def bits_and_not_count(d_words, d_exclude, n_bits, stream=None):
    """psb_bits_and_not_count: words &= ~exclude; returns the bits left."""
    c = ctypes.c_uint64()
    _check(lib().psb_bits_and_not_count(d_words, d_exclude, n_bits, ctypes.byref(c), stream))
    return c.value


def bits_or(d_words, d_other, n_bits, stream=None):
    """psb_bits_or: words |= other."""
    _check(lib().psb_bits_or(d_words, d_other, n_bits, stream))


def frontier_index(data):
    """Block table of a compressed frontier stream held in host memory (bytes)."""
    buf = ctypes.create_string_buffer(bytes(data), len(data))
    n = ctypes.c_uint32()
    _check(lib().psb_frontier_index(buf, len(data), None, 0, ctypes.byref(n)))
    blocks = (CodecBlock * max(n.value, 1))()
    _check(lib().psb_frontier_index(buf, len(data), blocks, n.value, ctypes.byref(n)))
    return blocks, n.value


def frontier_encode(d_bits, first_bit, n_bits, d_out=None, out_cap=0, stream=None):
    """Encodes a device bitmap range (device pointers as ints).  Returns
    (stream_bytes, block_table, n_blocks); with d_out=None only sizes it."""
    nbytes = ctypes.c_uint64()
    nb = ctypes.c_uint32()
    rc = lib().psb_frontier_encode(ctypes.cast(d_bits, u64p), first_bit, n_bits, d_out, out_cap,
                                   ctypes.byref(nbytes), None, 0, ctypes.byref(nb), stream)
    if d_out is None:
        if rc not in (0, -4):
            _check(rc)
        return nbytes.value, None, nb.value
    blocks = (CodecBlock * max(nb.value, 1))()
    _check(lib().psb_frontier_encode(ctypes.cast(d_bits, u64p), first_bit, n_bits, d_out, out_cap,
                                     ctypes.byref(nbytes), blocks, nb.value, ctypes.byref(nb), stream))
    return nbytes.value, blocks, nb.value


def frontier_decode(d_stream, blocks, n_blocks, d_bits, first_bit, n_bits, stream=None):
    _check(lib().psb_frontier_decode(d_stream, blocks, n_blocks, ctypes.cast(d_bits, u64p), first_bit, n_bits,
                                     stream))


def _run(puzzle, algo, initialState):
    return bfs(puzzle, algo, puzzle.Parse(initialState))["counts"]


def InMemoryClassicBFS(puzzle, initialState):
    """Common/InMemoryClassicBFS.cpp:4-45 on the GPU."""
    return _run(puzzle, CLASSIC, initialState)


def InMemoryTwoBitBFS(puzzle, initialState):
    """Common/InMemoryTwoBitBFS.cpp:24-69 on the GPU."""
    return _run(puzzle, TWO_BIT, initialState)


def InMemoryThreeBitBFS(puzzle, initialState):
    """Common/InMemoryThreeBitBFS.cpp:4-48 on the GPU."""
    return _run(puzzle, THREE_BIT, initialState)


def InMemoryFrontierSearch(puzzle, initialState):
    """Common/InMemoryFrontierSearch.cpp:57-112 on the GPU."""
    return _run(puzzle, FRONTIER, initialState)
