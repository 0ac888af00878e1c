"""ctypes binding of the CPU oracle (oracle/liboracle.so) and, when it has been
built, of the reference's own CPU path (oracle/_ref/libpsbref.so).

TEST INFRASTRUCTURE ONLY.  It is imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg, always as the checker or the baseline.  The product
package puzzlesearch_b200 never imports it.
"""
import ctypes
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
KIND = {"sliding": 1, "pancake": 2, "hanoi4": 3, "pancake_opt": 4, "hanoi4_opt": 5, "sliding_opt": 6}
ALGO = {"two_bit": 1, "three_bit": 2, "frontier": 3, "classic": 4}

u64p = ctypes.POINTER(ctypes.c_uint64)
u32p = ctypes.POINTER(ctypes.c_uint32)
u8p = ctypes.POINTER(ctypes.c_uint8)


class _Puzzle(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int), ("a", ctypes.c_int), ("b", ctypes.c_int)]


def build():
    subprocess.check_call(["make", "-s", "-C", HERE], stdout=subprocess.DEVNULL)


_lib = None


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        P = ctypes.POINTER(_Puzzle)
        L.orc_info.argtypes = [P, u64p, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]
        L.orc_parse.argtypes = [P, ctypes.c_char_p, u64p]
        L.orc_to_string.argtypes = [P, ctypes.c_uint64, ctypes.c_char_p, ctypes.c_int]
        L.orc_expand.restype = ctypes.c_int64
        L.orc_expand.argtypes = [P, u64p, u32p, ctypes.c_uint64, u64p, u32p, ctypes.c_uint64]
        L.orc_bfs.argtypes = [P, ctypes.c_int, ctypes.c_uint64, u64p, ctypes.c_int, u64p, ctypes.c_uint64]
        L.orc_final_words.restype = ctypes.c_uint64
        L.orc_final_words.argtypes = [P, ctypes.c_int]
        L.orc_depths.argtypes = [P, ctypes.c_uint64, ctypes.c_void_p]
        L.orc_perm_rank.restype = ctypes.c_uint64
        L.orc_perm_rank.argtypes = [ctypes.POINTER(ctypes.c_int), ctypes.c_int]
        L.orc_perm_unrank.argtypes = [ctypes.c_uint64, ctypes.POINTER(ctypes.c_int), ctypes.c_int]
        L.orc_perm_compact.argtypes = [ctypes.POINTER(ctypes.c_int), ctypes.c_int]
        L.orc_perm_uncompact.argtypes = [ctypes.POINTER(ctypes.c_int), ctypes.c_int]
        L.orc_svi_encode_tuple.argtypes = [u32p, u8p]
        L.orc_svi_decode_tuple.argtypes = [u8p, u32p]
        L.orc_svi_encode.argtypes = [ctypes.c_int, u32p, u8p]
        L.orc_svi_decode.argtypes = [ctypes.POINTER(ctypes.c_int), u8p, u32p]
        L.orc_svi_encode_bounds.argtypes = [ctypes.c_int, u32p, u8p, u8p]
        for f in ("orc_fc_encode", "orc_fc_encode_with_check"):
            getattr(L, f).argtypes = [ctypes.c_int, u32p, u8p]
        for f in ("orc_fc_encode_bitmap", "orc_fc_encode_bitmap_with_check"):
            getattr(L, f).argtypes = [ctypes.c_int, u32p, u8p]
        L.orc_fc_decode.argtypes = [ctypes.POINTER(ctypes.c_int), u8p, u32p]
        L.orc_fc_is_bitmap.argtypes = [u8p]
        for f in ("orc_opbits_encode", "orc_opbits_decode"):
            getattr(L, f).restype = ctypes.c_int64
            getattr(L, f).argtypes = [ctypes.c_int, ctypes.c_uint64, u8p, u8p]
        _lib = L
    return _lib


def _p(spec):
    kind, a, b = spec
    return ctypes.byref(_Puzzle(KIND[kind], a, b))


def info(spec):
    n = ctypes.c_uint64()
    ops, br, odd = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    if lib().orc_info(_p(spec), ctypes.byref(n), ctypes.byref(ops), ctypes.byref(br), ctypes.byref(odd)):
        raise ValueError(f"bad puzzle {spec}")
    return {"indexes": n.value, "ops": ops.value, "branching": br.value, "odd_cycles": bool(odd.value)}


def parse(spec, state):
    out = ctypes.c_uint64()
    if lib().orc_parse(_p(spec), state.encode(), ctypes.byref(out)):
        raise ValueError(f"cannot parse {state!r} for {spec}")
    return out.value


def to_string(spec, index):
    buf = ctypes.create_string_buffer(512)
    if lib().orc_to_string(_p(spec), index, buf, 512) < 0:
        raise ValueError("to_string failed")
    return buf.value.decode()


def expand(spec, parents, opbits=None):
    n = len(parents)
    P = (ctypes.c_uint64 * max(n, 1))(*parents)
    O = (ctypes.c_uint32 * max(n, 1))(*(opbits if opbits is not None else [0] * n))
    cap = max(n, 1) * 16
    C = (ctypes.c_uint64 * cap)()
    CO = (ctypes.c_uint32 * cap)()
    k = lib().orc_expand(_p(spec), P, O, n, C, CO, cap)
    if k < 0:
        raise RuntimeError(f"orc_expand failed {k}")
    return list(C[:k]), list(CO[:k])


def bfs(spec, algo, initial=0, final=False):
    """Returns (counts, final_words or None)."""
    cap = 1 << 16
    counts = (ctypes.c_uint64 * cap)()
    fin = None
    fw = 0
    if final:
        fw = lib().orc_final_words(_p(spec), ALGO[algo])
        fin = (ctypes.c_uint64 * fw)()
    n = lib().orc_bfs(_p(spec), ALGO[algo], initial, counts, cap, fin, fw)
    if n < 0:
        raise RuntimeError(f"orc_bfs failed {n}")
    return list(counts[:n]), (list(fin) if final else None)


def depths(spec, initial=0):
    """Distance of every state from initial as a numpy uint8 array (255 = not
    reached), and the number of depths."""
    import numpy as np
    n = info(spec)["indexes"]
    d = np.empty(n, dtype=np.uint8)
    k = lib().orc_depths(_p(spec), initial, d.ctypes.data)
    if k < 0:
        raise RuntimeError(f"orc_depths failed {k}")
    return d, k


def perm_rank(perm):
    arr = (ctypes.c_int * len(perm))(*perm)
    return lib().orc_perm_rank(arr, len(perm))


def perm_unrank(index, size):
    arr = (ctypes.c_int * size)()
    lib().orc_perm_unrank(index, arr, size)
    return list(arr)


def perm_compact(perm):
    arr = (ctypes.c_int * len(perm))(*perm)
    lib().orc_perm_compact(arr, len(perm))
    return list(arr)


def perm_uncompact(digits):
    arr = (ctypes.c_int * len(digits))(*digits)
    lib().orc_perm_uncompact(arr, len(digits))
    return list(arr)


def svi_encode_tuple(v4):
    out = (ctypes.c_uint8 * 32)()
    n = lib().orc_svi_encode_tuple((ctypes.c_uint32 * 4)(*v4), out)
    return bytes(out[:n])


def svi_decode_tuple(data):
    inp = (ctypes.c_uint8 * 32)(*data)
    v = (ctypes.c_uint32 * 4)()
    n = lib().orc_svi_decode_tuple(inp, v)
    return list(v), n


def _buf_for(count):
    return (ctypes.c_uint8 * (16 + 17 * ((count + 7) // 8 * 2) + 8 + (count + 64) // 8 * 1 + 64))()


def svi_encode(values):
    n = len(values)
    idx = (ctypes.c_uint32 * ((n + 7) // 8 * 8 + 8))(*values)
    out = _buf_for(n)
    k = lib().orc_svi_encode(n, idx, out)
    return bytes(out[:k])


def svi_decode(data):
    size = ctypes.c_int(len(data))
    inp = (ctypes.c_uint8 * (len(data) + 32))(*data)
    count = int.from_bytes(data[:4], "little") if data else 0
    idx = (ctypes.c_uint32 * ((count + 7) // 8 * 8 + 8))()
    n = lib().orc_svi_decode(ctypes.byref(size), inp, idx)
    return list(idx[:n]), size.value


def fc_encode(values, with_check=False):
    n = len(values)
    idx = (ctypes.c_uint32 * ((n + 7) // 8 * 8 + 8))(*values)
    span = (max(values) - min(values)) // 8 + 64 if values else 0
    out = (ctypes.c_uint8 * (17 * ((n + 7) // 8 * 2) + 64 + span))()
    f = lib().orc_fc_encode_with_check if with_check else lib().orc_fc_encode
    k = f(n, idx, out)
    return bytes(out[:k])


def fc_encode_bitmap(values, with_check=False):
    n = len(values)
    idx = (ctypes.c_uint32 * max(n, 1))(*values)
    span = abs(values[-1] - values[0]) // 8 + 64
    out = (ctypes.c_uint8 * (span + 16))()
    f = lib().orc_fc_encode_bitmap_with_check if with_check else lib().orc_fc_encode_bitmap
    k = f(n, idx, out)
    return k if k < 0 else bytes(out[:k])


def fc_decode(data, cap):
    size = ctypes.c_int(len(data))
    inp = (ctypes.c_uint8 * (len(data) + 32))(*data)
    idx = (ctypes.c_uint32 * (cap + 8))()
    n = lib().orc_fc_decode(ctypes.byref(size), inp, idx)
    return list(idx[:n]), size.value


def fc_is_bitmap(data):
    inp = (ctypes.c_uint8 * max(len(data), 8))(*data)
    return bool(lib().orc_fc_is_bitmap(inp))


# --------------------------------------------------------------------------
# The reference itself (oracle/_ref), when built.
# --------------------------------------------------------------------------
_ref = None


def ref_available():
    return os.path.exists(os.path.join(HERE, "_ref", "libpsbref.so"))


def ref():
    global _ref
    if _ref is None:
        L = ctypes.CDLL(os.path.join(HERE, "_ref", "libpsbref.so"))
        L.ref_bfs.argtypes = [ctypes.c_int] * 4 + [ctypes.c_char_p, u64p, ctypes.c_int, ctypes.c_int]
        L.ref_bfs_parents.restype = ctypes.c_int64
        L.ref_bfs_parents.argtypes = [ctypes.c_int] * 4 + [ctypes.c_char_p, u64p, ctypes.c_uint64]
        L.ref_expand.restype = ctypes.c_int64
        L.ref_expand.argtypes = [ctypes.c_int] * 3 + [u64p, u32p, ctypes.c_uint64, u64p, u32p, ctypes.c_uint64]
        L.ref_to_string.argtypes = [ctypes.c_int] * 3 + [ctypes.c_uint64, ctypes.c_char_p, ctypes.c_int]
        L.ref_parse.argtypes = [ctypes.c_int] * 3 + [ctypes.c_char_p, u64p]
        L.ref_indexes_count.restype = ctypes.c_uint64
        L.ref_indexes_count.argtypes = [ctypes.c_int] * 3
        L.ref_svi_encode.argtypes = [ctypes.c_int, u32p, u8p, ctypes.c_int]
        L.ref_fc_encode.argtypes = [ctypes.c_int, u32p, u8p, ctypes.c_int]
        L.ref_fc_encode_with_check.argtypes = [ctypes.c_int, u32p, u8p, ctypes.c_int]
        L.ref_svi_encode_bounds.argtypes = [ctypes.c_int, u32p, u8p, u8p, ctypes.c_int]
        _ref = L
    return _ref


def ref_parse(spec, state):
    """The reference class's own Parse (it exits the process on a board of the
    wrong parity: pass solvable states only)."""
    kind, a, b = spec
    out = ctypes.c_uint64()
    if ref().ref_parse(KIND[kind], a, b, state.encode(), ctypes.byref(out)):
        raise RuntimeError("ref_parse failed")
    return out.value


def ref_to_string(spec, index):
    kind, a, b = spec
    buf = ctypes.create_string_buffer(512)
    if ref().ref_to_string(KIND[kind], a, b, index, buf, 512) < 0:
        raise RuntimeError("ref_to_string failed")
    return buf.value.decode()


def ref_indexes_count(spec):
    kind, a, b = spec
    return ref().ref_indexes_count(KIND[kind], a, b)


def ref_bfs(spec, algo, start):
    kind, a, b = spec
    cap = 1 << 16
    counts = (ctypes.c_uint64 * cap)()
    n = ref().ref_bfs(KIND[kind], a, b, ALGO[algo], start.encode(), counts, cap, 1)
    if n < 0:
        raise RuntimeError(f"ref_bfs failed {n}")
    return list(counts[:n])


def ref_bfs_parents(spec, algo, start, cap):
    kind, a, b = spec
    buf = (ctypes.c_uint64 * cap)()
    n = ref().ref_bfs_parents(KIND[kind], a, b, ALGO[algo], start.encode(), buf, cap)
    if n < 0:
        raise RuntimeError(f"ref_bfs_parents failed {n}")
    return list(buf[:n])


def ref_expand(spec, parents, opbits=None):
    kind, a, b = spec
    n = len(parents)
    P = (ctypes.c_uint64 * max(n, 1))(*parents)
    O = (ctypes.c_uint32 * max(n, 1))(*(opbits if opbits is not None else [0] * n))
    cap = max(n, 1) * 16
    C = (ctypes.c_uint64 * cap)()
    CO = (ctypes.c_uint32 * cap)()
    k = ref().ref_expand(KIND[kind], a, b, P, O, n, C, CO, cap)
    if k < 0:
        raise RuntimeError(f"ref_expand failed {k}")
    return list(C[:k]), list(CO[:k])


def ref_fc_encode(values, with_check=False):
    n = len(values)
    idx = (ctypes.c_uint32 * ((n + 7) // 8 * 8 + 8))(*values)
    cap = 4 << 20
    out = (ctypes.c_uint8 * cap)()
    f = ref().ref_fc_encode_with_check if with_check else ref().ref_fc_encode
    k = f(n, idx, out, cap)
    return bytes(out[:k])


def ref_svi_encode_bounds(values, bounds):
    n = len(values)
    idx = (ctypes.c_uint32 * ((n + 7) // 8 * 8 + 8))(*values)
    bd = (ctypes.c_uint8 * ((n + 7) // 8 * 8 + 8))(*bounds)
    cap = 4 << 20
    out = (ctypes.c_uint8 * cap)()
    k = ref().ref_svi_encode_bounds(n, idx, bd, out, cap)
    return bytes(out[:k])


def segment_stream(offsets):
    """The reference's segment stream for ascending u32 offsets: blocks of
    262,144 FrontierCompression::Encode'd and concatenated
    (Common/CompressedFrontier.cpp:103-140).  offsets: numpy uint32 array."""
    import numpy as np
    out = []
    B = 256 * 1024
    for s in range(0, len(offsets), B):
        blk = np.ascontiguousarray(offsets[s:s + B], dtype=np.uint32)
        n = len(blk)
        idx = np.zeros((n + 7) // 8 * 8 + 8, dtype=np.uint32)
        idx[:n] = blk
        span = int(blk[-1]) - int(blk[0])
        cap = 17 * ((n + 7) // 8 * 2) + 64 + span // 8 + 64
        buf = (ctypes.c_uint8 * cap)()
        k = lib().orc_fc_encode(n, idx.ctypes.data_as(u32p), buf)
        out.append(bytes(buf[:k]))
    return b"".join(out)


def frontier_stream(offsets, nibbles):
    """The reference's frontier-search segment stream for ascending u32
    offsets and their operator bits: blocks of 262,144 StreamVInt::Encode'd
    with bounds and concatenated (CompressedFrontierWriter,
    Common/CompressedFrontier.cpp:56-70)."""
    import numpy as np
    L = lib()
    L.orc_svi_encode_ops.argtypes = [ctypes.c_int, u32p, u8p, u8p]
    out = []
    B = 256 * 1024
    for s in range(0, len(offsets), B):
        blk = np.ascontiguousarray(offsets[s:s + B], dtype=np.uint32)
        n = len(blk)
        adj = (n + 7) // 8 * 8
        idx = np.zeros(adj + 8, dtype=np.uint32)
        idx[:n] = blk
        nib = np.zeros(adj + 8, dtype=np.uint8)
        nib[:n] = nibbles[s:s + n]
        buf = (ctypes.c_uint8 * (4 + 17 * (adj // 4) + adj // 2 + 64))()
        k = L.orc_svi_encode_ops(n, idx.ctypes.data_as(u32p), nib.ctypes.data_as(u8p), buf)
        out.append(bytes(buf[:k]))
    return b"".join(out)


def frontier_nibbles(spec, dist):
    """Operator bits a frontier search holds for each state when its depth is
    the frontier: the OR of (1 << op) over the moves from its neighbours one
    depth closer (InMemoryFrontierSearch.cpp:57-112).  dist: orc_depths.
    One Expand per reached state: for small puzzles only."""
    import numpy as np
    nib = np.zeros(len(dist), dtype=np.uint8)
    P1 = (ctypes.c_uint64 * 1)()
    O1 = (ctypes.c_uint32 * 1)()
    C = (ctypes.c_uint64 * 16)()
    CO = (ctypes.c_uint32 * 16)()
    for p in np.nonzero(dist != 255)[0]:
        P1[0] = int(p)
        n = lib().orc_expand(_p(spec), P1, O1, 1, C, CO, 16)
        for j in range(n):
            c = C[j]
            if dist[c] == dist[p] + 1:
                nib[c] |= 1 << CO[j]
    return nib


def opbits_encode(bits, ops):
    """OpBitsCompression<bits>::Encode (Common/OpBitsCompression.cpp:57-65): bytes."""
    n = len(ops)
    src = (ctypes.c_uint8 * max(n, 1))(*ops)
    out = (ctypes.c_uint8 * max(n, 1))()
    k = lib().orc_opbits_encode(bits, n, src, out)
    if k < 0:
        raise ValueError("count must be a multiple of 8 and bits 2, 4 or 8")
    return bytes(out[:k])


def opbits_decode(bits, data, count):
    src = (ctypes.c_uint8 * max(len(data), 1))(*data)
    out = (ctypes.c_uint8 * max(count, 1))()
    if lib().orc_opbits_decode(bits, count, src, out) < 0:
        raise ValueError("count must be a multiple of 8 and bits 2, 4 or 8")
    return list(out[:count])


def ref_opbits_encode(bits, ops):
    """The reference's own OpBitsCompression<bits>::Encode (oracle/_ref)."""
    L = ref()
    L.ref_opbits_encode.restype = ctypes.c_int64
    L.ref_opbits_encode.argtypes = [ctypes.c_int, ctypes.c_uint64, u8p, u8p]
    n = len(ops)
    src = (ctypes.c_uint8 * max(n, 1))(*ops)
    out = (ctypes.c_uint8 * max(n, 1))()
    k = L.ref_opbits_encode(bits, n, src, out)
    return bytes(out[:k])
