"""CPU tests of the C ABI (include/psb200.h): the library loads, exports every
declared function, and its host-side logic (puzzle info, Parse, ToString,
argument checks) matches the oracle.  No kernels are launched."""
import ctypes
import math
import os
import random
import re
import subprocess

import pytest

import oracle as O
import puzzlesearch_b200 as psb
from _puzzles import make

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SPECS = [["sliding", 3, 2], ["sliding", 4, 4], ["sliding", 3, 4], ["sliding", 2, 8], ["sliding", 1, 2],
         ["pancake", 2, 0], ["pancake", 9, 0], ["pancake", 13, 0], ["pancake", 16, 0],
         ["hanoi4", 1, 0], ["hanoi4", 7, 1], ["hanoi4", 18, 0], ["hanoi4", 31, 0]]




def declared_functions():
    text = open(os.path.join(REPO, "include", "psb200.h")).read()
    return sorted(set(re.findall(r"^(?:int|const char\*)\s+(psb_\w+)\(", text, re.M)))


def test_library_exports_every_declared_symbol():
    lib = psb.lib()
    names = declared_functions()
    assert len(names) >= 15
    for name in names:
        assert hasattr(lib, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", psb.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (psb_\w+)", out))
    assert set(names) <= exported


def test_library_is_sm100a():
    out = subprocess.run(["cuobjdump", "--list-elf", psb.LIB_PATH], capture_output=True, text=True)
    if out.returncode != 0:
        pytest.skip("cuobjdump unavailable")
    assert "sm_100a" in out.stdout


def test_version():
    assert b"sm_100a" in psb.lib().psb_version()


@pytest.mark.parametrize("spec", SPECS, ids=lambda s: f"{s[0]}{s[1]}x{s[2]}")
def test_info_matches_oracle(spec):
    p = make(spec)
    info = O.info(spec)
    assert p.IndexesCount() == info["indexes"]
    assert p.OperatorsCount() == info["ops"]
    assert p.BranchingFactor() == info["branching"]
    assert p.HasOddLengthCycles() == info["odd_cycles"]


@pytest.mark.parametrize("spec", SPECS, ids=lambda s: f"{s[0]}{s[1]}x{s[2]}")
def test_parse_to_string_match_oracle(spec):
    p = make(spec)
    rng = random.Random(11)
    N = p.IndexesCount()
    for idx in [0, N - 1] + [rng.randrange(N) for _ in range(200)]:
        s = p.ToString(idx)
        assert s == O.to_string(spec, idx)
        assert p.Parse(s) == idx


def test_names():
    assert psb.SlidingTilePuzzleSimple(3, 4).Name() == "Sliding-Tile simple: 3 x 4"
    assert psb.PancakeSimple(13).Name() == "Pancake simple, size: 13"
    assert psb.FourPegHanoiSimple(18).Name() == "Four-Peg Hanoi Towers, size=18; symmetry=0"


def test_known_answer_parse(golden):
    for kat in golden["expand_kats"]:
        if kat["parent"] is None:
            continue
        p = make(kat["puzzle"])
        idx = p.Parse(kat["parent"])
        assert p.ToString(idx) == kat["parent"]
        if kat["parent_index"] is not None:
            assert idx == kat["parent_index"]


def test_argument_errors():
    with pytest.raises(psb.PsbError) as e:
        psb.PancakeSimple(17)
    assert e.value.code == -1
    with pytest.raises(psb.PsbError):
        psb.SlidingTilePuzzleSimple(5, 4)
    with pytest.raises(psb.PsbError):
        psb.FourPegHanoiSimple(0)
    p = psb.PancakeSimple(5)
    with pytest.raises(psb.PsbError):
        p.Parse("0 1 2 3")          # too short
    with pytest.raises(psb.PsbError):
        p.Parse("0 1 2 3 3")        # not a permutation
    with pytest.raises(psb.PsbError):
        p.ToString(math.factorial(5))
    with pytest.raises(psb.PsbError):
        psb.bfs(psb.PancakeSimple(5), "no_such_algo" if False else 9)


def test_frontier_search_rejects_more_than_four_operators():
    # FourBitArray keeps 4 operator bits per state (InMemoryFrontierSearch.cpp:8-53).
    with pytest.raises(psb.PsbError) as e:
        psb.bfs(psb.PancakeSimple(6), "frontier")
    assert e.value.code in (-5, -7)


def test_footprint():
    assert psb.PancakeSimple(13).footprint("three_bit") >= 3 * math.factorial(13) // 8
    assert psb.PancakeSimple(14).footprint("two_bit") >= 2 * math.factorial(14) // 8
    assert psb.FourPegHanoiSimple(18).footprint("two_bit") >= 2 * 4 ** 18 // 8
    assert psb.PancakeSimple(9).final_words("three_bit") == 3 * ((math.factorial(9) + 63) // 64)


def test_noalloc_rejects_unaligned_arrays_on_the_host():
    """psb_bfs_noalloc checks d_arrays' 256-byte alignment before it touches
    the device, so this address is never dereferenced (no GPU needed)."""
    p = psb.PancakeSimple(8)
    cap = 64
    counts = (ctypes.c_uint64 * cap)()
    nd = ctypes.c_uint32()
    for addr in (0x100008, 0x100080):
        rc = psb.lib().psb_bfs_noalloc(p.handle, psb.THREE_BIT, 0, ctypes.cast(addr, psb.u64p), 1 << 20, 0,
                                       None, counts, cap, ctypes.byref(nd))
        with pytest.raises(psb.PsbError) as e:
            psb._check(rc)
        assert e.value.code == -1 and "aligned" in str(e.value)


def test_no_device_error_without_gpu():
    if psb.device_count() > 0:
        pytest.skip("a GPU is visible")
    with pytest.raises(psb.PsbError) as e:
        psb.bfs(psb.PancakeSimple(5), "three_bit")
    assert e.value.code == -7


def test_struct_layouts_match_header(tmp_path):
    """The ctypes mirrors of the ABI structs have the header's size and field
    offsets (a C program compiled against include/psb200.h prints them)."""
    mirrors = {"psb_bfs_opts": psb.BfsOpts, "psb_bfs_stats": psb.BfsStats, "psb_engine_opts": psb.EngineOpts,
               "psb_server_opts": psb.ServerOpts, "psb_codec_block": psb.CodecBlock}
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "psb200.h"', "int main(void) {"]
    for cname, cls in mirrors.items():
        lines.append(f'    printf("{cname} %zu\\n", sizeof({cname}));')
        for f, _ in cls._fields_:
            lines.append(f'    printf("{cname}.{f} %zu\\n", offsetof({cname}, {f}));')
    lines += ["    return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(REPO, "include"), str(src), "-o", str(exe)], check=True)
    out = dict(line.rsplit(" ", 1) for line in subprocess.run([str(exe)], check=True, capture_output=True,
                                                               text=True).stdout.splitlines())
    for cname, cls in mirrors.items():
        assert int(out[cname]) == ctypes.sizeof(cls), cname
        for f, _ in cls._fields_:
            assert int(out[f"{cname}.{f}"]) == getattr(cls, f).offset, (cname, f)


def test_spill_wrapper_host_logic():
    """The Python spill wrapper: the callback sees a copy of the stream, a
    truthy return or an exception stops the search (non-zero to the C side),
    and the exception is raised again after the library call returns."""
    seen = []
    fn, runner = psb._spill_fn(lambda d, g, data, st: seen.append((d, g, data, st)) or d == 4)
    buf = (ctypes.c_uint8 * 5)(1, 2, 3, 4, 5)
    assert fn(None, 3, 1, buf, 5, 9) == 0 and fn(None, 4, 0, buf, 2, 1) == 1
    assert seen == [(3, 1, b"\x01\x02\x03\x04\x05", 9), (4, 0, b"\x01\x02", 1)]
    runner(lambda: 0)
    with pytest.raises(psb.PsbError):
        runner(lambda: -8)

    def boom(*a):
        raise ValueError("disk full")

    fn, runner = psb._spill_fn(boom)
    assert fn(None, 0, 0, buf, 1, 1) == 1
    with pytest.raises(ValueError):
        runner(lambda: -8)
    raw = psb.SPILL_FN(lambda *a: 0)
    assert psb._spill_fn(raw)[0] is raw and psb._spill_fn(None)[0] is None
