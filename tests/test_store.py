"""The segment store (psb_store_*, the reference's Common/Store.h:13-178 and
Common/Store.cpp): chunk order, rewind, delete, and the file layout of
StoreOptions (directories round-robin, filesPerPath 0 / 1 / k).  Host code
only: no GPU."""
import os

import pytest

import puzzlesearch_b200 as psb


def chunks(store, segment):
    out = []
    store.Rewind(segment)
    while True:
        c = store.Read(segment)
        if not c:
            return out
        out.append(c)


def test_memory_store_chunks():
    s = psb.Store(4, "mem")
    s.Write(1, b"abc")
    s.Write(2, b"xy")
    s.Write(1, b"defg")
    s.Write(1, b"")  # Store::Write skips empty chunks
    assert chunks(s, 1) == [b"abc", b"defg"] and chunks(s, 2) == [b"xy"] and chunks(s, 0) == []
    assert s.Length(1) == 7 and s.Length() == 9
    s.Rewind(1)
    assert s.Read(1) == b"abc"
    s.Delete(1)
    assert chunks(s, 1) == [] and s.Length() == 2
    with pytest.raises(psb.PsbError) as e:
        s.Write(4, b"z")
    assert e.value.code == -1
    s.Write(3, b"0123456789")
    with pytest.raises(psb.PsbError) as e:
        s.Read(3, cap=4)
    assert e.value.code == -4
    s.close()


def files(dirs):
    return sorted(os.path.relpath(os.path.join(d, f), os.path.dirname(dirs[0])) for d in dirs for f in os.listdir(d))


@pytest.mark.parametrize("fpp", [0, 1, 3])
def test_file_store_layout(tmp_path, fpp):
    """Segments round-robin over the directories; in each, one file per
    segment (0), one file (1) or k files of consecutive segments; a file
    exists while one of its segments holds data."""
    dirs = [str(tmp_path / "d0"), str(tmp_path / "d1")]
    s = psb.Store(6, "layer", dirs, fpp)
    assert files(dirs) == []
    for seg in range(6):
        s.Write(seg, bytes([seg]) * (seg + 1))
        s.Write(seg, b"|" * 3)
    for seg in range(6):
        assert chunks(s, seg) == [bytes([seg]) * (seg + 1), b"|||"]
    if fpp == 0:
        want = [f"d{seg % 2}/layer_{seg}" for seg in range(6)]
    elif fpp == 1:
        want = ["d0/layer", "d1/layer"]
    else:  # file i of a directory holds segments s with s * 3 // 6 == i
        want = [f"d{seg % 2}/layer_p{seg * 3 // 6}" for seg in range(6)]
    assert files(dirs) == sorted(set(want))
    assert s.Length() == sum(seg + 1 + 3 for seg in range(6))
    # deleting the segments of a file removes it
    for seg in (0, 2, 4):
        s.Delete(seg)
    left = files(dirs)  # the even segments were all of d0's
    assert left and not any(f.startswith("d0") for f in left)
    assert chunks(s, 1) == [b"\x01\x01", b"|||"]
    s.close()
    assert files(dirs) == []


def test_file_store_rewrites_after_emptying(tmp_path):
    d = str(tmp_path / "x")
    s = psb.Store(2, "seg", [d], 1)
    s.Write(0, b"first")
    s.Delete(0)
    assert os.listdir(d) == []
    s.Write(1, b"second")
    assert chunks(s, 1) == [b"second"] and os.path.getsize(os.path.join(d, "seg")) == 6
    s.close()


def test_bad_directory(tmp_path):
    f = tmp_path / "plain"
    f.write_text("not a directory")
    with pytest.raises(psb.PsbError) as e:
        psb.Store(2, "x", [str(f)], 1)
    assert e.value.code == -9
