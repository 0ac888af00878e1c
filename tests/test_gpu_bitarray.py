"""Device bit arrays (psb_bits_*) against the reference's BitArray test and numpy.

CommonTests/TestBoolArray.cpp:6-37 sets every 13th bit of a 2^32-bit array,
sums the indexes with ScanBitsAndClear (709490155855181350, twice), and then
expects an empty scan.  The random cases compare Set / ScanBits /
ScanBitsAndClearWithExcl / AndNotAndCount / Or with numpy on ragged sizes."""
import numpy as np
import pytest
import torch

import puzzlesearch_b200 as psb

pytestmark = pytest.mark.gpu
MASK = (1 << 64) - 1


def words(n_bits):
    return torch.zeros((n_bits + 63) // 64, dtype=torch.int64, device="cuda")


def np_bits(t, n_bits):
    w = t.cpu().numpy().view(np.uint64)
    bits = np.unpackbits(w.view(np.uint8), bitorder="little")
    return bits[:n_bits].astype(bool) if n_bits <= bits.size else bits.astype(bool)


def test_reference_kat_2pow32(golden):
    kat = golden["bitarray"]
    n, inc = kat["size"], kat["stride"]
    ba = words(n)  # 512 MB
    for _ in range(2):  # TRY = 2
        psb.bits_set_stride(ba.data_ptr(), n, 0, inc)
        count, total = psb.bits_scan(ba.data_ptr(), n, clear=True)
        assert count == (n + inc - 1) // inc
        assert total == kat["index_sum"], kat["source"]
    assert psb.bits_scan(ba.data_ptr(), n, clear=True) == (0, 0)
    del ba
    torch.cuda.empty_cache()


@pytest.mark.parametrize("n_bits", [1, 63, 64, 65, 1000, 12345, 1 << 20, (1 << 20) + 37])
def test_random_against_numpy(n_bits):
    g = torch.Generator(device="cpu").manual_seed(n_bits)
    nw = (n_bits + 63) // 64
    a = torch.randint(-(1 << 63), (1 << 63) - 1, (nw,), generator=g, dtype=torch.int64)
    b = torch.randint(-(1 << 63), (1 << 63) - 1, (nw,), generator=g, dtype=torch.int64)
    tail = n_bits % 64
    if tail:  # bits beyond the array size are never set
        m = (1 << tail) - 1
        a[-1] = int(np.int64(np.uint64(int(a[-1]) & MASK & m)))
        b[-1] = int(np.int64(np.uint64(int(b[-1]) & MASK & m)))
    da, db = a.cuda(), b.cuda()
    A, B = np_bits(a, n_bits), np_bits(b, n_bits)
    idx = np.nonzero(A)[0].astype(np.uint64)
    # ScanBits (no clear)
    assert psb.bits_scan(da.data_ptr(), n_bits) == (idx.size, int(idx.sum(dtype=np.uint64)))
    # ScanBitsAndClearWithExcl
    ex = np.nonzero(A & ~B)[0].astype(np.uint64)
    assert psb.bits_scan(da.data_ptr(), n_bits, clear=True, d_exclude=db.data_ptr()) == \
        (ex.size, int(ex.sum(dtype=np.uint64)))
    assert psb.bits_scan(da.data_ptr(), n_bits) == (0, 0)
    # Or, AndNotAndCount
    da.copy_(a.cuda())
    psb.bits_or(da.data_ptr(), db.data_ptr(), n_bits)
    assert np.array_equal(np_bits(da, n_bits), A | B)
    da.copy_(a.cuda())
    assert psb.bits_and_not_count(da.data_ptr(), db.data_ptr(), n_bits) == int((A & ~B).sum())
    assert np.array_equal(np_bits(da, n_bits), A & ~B)
    # Set with a stride, on top of existing bits
    for first, stride in ((0, 1), (5, 7), (n_bits // 2, 64), (n_bits - 1, 3)):
        da.copy_(a.cuda())
        psb.bits_set_stride(da.data_ptr(), n_bits, first, stride)
        want = A.copy()
        want[first::stride] = True
        assert np.array_equal(np_bits(da, n_bits), want), (first, stride)
    torch.cuda.synchronize()


def test_bad_arguments():
    with pytest.raises(psb.PsbError):
        psb.bits_set_stride(None, 10, 0, 1)
    t = words(64)
    with pytest.raises(psb.PsbError):
        psb.bits_set_stride(t.data_ptr(), 64, 0, 0)
