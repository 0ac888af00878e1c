"""Frontier compression on the GPU (psb_frontier_encode / decode): the stream
bytes equal the reference's segment stream (FrontierCompression::Encode per
262,144-offset block, concatenated as CompressedSegmentWriter does), checked
against the oracle restatement, which is pinned byte-exact to the reference
itself in tests/test_oracle.py."""
import numpy as np
import pytest

import oracle as O
import puzzlesearch_b200 as psb

CASES = [(1000, 0.01), (1000, 0.5), (100_000, 0.0005), (100_000, 0.2), (3_000_000, 0.003),
         (3_000_000, 0.3), (3_000_000, 0.95), (1 << 24, 0.02), (1 << 24, 0.08), (1 << 22, 0.0)]


def random_bits(n_bits, density, seed):
    rng = np.random.default_rng(seed)
    bits = rng.random(n_bits) < density
    words = np.zeros((n_bits + 63) // 64, dtype=np.uint64)
    pos = np.nonzero(bits)[0].astype(np.uint64)
    np.bitwise_or.at(words, (pos >> 6).astype(np.int64), np.left_shift(np.uint64(1), pos & np.uint64(63)))
    return words, pos.astype(np.uint32)


def test_index_of_oracle_streams():
    """Host block index of reference-format streams (no GPU needed)."""
    for n_bits, density in [(3_000_000, 0.3), (100_000, 0.01), (1 << 22, 0.2)]:
        _, offsets = random_bits(n_bits, density, 7)
        data = O.segment_stream(offsets)
        blocks, n = psb.frontier_index(data)
        assert n == (len(offsets) + 262143) // 262144
        assert sum(blocks[i].count for i in range(n)) == len(offsets)
        assert sum(blocks[i].bytes for i in range(n)) == len(data)
        for i in range(n):
            assert bool(blocks[i].is_bitmap) == O.fc_is_bitmap(data[blocks[i].offset:blocks[i].offset + 8])


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES, ids=lambda c: f"{c[0]}@{c[1]}")
def test_encode_bytes_and_roundtrip(case):
    torch = pytest.importorskip("torch")
    n_bits, density = case
    words, offsets = random_bits(n_bits, density, n_bits)
    d_bits = torch.from_numpy(words.view(np.int64)).cuda()
    expected = O.segment_stream(offsets) if len(offsets) else b""
    size, _, _ = psb.frontier_encode(d_bits.data_ptr(), 0, n_bits)
    assert size == len(expected)
    if size == 0:
        return
    d_out = torch.zeros(size, dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    size2, blocks, nb = psb.frontier_encode(d_bits.data_ptr(), 0, n_bits, d_out.data_ptr(), size)
    got = bytes(d_out.cpu().numpy().tobytes())
    assert got == expected
    d_back = torch.zeros_like(d_bits)
    torch.cuda.synchronize()
    psb.frontier_decode(d_out.data_ptr(), blocks, nb, d_back.data_ptr(), 0, n_bits)
    assert torch.equal(d_back.cpu(), d_bits.cpu())


@pytest.mark.gpu
def test_decode_reference_stream_and_offset_segment():
    torch = pytest.importorskip("torch")
    n_bits = 5_000_000
    words, offsets = random_bits(n_bits, 0.1, 3)
    data = O.segment_stream(offsets)
    blocks, nb = psb.frontier_index(data)
    d_in = torch.frombuffer(bytearray(data), dtype=torch.uint8).cuda()
    pad = 64 * 1000  # the segment starts inside a larger bitmap
    d_bits = torch.zeros((pad + n_bits + 63) // 64 + 1, dtype=torch.int64, device="cuda")
    torch.cuda.synchronize()
    psb.frontier_decode(d_in.data_ptr(), blocks, nb, d_bits.data_ptr(), pad, n_bits)
    got = d_bits.cpu().numpy().view(np.uint64)[pad // 64: pad // 64 + len(words)]
    assert np.array_equal(got, words)
    # and encoding from that offset reproduces the stream
    size, _, _ = psb.frontier_encode(d_bits.data_ptr(), pad, n_bits)
    d_out = torch.zeros(size, dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    psb.frontier_encode(d_bits.data_ptr(), pad, n_bits, d_out.data_ptr(), size)
    assert bytes(d_out.cpu().numpy().tobytes()) == data


@pytest.mark.gpu
def test_bfs_frontier_spill_roundtrip():
    """The last level of a three-bit search (final 'cur' array), compressed on
    the GPU, copied to pinned host memory and decoded back."""
    torch = pytest.importorskip("torch")
    p = psb.PancakeSimple(11)
    r = psb.bfs(p, "three_bit", 0, final=True)
    N = p.IndexesCount()
    W = (N + 63) // 64
    cur = np.array(r["final"][W:2 * W], dtype=np.uint64)
    d_cur = torch.from_numpy(cur.view(np.int64)).cuda()
    size, _, _ = psb.frontier_encode(d_cur.data_ptr(), 0, N)
    d_out = torch.zeros(size, dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    _, blocks, nb = psb.frontier_encode(d_cur.data_ptr(), 0, N, d_out.data_ptr(), size)
    host = torch.empty(size, dtype=torch.uint8, pin_memory=True)
    host.copy_(d_out)
    pos = np.nonzero(np.unpackbits(cur.view(np.uint8), bitorder="little"))[0].astype(np.uint32)
    assert bytes(host.numpy().tobytes()) == O.segment_stream(pos)
    assert sum(blocks[i].count for i in range(nb)) == r["counts"][-1]


def mixed_bits(n_bits, pieces, seed):
    """A bitmap whose density changes along it: pieces = [(fraction, density)]."""
    rng = np.random.default_rng(seed)
    bits = np.zeros(n_bits, dtype=bool)
    at = 0
    for frac, dens in pieces:
        n = int(n_bits * frac)
        bits[at:at + n] = rng.random(n) < dens
        at += n
    words = np.zeros((n_bits + 63) // 64, dtype=np.uint64)
    pos = np.nonzero(bits)[0].astype(np.uint64)
    np.bitwise_or.at(words, (pos >> 6).astype(np.int64), np.left_shift(np.uint64(1), pos & np.uint64(63)))
    return words, pos.astype(np.uint32)


MIXED = [
    (1 << 24, [(0.3, 0.5), (0.4, 0.004), (0.3, 0.9)]),
    (1 << 24, [(0.5, 0.001), (0.1, 0.6), (0.4, 0.03)]),
    (12_000_001, [(0.2, 0.0), (0.2, 0.15), (0.4, 0.06), (0.2, 1.0)]),
    (1 << 23, [(0.05, 1.0), (0.95, 0.0002)]),
]


@pytest.mark.gpu
@pytest.mark.parametrize("case", range(len(MIXED)))
def test_encode_mixed_density_segments(case):
    """Segments whose blocks are partly bitmap and partly StreamVInt coded,
    with block boundaries where the density changes."""
    torch = pytest.importorskip("torch")
    n_bits, pieces = MIXED[case]
    words, offsets = mixed_bits(n_bits, pieces, 100 + case)
    expected = O.segment_stream(offsets)
    d_bits = torch.from_numpy(words.view(np.int64)).cuda()
    size, _, _ = psb.frontier_encode(d_bits.data_ptr(), 0, n_bits)
    assert size == len(expected)
    d_out = torch.zeros(size, dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    _, blocks, nb = psb.frontier_encode(d_bits.data_ptr(), 0, n_bits, d_out.data_ptr(), size)
    assert bytes(d_out.cpu().numpy().tobytes()) == expected
    kinds = {bool(blocks[i].is_bitmap) for i in range(nb)}
    assert len(kinds) == 2
    d_back = torch.zeros_like(d_bits)
    torch.cuda.synchronize()
    psb.frontier_decode(d_out.data_ptr(), blocks, nb, d_back.data_ptr(), 0, n_bits)
    assert torch.equal(d_back.cpu(), d_bits.cpu())


@pytest.mark.gpu
@pytest.mark.parametrize("bits", [2, 4, 8])
def test_opbits_codec_matches_oracle(bits, golden):
    """psb_opbits_encode / decode (OpBitsCompression<bits>) on the GPU: the
    packed bytes equal the oracle's, which equal the reference's
    (tests/test_oracle.py), and decoding gives the op bits back; the
    reference's own test inputs and a large random array."""
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(bits)
    arrays = [np.array(v["values"], dtype=np.uint8) for v in golden["opbits"] if v["bits"] == bits]
    arrays.append(rng.integers(0, 1 << bits, size=1 << 20, dtype=np.uint8))
    for ops in arrays:
        d_ops = torch.from_numpy(ops).cuda()
        d_packed = torch.empty(len(ops) * bits // 8, dtype=torch.uint8, device="cuda")
        d_back = torch.empty(len(ops), dtype=torch.uint8, device="cuda")
        psb._check(psb.lib().psb_opbits_encode(bits, d_ops.data_ptr(), len(ops), d_packed.data_ptr(), None))
        psb._check(psb.lib().psb_opbits_decode(bits, d_packed.data_ptr(), len(ops), d_back.data_ptr(), None))
        torch.cuda.synchronize()
        assert bytes(d_packed.cpu().numpy().tobytes()) == O.opbits_encode(bits, ops.tolist())
        assert np.array_equal(d_back.cpu().numpy(), ops)


def test_opbits_argument_errors():
    """Checked on the host before anything reaches the device."""
    with pytest.raises(psb.PsbError):
        psb._check(psb.lib().psb_opbits_encode(3, 0x1000, 8, 0x2000, None))
    with pytest.raises(psb.PsbError):
        psb._check(psb.lib().psb_opbits_encode(4, 0x1000, 12, 0x2000, None))
    with pytest.raises(psb.PsbError):
        psb._check(psb.lib().psb_opbits_decode(4, 0x1002, 8, 0x2000, None))
