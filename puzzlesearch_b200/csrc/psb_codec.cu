// psb_codec.cu -- frontier compression on the GPU, byte-exact with the
// reference's segment stream:
//   FrontierCompression::Encode / Decode   Common/FrontierCompression.cpp:36-125
//   StreamVInt::Encode / Decode            Common/StreamVInt.cpp:116-251
//   CompressedSegmentWriter framing        Common/CompressedFrontier.cpp:103-140
//
// A segment's frontier (the set bits of a bitmap range of at most 2^32
// states, as u32 offsets in ascending order) is cut into blocks of 262,144
// offsets (StreamVInt::MAX_INDEXES_COUNT).  Each block becomes either
//   * a bitmap block: [u32 words | 0x80000000][u32 first][bitmap of v - first - 1],
//     chosen when count > 128 and the bitmap's bits < 10*count - 8; or
//   * a StreamVInt block: [u32 count], then the deltas (first value raw),
//     zero-padded to a multiple of 8 values, as tuples of four values:
//     one descriptor byte (2 bits per value = bytes - 1), then each value's
//     1..4 little-endian bytes.
// The blocks are concatenated.  Decoding needs each block's start; the
// encoder returns that as a side table (psb_codec_block), and
// psb_frontier_index builds it on the host for a stream from elsewhere.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <new>
#include <string>
#include <memory>
#include <vector>

#include "../../include/psb200.h"
#include "psb_internal.h"

namespace {

constexpr uint32_t kBlock = 256 * 1024;  // StreamVInt::MAX_INDEXES_COUNT (Common/StreamVInt.h:9)
constexpr uint32_t kMap = 0x80000000u;   // CODEC_MAP (Common/FrontierCompression.cpp:6)
constexpr int kT = 256;

#define CD_CUDA(call)                                                                           \
    do {                                                                                        \
        cudaError_t e_ = (call);                                                                \
        if (e_ != cudaSuccess)                                                                  \
            return psb_set_error(e_ == cudaErrorMemoryAllocation ? PSB_ERR_NOMEM : PSB_ERR_CUDA, \
                                 (std::string(#call) + ": " + cudaGetErrorString(e_)).c_str());  \
    } while (0)

__device__ __forceinline__ uint64_t masked_word(const uint64_t* bits, uint64_t w, uint64_t n_words, uint64_t n_bits) {
    uint64_t v = bits[w];
    if (w == n_words - 1 && (n_bits & 63)) v &= (uint64_t(1) << (n_bits & 63)) - 1;
    return v;
}

// Per-block sums of word popcounts (kT threads x 16 words per block).
__global__ void k_block_sums(const uint64_t* bits, uint64_t n_words, uint64_t n_bits, unsigned long long* bsum) {
    const uint64_t base = uint64_t(blockIdx.x) * kT * 16;
    uint32_t c = 0;
    for (int k = 0; k < 16; ++k) {
        const uint64_t w = base + uint64_t(k) * kT + threadIdx.x;
        if (w < n_words) c += __popcll(masked_word(bits, w, n_words, n_bits));
    }
    c = __reduce_add_sync(0xFFFFFFFFu, c);
    __shared__ uint32_t s[kT / 32];
    if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long t = 0;
        for (int i = 0; i < kT / 32; ++i) t += s[i];
        bsum[blockIdx.x] = t;
    }
}

// Exclusive scan of n u64 values in place by one CTA of kScanT threads
// (chunk sums, tuple-group sums: at most a few hundred thousand values), in
// tiles of kScanT * 16 values: thread t sums values 16 t .. 16 t + 15 of a
// tile, warp shuffles and one pass over the warp totals rank them.
constexpr int kScanT = 1024;
__global__ void __launch_bounds__(kScanT) k_scan_small(unsigned long long* v, uint64_t n, unsigned long long* total) {
    __shared__ unsigned long long warp_tot[kScanT / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned long long carry = 0;
    for (uint64_t base = 0; base < n; base += uint64_t(kScanT) * 16) {
        const uint64_t i0 = base + uint64_t(threadIdx.x) * 16;
        unsigned long long x[16], c = 0;
#pragma unroll
        for (int k = 0; k < 16; ++k) {
            x[k] = i0 + k < n ? v[i0 + k] : 0;
            c += x[k];
        }
        unsigned long long inc = c;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned long long y = __shfl_up_sync(0xFFFFFFFFu, inc, o);
            if (lane >= o) inc += y;
        }
        if (lane == 31) warp_tot[warp] = inc;
        __syncthreads();
        if (warp == 0) {
            unsigned long long t = warp_tot[lane];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const unsigned long long y = __shfl_up_sync(0xFFFFFFFFu, t, o);
                if (lane >= o) t += y;
            }
            warp_tot[lane] = t;  // inclusive over warps
        }
        __syncthreads();
        unsigned long long run = carry + (warp ? warp_tot[warp - 1] : 0) + inc - c;
#pragma unroll
        for (int k = 0; k < 16; ++k) {
            if (i0 + k < n) v[i0 + k] = run;
            run += x[k];
        }
        carry += warp_tot[kScanT / 32 - 1];
        __syncthreads();
    }
    if (threadIdx.x == 0) *total = carry;
}

// Large exclusive scan in place: group sums (4096 values per block), a scan of
// the group sums, then a per-group pass.
__global__ void k_group_sums(const unsigned long long* v, uint64_t n, unsigned long long* gsum) {
    const uint64_t base = uint64_t(blockIdx.x) * kT * 16 + uint64_t(threadIdx.x) * 16;
    unsigned long long c = 0;
    for (int k = 0; k < 16; ++k) if (base + k < n) c += v[base + k];
    __shared__ unsigned long long s[kT];
    s[threadIdx.x] = c;
    __syncthreads();
    for (int o = kT / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) s[threadIdx.x] += s[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) gsum[blockIdx.x] = s[0];
}

__global__ void k_group_scan(unsigned long long* v, uint64_t n, const unsigned long long* gsum) {
    const uint64_t base = uint64_t(blockIdx.x) * kT * 16 + uint64_t(threadIdx.x) * 16;
    unsigned long long x[16], c = 0;
    for (int k = 0; k < 16; ++k) { x[k] = base + k < n ? v[base + k] : 0; c += x[k]; }
    __shared__ unsigned long long s[kT];
    s[threadIdx.x] = c;
    __syncthreads();
    for (int o = 1; o < kT; o <<= 1) {
        const unsigned long long y = threadIdx.x >= o ? s[threadIdx.x - o] : 0;
        __syncthreads();
        s[threadIdx.x] += y;
        __syncthreads();
    }
    unsigned long long run = gsum[blockIdx.x] + s[threadIdx.x] - c;
    for (int k = 0; k < 16; ++k) {
        if (base + k < n) v[base + k] = run;
        run += x[k];
    }
}

// Inclusive block-wide sum scan of one value per thread (kT threads).
__device__ __forceinline__ uint32_t block_inclusive_scan(uint32_t v, uint32_t* warp_tot) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, v, o);
        if (lane >= o) v += y;
    }
    if (lane == 31) warp_tot[warp] = v;
    __syncthreads();
    uint32_t before = 0;
    for (int w = 0; w < warp; ++w) before += warp_tot[w];
    __syncthreads();
    return before + v;
}

// Sum of one value per thread over the CTA, written by thread 0.
__device__ __forceinline__ void chunk_total(uint32_t c, unsigned long long* out) {
    __shared__ uint32_t warp_tot[kT / 32];
    c = __reduce_add_sync(0xFFFFFFFFu, c);
    if ((threadIdx.x & 31) == 0) warp_tot[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long t = 0;
        for (int i = 0; i < kT / 32; ++i) t += warp_tot[i];
        *out = t;
    }
}

__device__ __forceinline__ uint32_t vbytes(uint32_t x) { return x >> 24 ? 4 : x >> 16 ? 3 : x >> 8 ? 2 : 1; }

struct BlockInfo {
    unsigned long long out_off;  // byte offset of the block in the stream
    uint32_t count, first, last, is_bitmap;
    unsigned long long bytes;
};

// A StreamVInt block in tuple order: its first tuple and its block number.
struct SviRef {
    unsigned long long tuple0;
    uint32_t block, pad;
};

// Writes the ascending offsets of the set bits that fall in StreamVInt
// blocks, at their rank (offset list position = rank; bitmap blocks need no
// list: their words are copied from the bitmap).  One CTA per chunk of
// kT * 16 words; warp w takes the chunk's words 512 w .. 512 w + 511, 32 at a
// time, lane l word 32 i + l, so every load is coalesced.  A first pass
// counts each warp's offsets (one CTA scan of the 8 warp totals gives the
// warps' first ranks); the second pass reloads the words (from L1) and ranks
// each lane's offsets by a warp scan, so neighbouring lanes store
// neighbouring ranks.
__global__ void __launch_bounds__(kT) k_compact(const uint64_t* bits, uint64_t n_words, uint64_t n_bits,
                                                const unsigned long long* bsum, uint64_t nbs, uint64_t count,
                                                const BlockInfo* blocks, uint32_t* idx) {
    __shared__ uint32_t warp_tot[kT / 32];
    // Chunks with no offsets, or whose offsets all fall in bitmap blocks,
    // have nothing to list (uniform over the CTA: the chunk's rank range).
    const unsigned long long r_lo = bsum[blockIdx.x];
    const unsigned long long r_hi = blockIdx.x + 1 < nbs ? bsum[blockIdx.x + 1] : count;
    if (r_hi == r_lo) return;
    bool all_bitmap = true;
    for (uint64_t b = r_lo / kBlock; b <= (r_hi - 1) / kBlock; ++b) all_bitmap = all_bitmap && blocks[b].is_bitmap;
    if (all_bitmap) return;
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const uint64_t w0 = uint64_t(blockIdx.x) * kT * 16 + uint64_t(warp) * 512 + lane;
    uint32_t c = 0;
#pragma unroll 4
    for (int i = 0; i < 16; ++i) {
        const uint64_t w = w0 + 32u * i;
        if (w < n_words) c += __popcll(masked_word(bits, w, n_words, n_bits));
    }
    // The CTA's ranks, warp by warp (warp order is word order).
    const uint32_t wsum = __reduce_add_sync(0xFFFFFFFFu, c);
    if (lane == 0) warp_tot[warp] = wsum;
    __syncthreads();
    unsigned long long r = r_lo;
    for (uint32_t k = 0; k < warp; ++k) r += warp_tot[k];
    if (wsum == 0) return;
    for (int i = 0; i < 16; ++i) {
        const uint64_t w = w0 + 32u * i;
        uint64_t m = w < n_words ? masked_word(bits, w, n_words, n_bits) : 0;
        const uint32_t cnt = __popcll(m);
        uint32_t incl = cnt;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
            if (lane >= uint32_t(o)) incl += y;
        }
        const uint32_t total = __shfl_sync(0xFFFFFFFFu, incl, 31);
        // The 32 words' offsets in rank order, 32 at a time: lane l stores
        // rank r + k, k = base + l, so a warp's stores are contiguous.
        for (uint32_t base = 0; base < total; base += 32) {
            const uint32_t k = base + lane;
            uint32_t lo = 0, hi = 31;  // source lane: the first whose inclusive count exceeds k
#pragma unroll
            for (int step = 0; step < 5; ++step) {
                const uint32_t mid = (lo + hi) >> 1;
                if (__shfl_sync(0xFFFFFFFFu, incl, int(mid)) > k) hi = mid;
                else lo = mid + 1;
            }
            const uint32_t before = __shfl_sync(0xFFFFFFFFu, incl - cnt, int(lo));
            const uint64_t word = __shfl_sync(0xFFFFFFFFu, m, int(lo));
            if (k < total) {
                const unsigned long long rank = r + k;
                if (!blocks[rank / kBlock].is_bitmap)
                    idx[rank] = uint32_t((w0 + 32u * i - lane + lo) * 64 + psb::select_bit(word, k - before));
            }
        }
        r += total;
    }
}

// First and last offset of every block (ranks b * kBlock and the block's
// last rank), by select: the chunk holding the rank from the chunk prefix
// sums (bsum, chunks of kT * 16 words), then a block scan of that chunk's
// per-thread counts (thread t: words 16 t .. 16 t + 15).  CTAs 2b and 2b + 1
// serve block b.
__global__ void __launch_bounds__(kT) k_select_blocks(const uint64_t* bits, uint64_t n_words, uint64_t n_bits,
                                                      const unsigned long long* bsum, uint64_t nbs, uint64_t count,
                                                      BlockInfo* blocks, uint32_t nb) {
    __shared__ uint32_t warp_tot[kT / 32];
    const uint32_t b = blockIdx.x / 2;
    const bool last = blockIdx.x & 1;
    const uint64_t end = (uint64_t(b) + 1) * kBlock < count ? (uint64_t(b) + 1) * kBlock : count;
    const uint64_t r = last ? end - 1 : uint64_t(b) * kBlock;
    uint64_t lo = 0, hi = nbs;  // largest chunk lo with bsum[lo] <= r (bsum[0] = 0)
    while (hi - lo > 1) {
        const uint64_t mid = (lo + hi) / 2;
        if (bsum[mid] <= r) lo = mid; else hi = mid;
    }
    const uint64_t rem = r - bsum[lo];
    const uint64_t w0 = lo * kT * 16 + uint64_t(threadIdx.x) * 16;
    uint64_t v[16];
    uint32_t c = 0;
#pragma unroll
    for (int k = 0; k < 16; ++k) {
        v[k] = w0 + k < n_words ? masked_word(bits, w0 + k, n_words, n_bits) : 0;
        c += __popcll(v[k]);
    }
    const uint32_t inc = block_inclusive_scan(c, warp_tot);
    const uint32_t exc = inc - c;
    if (rem < exc || rem >= inc) return;  // exactly one thread holds the rank
    uint64_t left = rem - exc;
    for (int k = 0; k < 16; ++k) {
        const uint32_t ck = __popcll(v[k]);
        if (left < ck) {
            uint64_t x = v[k];
            for (uint64_t i = 0; i < left; ++i) x &= x - 1;
            const uint32_t pos = uint32_t((w0 + k) * 64 + (__ffsll((long long)x) - 1));
            if (last) blocks[b].last = pos; else blocks[b].first = pos;
            return;
        }
        left -= ck;
    }
}

// FrontierCompression::Encode (FrontierCompression.cpp:92-102): a block is a
// bitmap block when it holds more than 128 offsets and its bitmap is smaller
// than 10 bits per offset.
// With operator bits (force_svi) every block is a StreamVInt block, as
// CompressedFrontierWriter writes them (Common/CompressedFrontier.cpp:63-70).
__global__ void k_block_decide(uint64_t count, BlockInfo* blocks, uint32_t nb, int force_svi) {
    const uint32_t b = blockIdx.x * kT + threadIdx.x;
    if (b >= nb) return;
    BlockInfo& bi = blocks[b];
    const uint64_t r0 = uint64_t(b) * kBlock;
    const uint32_t n = uint32_t(count - r0 < kBlock ? count - r0 : kBlock);
    bi.count = n;
    const uint64_t bm_bytes = (uint64_t(bi.last) - bi.first + 63) / 64 * 8 + 8;
    bi.is_bitmap = (!force_svi && n > 128 && bm_bytes * 8 < uint64_t(n) * 10 - 8) ? 1 : 0;
    bi.bytes = bi.is_bitmap ? bm_bytes : 0;
    bi.out_off = 0;
}

// Value of rank position k (0-based) of block b after the in-place delta, 0 past the count.
__device__ __forceinline__ uint32_t delta_at(const uint32_t* idx, uint64_t r0, uint32_t count, uint32_t k) {
    if (k >= count) return 0;
    const uint32_t v = idx[r0 + k];
    return k == 0 ? v : v - idx[r0 + k - 1];
}

// The StreamVInt block that holds tuple t (the last ref with tuple0 <= t).
__device__ __forceinline__ uint32_t svi_of(const SviRef* refs, uint32_t n_refs, uint64_t t) {
    uint32_t lo = 0, hi = n_refs;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) / 2;
        if (refs[mid].tuple0 <= t) lo = mid; else hi = mid;
    }
    return lo;
}

// Tuple lengths of the StreamVInt blocks: 1 descriptor byte + 1..4 bytes per value.
__global__ void k_tuple_len(const uint32_t* idx, const BlockInfo* blocks, const SviRef* refs, uint32_t n_refs,
                            uint64_t tuples, unsigned long long* tlen) {
    const uint64_t t = blockIdx.x * uint64_t(kT) + threadIdx.x;
    if (t >= tuples) return;
    const SviRef ref = refs[svi_of(refs, n_refs, t)];
    const uint32_t k = uint32_t(t - ref.tuple0) * 4;
    const uint32_t count = blocks[ref.block].count;
    const uint64_t r0 = uint64_t(ref.block) * kBlock;
    uint32_t len = 1;
    for (int q = 0; q < 4; ++q) len += vbytes(delta_at(idx, r0, count, k + q));
    tlen[t] = len;
}

// Bytes of each StreamVInt block: header, tuples and, with operator bits,
// the bounds (one nibble per padded value, StreamVInt.cpp:253-275).
__global__ void k_block_bytes(BlockInfo* blocks, const SviRef* refs, uint32_t n_refs,
                              const unsigned long long* tscan, uint64_t tuples, unsigned long long total,
                              int with_ops) {
    const uint32_t j = blockIdx.x * kT + threadIdx.x;
    if (j >= n_refs) return;
    BlockInfo& bi = blocks[refs[j].block];
    const uint64_t t0 = refs[j].tuple0, t1 = j + 1 < n_refs ? refs[j + 1].tuple0 : tuples;
    const unsigned long long end = t1 < tuples ? tscan[t1] : total;
    bi.bytes = 4 + (end - tscan[t0]) + (with_ops ? (uint64_t(bi.count) + 7) / 8 * 4 : 0);
}

// Bounds of the StreamVInt blocks (StreamVInt::EncodeBounds,
// StreamVInt.cpp:139-147,193-198): the operator nibble of each value, 8 per
// group packed as bytes b_q | b_(q+4) << 4, after the block's tuples.  The
// nibble of offset v is state nib_first + v of the 4-bit array `nib` (NULL:
// every nibble is 0); values past the count have nibble 0.  One thread per
// group of 8 values (two tuples).
__global__ void k_write_bounds(const uint32_t* idx, const BlockInfo* blocks, const SviRef* refs, uint32_t n_refs,
                               uint64_t groups, const uint64_t* nib, uint64_t nib_first, uint8_t* out) {
    const uint64_t g = blockIdx.x * uint64_t(kT) + threadIdx.x;
    if (g >= groups) return;
    const SviRef ref = refs[svi_of(refs, n_refs, 2 * g)];
    const uint32_t k = uint32_t(2 * g - ref.tuple0) * 4;  // first value of the group in its block
    const BlockInfo bi = blocks[ref.block];
    const uint64_t r0 = uint64_t(ref.block) * kBlock;
    const uint64_t adj = (uint64_t(bi.count) + 7) / 8 * 8;
    uint8_t* p = out + bi.out_off + bi.bytes - adj / 2 + k / 2;
    uint32_t b[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        b[j] = 0;
        if (nib && k + j < bi.count) {
            const uint64_t state = nib_first + idx[r0 + k + j];
            b[j] = uint32_t(nib[state >> 4] >> (4 * (state & 15))) & 15u;
        }
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) p[q] = uint8_t(b[q] | (b[q + 4] << 4));
}

__global__ void k_write_svi(const uint32_t* idx, const BlockInfo* blocks, const SviRef* refs, uint32_t n_refs,
                            uint64_t tuples, const unsigned long long* tscan, uint8_t* out) {
    const uint64_t t = blockIdx.x * uint64_t(kT) + threadIdx.x;
    if (t >= tuples) return;
    const SviRef ref = refs[svi_of(refs, n_refs, t)];
    const uint32_t k = uint32_t(t - ref.tuple0) * 4;
    const BlockInfo bi = blocks[ref.block];
    const uint64_t r0 = uint64_t(ref.block) * kBlock;
    uint8_t* p = out + bi.out_off + 4 + (tscan[t] - tscan[ref.tuple0]);
    if (k == 0) {
        uint8_t* h = out + bi.out_off;
        h[0] = uint8_t(bi.count); h[1] = uint8_t(bi.count >> 8); h[2] = uint8_t(bi.count >> 16); h[3] = uint8_t(bi.count >> 24);
    }
    uint8_t desc = 0;
    int pos = 1;
    for (int q = 0; q < 4; ++q) {
        const uint32_t x = delta_at(idx, r0, bi.count, k + q);
        const uint32_t nbytes = vbytes(x);
        desc |= uint8_t((nbytes - 1) << (2 * q));
        for (uint32_t i = 0; i < nbytes; ++i) p[pos++] = uint8_t(x >> (8 * i));
    }
    p[0] = desc;
}

// Bitmap block: bit j of output word i is state first + 1 + 64 i + j (<= last).
// A chunk (kT * 16 words) with no set bits; its words may be stale scratch
// (an extraction skips chunks of windows that hold no frontier state).
__device__ __forceinline__ bool chunk_empty(const unsigned long long* bsum, uint64_t nbs, uint64_t count,
                                            uint64_t w) {
    const uint64_t k = w / (kT * 16);
    return (k + 1 < nbs ? bsum[k + 1] : count) == bsum[k];
}

__device__ __forceinline__ uint64_t live_word(const uint64_t* bits, uint64_t w, uint64_t n_words, uint64_t n_bits,
                                              const unsigned long long* bsum, uint64_t nbs, uint64_t count) {
    return chunk_empty(bsum, nbs, count, w) ? 0 : masked_word(bits, w, n_words, n_bits);
}

__global__ void k_write_bitmap(const uint64_t* bits, uint64_t n_words, uint64_t n_bits, const BlockInfo* blocks,
                               const unsigned long long* bsum, uint64_t nbs, uint64_t count, uint8_t* out) {
    const BlockInfo bi = blocks[blockIdx.y];
    if (!bi.is_bitmap) return;
    const uint64_t words = (uint64_t(bi.last) - bi.first + 63) / 64;
    uint8_t* p = out + bi.out_off;
    const uint64_t i = blockIdx.x * uint64_t(kT) + threadIdx.x;
    if (i == 0) {
        const uint32_t h = uint32_t(words) | kMap;
        for (int q = 0; q < 4; ++q) p[q] = uint8_t(h >> (8 * q));
        for (int q = 0; q < 4; ++q) p[4 + q] = uint8_t(bi.first >> (8 * q));
    }
    if (i >= words) return;
    const uint64_t start = uint64_t(bi.first) + 1 + 64 * i;  // first state of this output word
    const uint64_t w0 = start >> 6, sh = start & 63;
    uint64_t v = live_word(bits, w0, n_words, n_bits, bsum, nbs, count) >> sh;
    if (sh && w0 + 1 < n_words) v |= live_word(bits, w0 + 1, n_words, n_bits, bsum, nbs, count) << (64 - sh);
    const uint64_t hi = start + 63;  // last state this word covers
    if (hi > bi.last) {
        const uint64_t keep = uint64_t(bi.last) - start + 1;  // 0..63
        v &= keep >= 64 ? ~uint64_t(0) : ((uint64_t(1) << keep) - 1);
    }
    for (int q = 0; q < 8; ++q) p[8 + 8 * i + q] = uint8_t(v >> (8 * q));
}

// Decode: one warp per block; StreamVInt blocks are walked by lane 0 (the
// tuple chain is sequential), bitmap blocks are spread over the lanes.
__global__ void k_decode(const uint8_t* in, const psb_codec_block* blocks, uint32_t nb, uint64_t* bits,
                         uint64_t n_bits, unsigned long long* err, int bitmaps_only = 0) {
    const uint32_t b = blockIdx.x;
    if (b >= nb) return;
    const psb_codec_block bk = blocks[b];
    if (bitmaps_only && !bk.is_bitmap) return;
    const uint8_t* p = in + bk.offset;
    auto put = [&](uint64_t v) {
        if (v >= n_bits) { atomicOr(err, 1ull); return; }
        atomicOr(reinterpret_cast<unsigned long long*>(bits) + (v >> 6), 1ull << (v & 63));
    };
    if (bk.is_bitmap) {
        const uint64_t words = (uint64_t(p[0]) | (uint64_t(p[1]) << 8) | (uint64_t(p[2]) << 16) | (uint64_t(p[3] & 0x7F) << 24));
        const uint32_t first = uint32_t(p[4]) | (uint32_t(p[5]) << 8) | (uint32_t(p[6]) << 16) | (uint32_t(p[7]) << 24);
        if (8 + 8 * words > bk.bytes) {  // a stream shorter than its block table
            if (threadIdx.x == 0) atomicOr(err, 1ull);
            return;
        }
        if (threadIdx.x == 0) put(first);
        for (uint64_t i = threadIdx.x; i < words; i += 32) {
            uint64_t w = 0;
            for (int q = 0; q < 8; ++q) w |= uint64_t(p[8 + 8 * i + q]) << (8 * q);
            while (w) {
                const uint32_t j = __ffsll((long long)w) - 1;
                w &= w - 1;
                put(uint64_t(first) + 1 + 64 * i + j);
            }
        }
        return;
    }
    if (threadIdx.x != 0) return;
    const uint32_t count = uint32_t(p[0]) | (uint32_t(p[1]) << 8) | (uint32_t(p[2]) << 16) | (uint32_t(p[3]) << 24);
    const uint32_t padded = (count + 7) / 8 * 8;
    uint64_t pos = 4;
    uint32_t cur = 0, k = 0;
    while (k < padded) {
        const uint8_t desc = p[pos++];
        for (int q = 0; q < 4; ++q, ++k) {
            const int nbytes = 1 + ((desc >> (2 * q)) & 3);
            uint32_t x = 0;
            for (int i = 0; i < nbytes; ++i) x |= uint32_t(p[pos++]) << (8 * i);
            cur += x;  // DecodeIndexesAndDiff (StreamVInt.cpp:132-145)
            if (k < count) put(cur);
        }
    }
}

// Parallel StreamVInt decode.  A block's tuples form a chain (each
// descriptor byte gives the tuple's length), so the chain is cut into chunks
// of kSviChunk tuples whose first byte offsets are found by one walk over
// the descriptors (on the host when it has the stream, else k_svi_walk);
// then one thread per chunk sums its deltas (pass 1), an exclusive scan over
// the chunks gives each chunk's first value, and one thread per chunk
// decodes again and sets the bits (pass 2).  The values are those of
// DecodeIndexesAndDiff (StreamVInt.cpp:132-145): a running sum of the
// deltas, mod 2^32, from 0 at each block.
constexpr uint32_t kSviChunk = 8;
struct SviChunk {
    uint64_t off;     // stream offset of the chunk's first descriptor
    uint32_t block;   // its block
    uint32_t tuple0;  // index of its first tuple in the block
};

__device__ __forceinline__ uint32_t svi_tuple_bytes(uint8_t d) {
    return 5u + (d & 3u) + ((d >> 2) & 3u) + ((d >> 4) & 3u) + ((d >> 6) & 3u);
}

// One thread per block: the chunk offsets of the StreamVInt blocks.
__global__ void k_svi_walk(const uint8_t* in, const psb_codec_block* blocks, uint32_t nb,
                           const unsigned long long* chunk_first, SviChunk* chunks) {
    for (uint32_t b = blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += gridDim.x * blockDim.x) {
        const psb_codec_block bk = blocks[b];
        if (bk.is_bitmap) continue;
        const uint32_t tuples = (bk.count + 7) / 8 * 2;
        const uint64_t end = bk.offset + bk.bytes;
        uint64_t pos = bk.offset + 4, c = chunk_first[b];
        for (uint32_t t = 0; t < tuples; ++t) {
            if (t % kSviChunk == 0) chunks[c++] = SviChunk{pos, b, t};
            if (pos < end) pos += svi_tuple_bytes(in[pos]);  // a short block is caught by k_svi_chunks
        }
    }
}

// Pass 1 (kFinal false): sums[c] = the sum of chunk c's deltas.  Pass 2:
// sums holds the exclusive scan over all chunks; chunk c's first value is
// sums[c] - sums[first chunk of its block].
template <bool kFinal>
__global__ void k_svi_chunks(const uint8_t* in, const psb_codec_block* blocks, const SviChunk* chunks,
                             uint64_t n_chunks, const unsigned long long* chunk_first, unsigned long long* sums,
                             uint64_t* bits, uint64_t n_bits, unsigned long long* err) {
    for (uint64_t c = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; c < n_chunks;
         c += uint64_t(gridDim.x) * blockDim.x) {
        const SviChunk ck = chunks[c];
        const psb_codec_block bk = blocks[ck.block];
        const uint32_t count = bk.count;
        const uint32_t tuples = (count + 7) / 8 * 2;
        const uint32_t t_end = ck.tuple0 + kSviChunk < tuples ? ck.tuple0 + kSviChunk : tuples;
        const uint64_t end = bk.offset + bk.bytes;
        uint32_t cur = kFinal ? uint32_t(sums[c] - sums[chunk_first[ck.block]]) : 0u;
        uint64_t pos = ck.off;
        uint32_t k = 4 * ck.tuple0;
        for (uint32_t t = ck.tuple0; t < t_end; ++t) {
            if (pos >= end || pos + svi_tuple_bytes(in[pos]) > end) {  // a stream shorter than its block table
                atomicOr(err, 1ull);
                break;
            }
            const uint8_t d = in[pos++];
            for (int q = 0; q < 4; ++q, ++k) {
                const uint32_t nbytes = 1u + ((d >> (2 * q)) & 3u);
                uint32_t x = 0;
                for (uint32_t i = 0; i < nbytes; ++i) x |= uint32_t(in[pos + i]) << (8 * i);
                pos += nbytes;
                cur += x;
                if (kFinal && k < count) {
                    if (cur >= n_bits) atomicOr(err, 1ull);
                    else atomicOr(reinterpret_cast<unsigned long long*>(bits) + (cur >> 6), 1ull << (cur & 63));
                }
            }
        }
        if (!kFinal) sums[c] = cur;
    }
}

// Device scratch of the encoder, grown on demand and kept between segments
// (a search that spills every level's frontier encodes many segments).
struct Scratch {
    unsigned long long *bsum = nullptr, *tot = nullptr, *tlen = nullptr, *gsum = nullptr;
    uint32_t* idx = nullptr;
    BlockInfo* blocks = nullptr;
    SviRef* refs = nullptr;
    size_t cap_bsum = 0, cap_tot = 0, cap_tlen = 0, cap_gsum = 0, cap_idx = 0, cap_blocks = 0, cap_refs = 0;
};

template <class T>
int grow(T** p, size_t* cap, size_t need) {
    if (need <= *cap) return PSB_OK;
    const size_t want = need + need / 4;
    CD_CUDA(cudaFree(*p));
    *p = nullptr;
    *cap = 0;
    CD_CUDA(cudaMalloc(reinterpret_cast<void**>(p), want));
    *cap = want;
    return PSB_OK;
}

}  // namespace

namespace psb {

struct SegmentEncoder {
    Scratch x;
    std::vector<BlockInfo> hb;
    std::vector<SviRef> hrefs;
    // The planned segment.
    const uint64_t* bits = nullptr;
    uint64_t n_bits = 0, n_words = 0, count = 0, tuples = 0, bytes = 0, max_words = 1;
    uint32_t nb = 0, n_refs = 0;
    bool any_bitmap = false;
    uint64_t launches = 0;  // kernels launched since the last encoder_take_launches
    // Operator bits (set_ops): every block StreamVInt with bounds, the nibble
    // of offset v being state ops_first + v of ops_nib (NULL: all zero).
    bool with_ops = false;
    const uint64_t* ops_nib = nullptr;
    uint64_t ops_first = 0;

    void set_ops(bool on, const uint64_t* nib, uint64_t first) {
        with_ops = on;
        ops_nib = nib;
        ops_first = first;
    }

    ~SegmentEncoder() {
        cudaFree(x.bsum); cudaFree(x.tot); cudaFree(x.tlen); cudaFree(x.gsum);
        cudaFree(x.idx); cudaFree(x.blocks); cudaFree(x.refs);
    }

    // First half: counts the set bits (chunk prefix sums), cuts them into
    // blocks of kBlock offsets, finds each block's first and last offset by
    // select and picks its coding; only StreamVInt blocks get an offset list
    // and tuple lengths.  Afterwards `count` = offsets, `nb` = blocks,
    // `bytes` = stream size and hb[b].out_off = block b's offset.
    // Device buffer for the chunk sums of an n-bit segment (one per kT * 16
    // words), for a producer that computes them itself (plan(.., true)).
    int chunk_sums(uint64_t n, unsigned long long** out) {
        const uint64_t nbs = ((n + 63) / 64 + kT * 16 - 1) / (kT * 16);
        if (int rc = grow(&x.bsum, &x.cap_bsum, (nbs + 1) * 8)) return rc;
        *out = x.bsum;
        return PSB_OK;
    }

    int plan(const uint64_t* b, uint64_t n, cudaStream_t s, bool sums_ready) {
        bits = b;
        n_bits = n;
        count = tuples = bytes = 0;
        nb = n_refs = 0;
        any_bitmap = false;
        max_words = 1;
        n_words = (n + 63) / 64;
        if (n == 0) return PSB_OK;
        const uint64_t nbs = (n_words + kT * 16 - 1) / (kT * 16);
        if (int rc = grow(&x.bsum, &x.cap_bsum, (nbs + 1) * 8)) return rc;
        if (int rc = grow(&x.tot, &x.cap_tot, 8)) return rc;
        if (!sums_ready) {
            k_block_sums<<<unsigned(nbs), kT, 0, s>>>(bits, n_words, n_bits, x.bsum);
            launches++;
        }
        k_scan_small<<<1, kScanT, 0, s>>>(x.bsum, nbs, x.tot);
        launches++;
        CD_CUDA(cudaGetLastError());
        unsigned long long c = 0;
        CD_CUDA(cudaMemcpyAsync(&c, x.tot, 8, cudaMemcpyDeviceToHost, s));
        CD_CUDA(cudaStreamSynchronize(s));
        count = c;
        if (count == 0) return PSB_OK;  // an empty segment writes nothing (CompressedSegmentWriter)
        nb = uint32_t((count + kBlock - 1) / kBlock);
        if (int rc = grow(&x.blocks, &x.cap_blocks, size_t(nb) * sizeof(BlockInfo))) return rc;
        k_select_blocks<<<2 * nb, kT, 0, s>>>(bits, n_words, n_bits, x.bsum, nbs, count, x.blocks, nb);
        k_block_decide<<<(nb + kT - 1) / kT, kT, 0, s>>>(count, x.blocks, nb, with_ops ? 1 : 0);
        launches += 2;
        CD_CUDA(cudaGetLastError());
        hb.resize(nb);
        CD_CUDA(cudaMemcpyAsync(hb.data(), x.blocks, size_t(nb) * sizeof(BlockInfo), cudaMemcpyDeviceToHost, s));
        CD_CUDA(cudaStreamSynchronize(s));
        // StreamVInt blocks in order: 2 tuples per 8 values (count padded to a multiple of 8).
        hrefs.clear();
        for (uint32_t k = 0; k < nb; k++) {
            if (hb[k].is_bitmap) {
                any_bitmap = true;
                max_words = std::max<uint64_t>(max_words, (uint64_t(hb[k].last) - hb[k].first + 63) / 64);
                continue;
            }
            hrefs.push_back(SviRef{tuples, k, 0});
            tuples += (uint64_t(hb[k].count) + 7) / 8 * 2;
        }
        n_refs = uint32_t(hrefs.size());
        if (tuples) {
            if (int rc = grow(&x.refs, &x.cap_refs, size_t(n_refs) * sizeof(SviRef))) return rc;
            CD_CUDA(cudaMemcpyAsync(x.refs, hrefs.data(), size_t(n_refs) * sizeof(SviRef), cudaMemcpyHostToDevice, s));
            if (int rc = grow(&x.idx, &x.cap_idx, count * 4)) return rc;
            k_compact<<<unsigned(nbs), kT, 0, s>>>(bits, n_words, n_bits, x.bsum, nbs, count, x.blocks, x.idx);
            if (int rc = grow(&x.tlen, &x.cap_tlen, (tuples + 1) * 8)) return rc;
            k_tuple_len<<<unsigned((tuples + kT - 1) / kT), kT, 0, s>>>(x.idx, x.blocks, x.refs, n_refs, tuples,
                                                                       x.tlen);
            CD_CUDA(cudaGetLastError());
            // Tuple offsets: exclusive scan of the tuple lengths (two levels: groups of 4096).
            const uint64_t groups = (tuples + kT * 16 - 1) / (kT * 16);
            if (int rc = grow(&x.gsum, &x.cap_gsum, (groups + 1) * 8)) return rc;
            k_group_sums<<<unsigned(groups), kT, 0, s>>>(x.tlen, tuples, x.gsum);
            k_scan_small<<<1, kScanT, 0, s>>>(x.gsum, groups, x.tot);
            k_group_scan<<<unsigned(groups), kT, 0, s>>>(x.tlen, tuples, x.gsum);
            unsigned long long svi_total = 0;
            CD_CUDA(cudaMemcpyAsync(&svi_total, x.tot, 8, cudaMemcpyDeviceToHost, s));
            CD_CUDA(cudaStreamSynchronize(s));
            k_block_bytes<<<(n_refs + kT - 1) / kT, kT, 0, s>>>(x.blocks, x.refs, n_refs, x.tlen, tuples, svi_total,
                                                              with_ops ? 1 : 0);
            launches += 6;
            CD_CUDA(cudaGetLastError());
            CD_CUDA(cudaMemcpyAsync(hb.data(), x.blocks, size_t(nb) * sizeof(BlockInfo), cudaMemcpyDeviceToHost, s));
            CD_CUDA(cudaStreamSynchronize(s));
        }
        unsigned long long off = 0;
        for (uint32_t k = 0; k < nb; k++) {
            hb[k].out_off = off;
            off += hb[k].bytes;
        }
        bytes = off;
        return PSB_OK;
    }

    // Second half: writes the planned stream (`bytes` bytes) to d_out.
    int write(uint8_t* d_out, cudaStream_t s) {
        if (count == 0) return PSB_OK;
        CD_CUDA(cudaMemcpyAsync(x.blocks, hb.data(), size_t(nb) * sizeof(BlockInfo), cudaMemcpyHostToDevice, s));
        if (tuples) {
            k_write_svi<<<unsigned((tuples + kT - 1) / kT), kT, 0, s>>>(x.idx, x.blocks, x.refs, n_refs, tuples, x.tlen,
                                                                       d_out);
            launches++;
            if (with_ops) {
                const uint64_t groups = tuples / 2;
                k_write_bounds<<<unsigned((groups + kT - 1) / kT), kT, 0, s>>>(x.idx, x.blocks, x.refs, n_refs, groups,
                                                                              ops_nib, ops_first, d_out);
                launches++;
            }
        }
        if (any_bitmap) {
            k_write_bitmap<<<dim3(unsigned((max_words + kT - 1) / kT), nb), kT, 0, s>>>(
                bits, n_words, n_bits, x.blocks, x.bsum, (n_words + kT * 16 - 1) / (kT * 16), count, d_out);
            launches++;
        }
        CD_CUDA(cudaGetLastError());
        return PSB_OK;
    }
};

// Bit t of the result = bit 2t of x (t < 32): the even bits, packed.
__device__ __forceinline__ uint64_t even_bits(uint64_t x) {
    x &= 0x5555555555555555ull;
    x = (x | (x >> 1)) & 0x3333333333333333ull;
    x = (x | (x >> 2)) & 0x0F0F0F0F0F0F0F0Full;
    x = (x | (x >> 4)) & 0x00FF00FF00FF00FFull;
    x = (x | (x >> 8)) & 0x0000FFFF0000FFFFull;
    return (x | (x >> 16)) & 0x00000000FFFFFFFFull;
}

// Bit t of the result = bit 4t of x (t < 16).
__device__ __forceinline__ uint64_t every_fourth_bit(uint64_t x) {
    x &= 0x1111111111111111ull;
    x = (x | (x >> 3)) & 0x0303030303030303ull;
    x = (x | (x >> 6)) & 0x000F000F000F000Full;
    x = (x | (x >> 12)) & 0x000000FF000000FFull;
    return (x | (x >> 24)) & 0x000000000000FFFFull;
}

// Frontier bitmap of a two-bit array segment: states whose code is `code`
// (InMemoryTwoBitBFS.cpp:6-20 layout: bit 2i = code / 2, bit 2i+1 = code % 2).
// Out word j covers states first + 64 j .. + 63, i.e. code words
// 2 (first/64 + j) + {0, 1}.  One CTA per chunk of kT * 16 out words, whose
// popcount goes to sums[chunk] (the encoder's chunk sums); codes past the
// last state are 0 and never match.
// With active-window flags (one byte per 2^wb states, a superset of the
// windows holding the depth's states), a chunk none of whose windows is
// flagged is empty: it counts 0 and its words are left unwritten.
__device__ __forceinline__ bool chunk_flagged(const uint8_t* flags, int wb, uint64_t n_windows, uint64_t first,
                                              uint64_t n_out, uint64_t base) {
    if (!flags) return true;
    const uint64_t s0 = first + base * 64;
    const uint64_t end_out = base + kT * 16 < n_out ? base + kT * 16 : n_out;
    const uint64_t s1 = first + end_out * 64 - 1;
    const uint64_t w0 = s0 >> wb, w1 = (s1 >> wb) < n_windows ? (s1 >> wb) : n_windows - 1;
    int any = 0;
    for (uint64_t w = w0 + threadIdx.x; w <= w1; w += kT) any |= flags[w];
    return __syncthreads_or(any) != 0;
}

__global__ void __launch_bounds__(kT) k_frontier_two_bit(const uint64_t* __restrict__ codes, uint64_t first,
                                                          uint64_t n_out, uint32_t code, uint64_t* __restrict__ out,
                                                          unsigned long long* __restrict__ sums,
                                                          const uint8_t* __restrict__ flags, int wb,
                                                          uint64_t n_windows) {
    const uint64_t hi_sel = (code & 2) ? 0 : ~uint64_t(0), lo_sel = (code & 1) ? 0 : ~uint64_t(0);
    const uint64_t base = uint64_t(blockIdx.x) * kT * 16;
    if (!chunk_flagged(flags, wb, n_windows, first, n_out, base)) {
        if (threadIdx.x == 0) sums[blockIdx.x] = 0;
        return;
    }
    uint32_t c = 0;
#pragma unroll 4
    for (int k = 0; k < 16; ++k) {
        const uint64_t j = base + uint64_t(k) * kT + threadIdx.x;
        if (j < n_out) {
            const uint64_t w = 2 * (first / 64 + j);
            const uint64_t a = codes[w], b = codes[w + 1];
            const uint64_t ma = (a ^ hi_sel) & ((a >> 1) ^ lo_sel);
            const uint64_t mb = (b ^ hi_sel) & ((b >> 1) ^ lo_sel);
            const uint64_t v = even_bits(ma) | (even_bits(mb) << 32);
            out[j] = v;
            c += __popcll(v);
        }
    }
    chunk_total(c, sums + blockIdx.x);
}

// Frontier bitmap of a frontier-search segment: states whose four operator
// bits are not all zero (InMemoryFrontierSearch.cpp:57-112), less the states
// of `excl` (the previous level's, on puzzles with odd cycles; may be NULL).
// Same CTA layout and chunk sums as k_frontier_two_bit.
__global__ void __launch_bounds__(kT) k_frontier_nibbles(const uint64_t* __restrict__ nib,
                                                          const uint64_t* __restrict__ excl, uint64_t first,
                                                          uint64_t n_out, uint64_t* __restrict__ out,
                                                          unsigned long long* __restrict__ sums) {
    const uint64_t base = uint64_t(blockIdx.x) * kT * 16;
    uint32_t c = 0;
    for (int k = 0; k < 16; ++k) {
        const uint64_t j = base + uint64_t(k) * kT + threadIdx.x;
        if (j < n_out) {
            const uint64_t w = 4 * (first / 64 + j);
            uint64_t v = 0;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const uint64_t x = nib[w + q];
                v |= every_fourth_bit(x | (x >> 1) | (x >> 2) | (x >> 3)) << (16 * q);
            }
            if (excl) v &= ~excl[first / 64 + j];
            out[j] = v;
            c += __popcll(v);
        }
    }
    chunk_total(c, sums + blockIdx.x);
}

unsigned chunks_of(uint64_t n_out) { return unsigned((n_out + kT * 16 - 1) / (kT * 16)); }

int frontier_bits_two_bit(const uint64_t* codes, uint64_t first_state, uint64_t n_states, uint32_t code,
                          uint64_t* out, unsigned long long* sums, const uint8_t* flags, int window_bits,
                          uint64_t n_windows, cudaStream_t s) {
    const uint64_t n_out = (n_states + 63) / 64;
    k_frontier_two_bit<<<chunks_of(n_out), kT, 0, s>>>(codes, first_state, n_out, code, out, sums, flags,
                                                        window_bits, n_windows);
    CD_CUDA(cudaGetLastError());
    return PSB_OK;
}

int frontier_bits_nibbles(const uint64_t* nibbles, const uint64_t* excl, uint64_t first_state, uint64_t n_states,
                          uint64_t* out, unsigned long long* sums, cudaStream_t s) {
    const uint64_t n_out = (n_states + 63) / 64;
    k_frontier_nibbles<<<chunks_of(n_out), kT, 0, s>>>(nibbles, excl, first_state, n_out, out, sums);
    CD_CUDA(cudaGetLastError());
    return PSB_OK;
}

// OpBitsCompression<BITS> (Common/OpBitsCompression.cpp:10-76): each group of
// 8 op-bit bytes (a little-endian u64 `all`) packs into BITS bytes,
//   BITS 2: u16 (all | all >> 14 | all >> 28 | all >> 42)
//   BITS 4: u32 (all | all >> 28)   (also StreamVInt's bounds, StreamVInt.cpp:139-147)
//   BITS 8: unchanged.
// One thread per group: one 8-byte load, one BITS-byte store.
template <int BITS>
__global__ void k_opbits_encode(const uint64_t* __restrict__ in, uint64_t groups, uint8_t* __restrict__ out) {
    for (uint64_t g = blockIdx.x * uint64_t(kT) + threadIdx.x; g < groups; g += uint64_t(gridDim.x) * kT) {
        const uint64_t all = in[g];
        if constexpr (BITS == 2) reinterpret_cast<uint16_t*>(out)[g] = uint16_t(all | (all >> 14) | (all >> 28) | (all >> 42));
        else if constexpr (BITS == 4) reinterpret_cast<uint32_t*>(out)[g] = uint32_t(all | (all >> 28));
        else reinterpret_cast<uint64_t*>(out)[g] = all;
    }
}
template <int BITS>
__global__ void k_opbits_decode(const uint8_t* __restrict__ in, uint64_t groups, uint64_t* __restrict__ out) {
    for (uint64_t g = blockIdx.x * uint64_t(kT) + threadIdx.x; g < groups; g += uint64_t(gridDim.x) * kT) {
        uint64_t all;
        if constexpr (BITS == 2) {
            const uint64_t st = reinterpret_cast<const uint16_t*>(in)[g];
            all = (st & 0x0303ull) | ((st & 0x0C0Cull) << 14) | ((st & 0x3030ull) << 28) | ((st & 0xC0C0ull) << 42);
        } else if constexpr (BITS == 4) {
            const uint64_t st = reinterpret_cast<const uint32_t*>(in)[g];
            all = (st & 0x0F0F0F0Full) | ((st & 0xF0F0F0F0ull) << 28);
        } else {
            all = reinterpret_cast<const uint64_t*>(in)[g];
        }
        out[g] = all;
    }
}

SegmentEncoder* encoder_create() { return new (std::nothrow) SegmentEncoder(); }
void encoder_destroy(SegmentEncoder* e) { delete e; }

int encoder_chunk_sums(SegmentEncoder* e, uint64_t n_bits, unsigned long long** sums) {
    return e->chunk_sums(n_bits, sums);
}

int encoder_plan(SegmentEncoder* e, const uint64_t* d_bits, uint64_t n_bits, cudaStream_t s, bool sums_ready,
                 uint64_t* bytes, uint64_t* count) {
    if (int rc = e->plan(d_bits, n_bits, s, sums_ready)) return rc;
    *bytes = e->bytes;
    *count = e->count;
    return PSB_OK;
}

int encoder_write(SegmentEncoder* e, uint8_t* d_out, cudaStream_t s) { return e->write(d_out, s); }

void encoder_set_ops(SegmentEncoder* e, bool on, const uint64_t* nibbles, uint64_t first_state) {
    e->set_ops(on, nibbles, first_state);
}

uint64_t encoder_take_launches(SegmentEncoder* e) {
    const uint64_t n = e->launches;
    e->launches = 0;
    return n;
}

}  // namespace psb

extern "C" int psb_frontier_encode(const uint64_t* d_bits, uint64_t first_bit, uint64_t n_bits, uint8_t* d_out,
                                   uint64_t out_cap, uint64_t* out_bytes, psb_codec_block* blocks,
                                   uint32_t blocks_cap, uint32_t* n_blocks, void* stream) {
    if (!d_bits || !out_bytes || !n_blocks) return psb_set_error(PSB_ERR_ARG, "bad argument");
    if (first_bit & 63) return psb_set_error(PSB_ERR_ARG, "first_bit must be a multiple of 64");
    if (n_bits > (uint64_t(1) << 32)) return psb_set_error(PSB_ERR_ARG, "a segment holds at most 2^32 states");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    *out_bytes = 0;
    *n_blocks = 0;
    psb::SegmentEncoder E;
    if (int rc = E.plan(d_bits + first_bit / 64, n_bits, s, false)) return rc;
    *out_bytes = E.bytes;
    *n_blocks = E.nb;
    if (E.count == 0) return PSB_OK;
    if (blocks) {
        if (blocks_cap < E.nb) return psb_set_error(PSB_ERR_CAPACITY, "blocks table too small");
        for (uint32_t b = 0; b < E.nb; b++)
            blocks[b] = psb_codec_block{E.hb[b].out_off, E.hb[b].count, uint32_t(E.hb[b].bytes), E.hb[b].first,
                                        E.hb[b].is_bitmap};
    }
    if (!d_out || out_cap < E.bytes) return psb_set_error(PSB_ERR_CAPACITY, "output needs more bytes (see *out_bytes)");
    if (int rc = E.write(d_out, s)) return rc;
    CD_CUDA(cudaStreamSynchronize(s));
    return PSB_OK;
}

extern "C" int psb_frontier_index(const uint8_t* in, uint64_t in_bytes, psb_codec_block* blocks, uint32_t cap,
                                  uint32_t* n) {
    if (!n || (!in && in_bytes)) return psb_set_error(PSB_ERR_ARG, "bad argument");
    uint64_t pos = 0;
    uint32_t k = 0;
    auto u32 = [&](uint64_t at) {
        return uint32_t(in[at]) | (uint32_t(in[at + 1]) << 8) | (uint32_t(in[at + 2]) << 16) | (uint32_t(in[at + 3]) << 24);
    };
    while (pos < in_bytes) {
        if (pos + 4 > in_bytes) return psb_set_error(PSB_ERR_ARG, "truncated block header");
        const uint32_t h = u32(pos);
        psb_codec_block b{};
        b.offset = pos;
        if (h & kMap) {
            if (pos + 8 > in_bytes) return psb_set_error(PSB_ERR_ARG, "truncated bitmap header");
            const uint64_t words = h & ~kMap;
            b.is_bitmap = 1;
            b.first = u32(pos + 4);
            const uint64_t size = 8 + words * 8;
            if (pos + size > in_bytes) return psb_set_error(PSB_ERR_ARG, "truncated bitmap block");
            uint32_t c = 1;
            for (uint64_t i = 0; i < words * 8; i++) c += __builtin_popcount(in[pos + 8 + i]);
            b.count = c;
            b.bytes = uint32_t(size);
        } else {
            b.count = h;
            const uint64_t tuples = (uint64_t(h) + 7) / 8 * 2;
            uint64_t q = pos + 4;
            for (uint64_t t = 0; t < tuples; t++) {
                if (q >= in_bytes) return psb_set_error(PSB_ERR_ARG, "truncated StreamVInt block");
                const uint8_t d = in[q];
                q += 1 + 4 + (d & 3) + ((d >> 2) & 3) + ((d >> 4) & 3) + ((d >> 6) & 3);
            }
            if (q > in_bytes) return psb_set_error(PSB_ERR_ARG, "truncated StreamVInt block");
            if (h) {  // first value: the first delta of the first tuple
                const uint8_t d = in[pos + 4];
                uint32_t v = 0;
                for (int i = 0; i <= (d & 3); i++) v |= uint32_t(in[pos + 5 + i]) << (8 * i);
                b.first = v;
            }
            b.bytes = uint32_t(q - pos);
        }
        if (blocks) {
            if (k >= cap) return psb_set_error(PSB_ERR_CAPACITY, "blocks table too small");
            blocks[k] = b;
        }
        k++;
        pos += b.bytes;
    }
    *n = k;
    return PSB_OK;
}

namespace psb {

struct DecodeScratch {
    SviChunk* chunks = nullptr;
    unsigned long long *sums = nullptr, *first = nullptr, *gsum = nullptr, *tot = nullptr;
    size_t cap_chunks = 0, cap_sums = 0, cap_first = 0, cap_gsum = 0, cap_tot = 0;
    std::vector<SviChunk> h_chunks;
    std::vector<unsigned long long> h_first;
    ~DecodeScratch() { cudaFree(chunks); cudaFree(sums); cudaFree(first); cudaFree(gsum); cudaFree(tot); }
};
DecodeScratch* decoder_create() { return new (std::nothrow) DecodeScratch(); }
void decoder_destroy(DecodeScratch* d) { delete d; }

int frontier_decode_async(const uint8_t* d_in, const uint8_t* h_in, const psb_codec_block* h_blocks,
                          const psb_codec_block* d_blocks, uint32_t n_blocks, uint64_t* d_bits, uint64_t n_bits,
                          unsigned long long* d_err, DecodeScratch* x, cudaStream_t s) {
    if (n_blocks == 0) return PSB_OK;
    // Chunks per StreamVInt block, and where each block's chunks start.
    x->h_first.assign(size_t(n_blocks) + 1, 0);
    uint64_t n_chunks = 0;
    bool any_bitmap = false;
    for (uint32_t b = 0; b < n_blocks; ++b) {
        x->h_first[b] = n_chunks;
        if (h_blocks[b].is_bitmap) { any_bitmap = true; continue; }
        const uint64_t tuples = (uint64_t(h_blocks[b].count) + 7) / 8 * 2;
        n_chunks += (tuples + kSviChunk - 1) / kSviChunk;
    }
    x->h_first[n_blocks] = n_chunks;
    if (any_bitmap) {
        k_decode<<<n_blocks, 32, 0, s>>>(d_in, d_blocks, n_blocks, d_bits, n_bits, d_err, 1);
        CD_CUDA(cudaGetLastError());
    }
    if (n_chunks == 0) return PSB_OK;
    if (int rc = grow(&x->chunks, &x->cap_chunks, n_chunks * sizeof(SviChunk))) return rc;
    if (int rc = grow(&x->sums, &x->cap_sums, n_chunks * 8)) return rc;
    if (int rc = grow(&x->first, &x->cap_first, (size_t(n_blocks) + 1) * 8)) return rc;
    const uint64_t groups = (n_chunks + kT * 16 - 1) / (kT * 16);
    if (int rc = grow(&x->gsum, &x->cap_gsum, (groups + 1) * 8)) return rc;
    if (int rc = grow(&x->tot, &x->cap_tot, 8)) return rc;
    CD_CUDA(cudaMemcpyAsync(x->first, x->h_first.data(), (size_t(n_blocks) + 1) * 8, cudaMemcpyHostToDevice, s));
    if (h_in) {  // the host walks the descriptors
        x->h_chunks.resize(n_chunks);
        for (uint32_t b = 0; b < n_blocks; ++b) {
            if (h_blocks[b].is_bitmap) continue;
            const uint32_t tuples = (h_blocks[b].count + 7) / 8 * 2;
            uint64_t pos = h_blocks[b].offset + 4, c = x->h_first[b];
            for (uint32_t t = 0; t < tuples; ++t) {
                if (t % kSviChunk == 0) x->h_chunks[c++] = SviChunk{pos, b, t};
                const uint8_t d = h_in[pos];
                pos += 5u + (d & 3u) + ((d >> 2) & 3u) + ((d >> 4) & 3u) + ((d >> 6) & 3u);
            }
        }
        CD_CUDA(cudaMemcpyAsync(x->chunks, x->h_chunks.data(), n_chunks * sizeof(SviChunk), cudaMemcpyHostToDevice, s));
    } else {
        k_svi_walk<<<(n_blocks + 127) / 128, 128, 0, s>>>(d_in, d_blocks, n_blocks, x->first, x->chunks);
    }
    const unsigned grid = unsigned(std::min<uint64_t>((n_chunks + kT - 1) / kT, 148 * 16));
    k_svi_chunks<false><<<grid, kT, 0, s>>>(d_in, d_blocks, x->chunks, n_chunks, x->first, x->sums, d_bits, n_bits,
                                           d_err);
    k_group_sums<<<unsigned(groups), kT, 0, s>>>(x->sums, n_chunks, x->gsum);
    k_scan_small<<<1, kScanT, 0, s>>>(x->gsum, groups, x->tot);
    k_group_scan<<<unsigned(groups), kT, 0, s>>>(x->sums, n_chunks, x->gsum);
    k_svi_chunks<true><<<grid, kT, 0, s>>>(d_in, d_blocks, x->chunks, n_chunks, x->first, x->sums, d_bits, n_bits,
                                          d_err);
    CD_CUDA(cudaGetLastError());
    return PSB_OK;
}
}  // namespace psb

extern "C" int psb_frontier_decode(const uint8_t* d_in, const psb_codec_block* blocks, uint32_t n_blocks,
                                   uint64_t* d_bits, uint64_t first_bit, uint64_t n_bits, void* stream) {
    if (!d_bits || (n_blocks && (!d_in || !blocks))) return psb_set_error(PSB_ERR_ARG, "bad argument");
    if (first_bit & 63) return psb_set_error(PSB_ERR_ARG, "first_bit must be a multiple of 64");
    if (n_blocks == 0) return PSB_OK;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    psb_codec_block* d_blocks = nullptr;
    unsigned long long* d_err = nullptr;
    CD_CUDA(cudaMalloc(&d_blocks, size_t(n_blocks) * sizeof(psb_codec_block)));
    cudaError_t e = cudaMalloc(&d_err, 8);
    if (e != cudaSuccess) { cudaFree(d_blocks); CD_CUDA(e); }
    std::unique_ptr<psb::DecodeScratch> x(psb::decoder_create());
    unsigned long long err = 0;
    int rc = x ? PSB_OK : psb_set_error(PSB_ERR_NOMEM, "decoder scratch");
    e = cudaMemcpyAsync(d_blocks, blocks, size_t(n_blocks) * sizeof(psb_codec_block), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_err, 0, 8, s);
    if (e == cudaSuccess && rc == PSB_OK)
        rc = psb::frontier_decode_async(d_in, nullptr, blocks, d_blocks, n_blocks, d_bits + first_bit / 64, n_bits,
                                        d_err, x.get(), s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&err, d_err, 8, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    x.reset();
    cudaFree(d_blocks);
    cudaFree(d_err);
    CD_CUDA(e);
    if (rc) return rc;
    if (err) return psb_set_error(PSB_ERR_ARG, "a decoded offset lies outside the segment");
    return PSB_OK;
}

namespace {
int opbits_check(int bits, const void* in, uint64_t count, const void* out) {
    if (bits != 2 && bits != 4 && bits != 8) return psb_set_error(PSB_ERR_ARG, "bits must be 2, 4 or 8");
    if (count & 7) return psb_set_error(PSB_ERR_ARG, "count must be a multiple of 8");
    if (count && (!in || !out)) return psb_set_error(PSB_ERR_ARG, "bad argument");
    return PSB_OK;
}
unsigned opbits_grid(uint64_t groups) {
    return unsigned(std::min<uint64_t>((groups + kT - 1) / kT, 148ull * 16));
}
}  // namespace

extern "C" int psb_opbits_encode(int bits, const uint8_t* d_op_bits, uint64_t count, uint8_t* d_out, void* stream) {
    if (int rc = opbits_check(bits, d_op_bits, count, d_out)) return rc;
    if (reinterpret_cast<uintptr_t>(d_op_bits) % 8 || reinterpret_cast<uintptr_t>(d_out) % bits)
        return psb_set_error(PSB_ERR_ARG, "op bits must be 8-byte aligned and the output aligned to `bits` bytes");
    const uint64_t groups = count / 8;
    if (!groups) return PSB_OK;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const uint64_t* in = reinterpret_cast<const uint64_t*>(d_op_bits);
    if (bits == 2) psb::k_opbits_encode<2><<<opbits_grid(groups), kT, 0, s>>>(in, groups, d_out);
    else if (bits == 4) psb::k_opbits_encode<4><<<opbits_grid(groups), kT, 0, s>>>(in, groups, d_out);
    else psb::k_opbits_encode<8><<<opbits_grid(groups), kT, 0, s>>>(in, groups, d_out);
    CD_CUDA(cudaGetLastError());
    return PSB_OK;
}

extern "C" int psb_opbits_decode(int bits, const uint8_t* d_in, uint64_t count, uint8_t* d_op_bits, void* stream) {
    if (int rc = opbits_check(bits, d_in, count, d_op_bits)) return rc;
    if (reinterpret_cast<uintptr_t>(d_op_bits) % 8 || reinterpret_cast<uintptr_t>(d_in) % bits)
        return psb_set_error(PSB_ERR_ARG, "op bits must be 8-byte aligned and the input aligned to `bits` bytes");
    const uint64_t groups = count / 8;
    if (!groups) return PSB_OK;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    uint64_t* out = reinterpret_cast<uint64_t*>(d_op_bits);
    if (bits == 2) psb::k_opbits_decode<2><<<opbits_grid(groups), kT, 0, s>>>(d_in, groups, out);
    else if (bits == 4) psb::k_opbits_decode<4><<<opbits_grid(groups), kT, 0, s>>>(d_in, groups, out);
    else psb::k_opbits_decode<8><<<opbits_grid(groups), kT, 0, s>>>(d_in, groups, out);
    CD_CUDA(cudaGetLastError());
    return PSB_OK;
}
