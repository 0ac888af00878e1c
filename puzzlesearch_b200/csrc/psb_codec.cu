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
#include <string>
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

// Exclusive scan of n u64 values in place by one block (n is small: block sums, tuple groups).
__global__ void k_scan_small(unsigned long long* v, uint64_t n, unsigned long long* total) {
    __shared__ unsigned long long s[kT];
    unsigned long long carry = 0;
    for (uint64_t base = 0; base < n; base += kT) {
        const uint64_t i = base + threadIdx.x;
        const unsigned long long x = i < n ? v[i] : 0;
        s[threadIdx.x] = x;
        __syncthreads();
        for (int o = 1; o < kT; o <<= 1) {
            const unsigned long long y = threadIdx.x >= o ? s[threadIdx.x - o] : 0;
            __syncthreads();
            s[threadIdx.x] += y;
            __syncthreads();
        }
        if (i < n) v[i] = carry + s[threadIdx.x] - x;
        const unsigned long long blk = s[kT - 1];
        __syncthreads();
        carry += blk;
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

// Writes the ascending offsets of all set bits: offset list position = rank.
__global__ void k_compact(const uint64_t* bits, uint64_t n_words, uint64_t n_bits, const unsigned long long* bsum,
                          uint32_t* idx) {
    // Recompute the per-word exclusive rank inside the block (16 words per thread, interleaved).
    __shared__ uint32_t s[kT];
    const uint64_t base = uint64_t(blockIdx.x) * kT * 16;
    unsigned long long run = bsum[blockIdx.x];
    for (int k = 0; k < 16; ++k) {
        const uint64_t w = base + uint64_t(k) * kT + threadIdx.x;
        const uint64_t word = w < n_words ? masked_word(bits, w, n_words, n_bits) : 0;
        const uint32_t c = __popcll(word);
        s[threadIdx.x] = c;
        __syncthreads();
        for (int o = 1; o < kT; o <<= 1) {
            const uint32_t y = threadIdx.x >= o ? s[threadIdx.x - o] : 0;
            __syncthreads();
            s[threadIdx.x] += y;
            __syncthreads();
        }
        unsigned long long r = run + s[threadIdx.x] - c;
        uint64_t m = word;
        while (m) {
            const uint32_t j = __ffsll((long long)m) - 1;
            m &= m - 1;
            idx[r++] = uint32_t(w * 64 + j);
        }
        const uint32_t tot = s[kT - 1];
        __syncthreads();
        run += tot;
    }
}

__device__ __forceinline__ uint32_t vbytes(uint32_t x) { return x >> 24 ? 4 : x >> 16 ? 3 : x >> 8 ? 2 : 1; }

struct BlockInfo {
    unsigned long long out_off;  // byte offset of the block in the stream
    uint32_t count, first, last, is_bitmap;
    unsigned long long bytes;
    unsigned long long tuple0;   // first tuple (StreamVInt blocks)
};

// Value of rank position k (0-based) of block b after the in-place delta, 0 past the count.
__device__ __forceinline__ uint32_t delta_at(const uint32_t* idx, uint64_t r0, uint32_t count, uint32_t k) {
    if (k >= count) return 0;
    const uint32_t v = idx[r0 + k];
    return k == 0 ? v : v - idx[r0 + k - 1];
}

// Tuple lengths of every StreamVInt block (bitmap blocks contribute zero).
__global__ void k_tuple_len(const uint32_t* idx, const BlockInfo* blocks, uint32_t nb, uint64_t tuples,
                            unsigned long long* tlen) {
    const uint64_t t = blockIdx.x * uint64_t(kT) + threadIdx.x;
    if (t >= tuples) return;
    const uint32_t b = uint32_t(t / (kBlock / 4));
    const uint32_t k = uint32_t(t % (kBlock / 4)) * 4;
    const BlockInfo bi = blocks[b];
    const uint32_t padded = (bi.count + 7) / 8 * 8;
    if (bi.is_bitmap || k >= padded) { tlen[t] = 0; return; }
    const uint64_t r0 = uint64_t(b) * kBlock;
    uint32_t len = 1;
    for (int q = 0; q < 4; ++q) len += vbytes(delta_at(idx, r0, bi.count, k + q));
    tlen[t] = len;
}

__global__ void k_block_bytes(BlockInfo* blocks, uint32_t nb, const unsigned long long* tscan, uint64_t tuples,
                              unsigned long long total) {
    const uint32_t b = blockIdx.x * kT + threadIdx.x;
    if (b >= nb) return;
    BlockInfo& bi = blocks[b];
    if (bi.is_bitmap) return;
    const uint64_t t0 = bi.tuple0, t1 = t0 + (bi.count + 7) / 8 * 2;
    const unsigned long long end = t1 < tuples ? tscan[t1] : total;
    bi.bytes = 4 + (end - tscan[t0]);
}

__global__ void k_write_svi(const uint32_t* idx, const BlockInfo* blocks, uint64_t tuples,
                            const unsigned long long* tscan, uint8_t* out) {
    const uint64_t t = blockIdx.x * uint64_t(kT) + threadIdx.x;
    if (t >= tuples) return;
    const uint32_t b = uint32_t(t / (kBlock / 4));
    const uint32_t k = uint32_t(t % (kBlock / 4)) * 4;
    const BlockInfo bi = blocks[b];
    const uint32_t padded = (bi.count + 7) / 8 * 8;
    if (bi.is_bitmap || k >= padded) return;
    const uint64_t r0 = uint64_t(b) * kBlock;
    uint8_t* p = out + bi.out_off + 4 + (tscan[t] - tscan[bi.tuple0]);
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
__global__ void k_write_bitmap(const uint64_t* bits, uint64_t n_words, uint64_t n_bits, const BlockInfo* blocks,
                               uint8_t* out) {
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
    uint64_t v = masked_word(bits, w0, n_words, n_bits) >> sh;
    if (sh && w0 + 1 < n_words) v |= masked_word(bits, w0 + 1, n_words, n_bits) << (64 - sh);
    const uint64_t hi = start + 63;  // last state this word covers
    if (hi > bi.last) {
        const uint64_t keep = uint64_t(bi.last) - start + 1;  // 0..63
        v &= keep >= 64 ? ~uint64_t(0) : ((uint64_t(1) << keep) - 1);
    }
    for (int q = 0; q < 8; ++q) p[8 + 8 * i + q] = uint8_t(v >> (8 * q));
}

__global__ void k_block_info(const uint32_t* idx, uint64_t count, BlockInfo* blocks, uint32_t nb) {
    const uint32_t b = blockIdx.x * kT + threadIdx.x;
    if (b >= nb) return;
    const uint64_t r0 = uint64_t(b) * kBlock;
    const uint32_t n = uint32_t(count - r0 < kBlock ? count - r0 : kBlock);
    BlockInfo bi{};
    bi.count = n;
    bi.first = idx[r0];
    bi.last = idx[r0 + n - 1];
    // FrontierCompression::Encode (FrontierCompression.cpp:92-102)
    const uint64_t bm_bytes = (uint64_t(bi.last) - bi.first + 63) / 64 * 8 + 8;
    bi.is_bitmap = (n > 128 && bm_bytes * 8 < uint64_t(n) * 10 - 8) ? 1 : 0;
    bi.bytes = bi.is_bitmap ? bm_bytes : 0;
    bi.tuple0 = uint64_t(b) * (kBlock / 4);
    blocks[b] = bi;
}

// Decode: one warp per block; StreamVInt blocks are walked by lane 0 (the
// tuple chain is sequential), bitmap blocks are spread over the lanes.
__global__ void k_decode(const uint8_t* in, const psb_codec_block* blocks, uint32_t nb, uint64_t* bits,
                         uint64_t n_bits, unsigned long long* err) {
    const uint32_t b = blockIdx.x;
    if (b >= nb) return;
    const psb_codec_block bk = blocks[b];
    const uint8_t* p = in + bk.offset;
    auto put = [&](uint64_t v) {
        if (v >= n_bits) { atomicOr(err, 1ull); return; }
        atomicOr(reinterpret_cast<unsigned long long*>(bits) + (v >> 6), 1ull << (v & 63));
    };
    if (bk.is_bitmap) {
        const uint64_t words = (uint64_t(p[0]) | (uint64_t(p[1]) << 8) | (uint64_t(p[2]) << 16) | (uint64_t(p[3] & 0x7F) << 24));
        const uint32_t first = uint32_t(p[4]) | (uint32_t(p[5]) << 8) | (uint32_t(p[6]) << 16) | (uint32_t(p[7]) << 24);
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

}  // namespace

extern "C" int psb_frontier_encode(const uint64_t* d_bits, uint64_t first_bit, uint64_t n_bits, uint8_t* d_out,
                                   uint64_t out_cap, uint64_t* out_bytes, psb_codec_block* blocks,
                                   uint32_t blocks_cap, uint32_t* n_blocks, void* stream) {
    if (!d_bits || !out_bytes || !n_blocks) return psb_set_error(PSB_ERR_ARG, "bad argument");
    if (first_bit & 63) return psb_set_error(PSB_ERR_ARG, "first_bit must be a multiple of 64");
    if (n_bits > (uint64_t(1) << 32)) return psb_set_error(PSB_ERR_ARG, "a segment holds at most 2^32 states");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    *out_bytes = 0;
    *n_blocks = 0;
    if (n_bits == 0) return PSB_OK;
    const uint64_t* bits = d_bits + first_bit / 64;
    const uint64_t n_words = (n_bits + 63) / 64;
    const uint64_t nbs = (n_words + kT * 16 - 1) / (kT * 16);

    unsigned long long *d_bsum = nullptr, *d_tot = nullptr, *d_tlen = nullptr;
    uint32_t* d_idx = nullptr;
    BlockInfo* d_blocks = nullptr;
    struct Guard {
        std::vector<void*> p;
        ~Guard() { for (void* x : p) cudaFree(x); }
    } g;
    CD_CUDA(cudaMalloc(&d_bsum, (nbs + 1) * 8)); g.p.push_back(d_bsum);
    CD_CUDA(cudaMalloc(&d_tot, 8)); g.p.push_back(d_tot);
    k_block_sums<<<unsigned(nbs), kT, 0, s>>>(bits, n_words, n_bits, d_bsum);
    k_scan_small<<<1, kT, 0, s>>>(d_bsum, nbs, d_tot);
    CD_CUDA(cudaGetLastError());
    unsigned long long count = 0;
    CD_CUDA(cudaMemcpyAsync(&count, d_tot, 8, cudaMemcpyDeviceToHost, s));
    CD_CUDA(cudaStreamSynchronize(s));
    if (count == 0) return PSB_OK;  // an empty segment writes nothing (CompressedSegmentWriter)
    const uint32_t nb = uint32_t((count + kBlock - 1) / kBlock);
    CD_CUDA(cudaMalloc(&d_idx, count * 4)); g.p.push_back(d_idx);
    k_compact<<<unsigned(nbs), kT, 0, s>>>(bits, n_words, n_bits, d_bsum, d_idx);
    CD_CUDA(cudaMalloc(&d_blocks, size_t(nb) * sizeof(BlockInfo))); g.p.push_back(d_blocks);
    k_block_info<<<(nb + kT - 1) / kT, kT, 0, s>>>(d_idx, count, d_blocks, nb);
    const uint64_t tuples = uint64_t(nb) * (kBlock / 4);
    CD_CUDA(cudaMalloc(&d_tlen, (tuples + 1) * 8)); g.p.push_back(d_tlen);
    k_tuple_len<<<unsigned((tuples + kT - 1) / kT), kT, 0, s>>>(d_idx, d_blocks, nb, tuples, d_tlen);
    CD_CUDA(cudaGetLastError());
    // Tuple offsets: exclusive scan of the tuple lengths (two levels: groups of 4096).
    const uint64_t groups = (tuples + kT * 16 - 1) / (kT * 16);
    unsigned long long* d_gsum = nullptr;
    CD_CUDA(cudaMalloc(&d_gsum, (groups + 1) * 8)); g.p.push_back(d_gsum);
    k_group_sums<<<unsigned(groups), kT, 0, s>>>(d_tlen, tuples, d_gsum);
    k_scan_small<<<1, kT, 0, s>>>(d_gsum, groups, d_tot);
    k_group_scan<<<unsigned(groups), kT, 0, s>>>(d_tlen, tuples, d_gsum);
    unsigned long long svi_total = 0;
    CD_CUDA(cudaMemcpyAsync(&svi_total, d_tot, 8, cudaMemcpyDeviceToHost, s));
    CD_CUDA(cudaStreamSynchronize(s));
    k_block_bytes<<<(nb + kT - 1) / kT, kT, 0, s>>>(d_blocks, nb, d_tlen, tuples, svi_total);
    CD_CUDA(cudaGetLastError());
    std::vector<BlockInfo> hb(nb);
    CD_CUDA(cudaMemcpyAsync(hb.data(), d_blocks, size_t(nb) * sizeof(BlockInfo), cudaMemcpyDeviceToHost, s));
    CD_CUDA(cudaStreamSynchronize(s));
    unsigned long long off = 0;
    uint64_t max_words = 1;
    for (uint32_t b = 0; b < nb; b++) {
        hb[b].out_off = off;
        off += hb[b].bytes;
        if (hb[b].is_bitmap) max_words = std::max<uint64_t>(max_words, (uint64_t(hb[b].last) - hb[b].first + 63) / 64);
    }
    *out_bytes = off;
    *n_blocks = nb;
    if (blocks) {
        if (blocks_cap < nb) return psb_set_error(PSB_ERR_CAPACITY, "blocks table too small");
        for (uint32_t b = 0; b < nb; b++)
            blocks[b] = psb_codec_block{hb[b].out_off, hb[b].count, uint32_t(hb[b].bytes), hb[b].first, hb[b].is_bitmap};
    }
    if (!d_out || out_cap < off) return psb_set_error(PSB_ERR_CAPACITY, "output needs more bytes (see *out_bytes)");
    CD_CUDA(cudaMemcpyAsync(d_blocks, hb.data(), size_t(nb) * sizeof(BlockInfo), cudaMemcpyHostToDevice, s));
    k_write_svi<<<unsigned((tuples + kT - 1) / kT), kT, 0, s>>>(d_idx, d_blocks, tuples, d_tlen, d_out);
    k_write_bitmap<<<dim3(unsigned((max_words + kT - 1) / kT), nb), kT, 0, s>>>(bits, n_words, n_bits, d_blocks, d_out);
    CD_CUDA(cudaGetLastError());
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
    unsigned long long err = 0;
    e = cudaMemcpyAsync(d_blocks, blocks, size_t(n_blocks) * sizeof(psb_codec_block), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_err, 0, 8, s);
    if (e == cudaSuccess) {
        k_decode<<<n_blocks, 32, 0, s>>>(d_in, d_blocks, n_blocks, d_bits + first_bit / 64, n_bits, d_err);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(&err, d_err, 8, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    cudaFree(d_blocks);
    cudaFree(d_err);
    CD_CUDA(e);
    if (err) return psb_set_error(PSB_ERR_ARG, "a decoded offset lies outside the segment");
    return PSB_OK;
}
