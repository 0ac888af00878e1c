// psb_host.cu -- host side of the C ABI declared in include/psb200.h:
// puzzle handles, Parse/ToString, batched Expand and the in-memory search
// drivers that keep every bit array in device memory and launch one fused
// level kernel (plus a finalize pass for three-bit and classic) per BFS level.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/psb200.h"
#include "psb_internal.h"
#include "psb_kernels.cuh"

using psb::LevelArgs;
using psb::PuzzleArgs;
using psb::PuzzleKernels;


namespace psb {

// Three-bit level end (InMemoryThreeBitBFS.cpp:31-42):
//   if odd cycles: new &= ~cur;  count = popcount(new &= ~old);  optionally old = 0.
__global__ void __launch_bounds__(kThreads) finalize_three_bit(const ulonglong2* __restrict__ cur,
                                                              ulonglong2* __restrict__ nw,
                                                              ulonglong2* __restrict__ old, uint64_t n2,
                                                              int odd, int zero_old,
                                                              unsigned long long* count) {
    uint32_t c = 0;
    for (uint64_t i = blockIdx.x * uint64_t(kThreads) + threadIdx.x; i < n2; i += uint64_t(gridDim.x) * kThreads) {
        ulonglong2 n = nw[i];
        const ulonglong2 o = old[i];
        n.x &= ~o.x;
        n.y &= ~o.y;
        if (odd) {
            const ulonglong2 k = cur[i];
            n.x &= ~k.x;
            n.y &= ~k.y;
        }
        nw[i] = n;
        if (zero_old) old[i] = make_ulonglong2(0, 0);
        c += __popcll(n.x) + __popcll(n.y);
    }
    c = __reduce_add_sync(0xFFFFFFFFu, c);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(count, (unsigned long long)c);
}

// Classic level end (InMemoryClassicBFS.cpp:36-37):
//   count = popcount(newOpen &= ~closed);  closed |= newOpen.
__global__ void __launch_bounds__(kThreads) finalize_classic(ulonglong2* __restrict__ nw,
                                                            ulonglong2* __restrict__ closed, uint64_t n2,
                                                            unsigned long long* count) {
    uint32_t c = 0;
    for (uint64_t i = blockIdx.x * uint64_t(kThreads) + threadIdx.x; i < n2; i += uint64_t(gridDim.x) * kThreads) {
        ulonglong2 n = nw[i];
        ulonglong2 k = closed[i];
        n.x &= ~k.x;
        n.y &= ~k.y;
        nw[i] = n;
        k.x |= n.x;
        k.y |= n.y;
        closed[i] = k;
        c += __popcll(n.x) + __popcll(n.y);
    }
    c = __reduce_add_sync(0xFFFFFFFFu, c);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(count, (unsigned long long)c);
}

// Three-bit level end of a search that keeps a visited array for bottom-up
// levels: as finalize_three_bit, plus visited |= new.  The visited array is
// not one of the reference's arrays; old/cur/new stay bit-identical.
__global__ void __launch_bounds__(kThreads) finalize_three_bit_visited(const ulonglong2* __restrict__ cur,
                                                                      ulonglong2* __restrict__ nw,
                                                                      ulonglong2* __restrict__ old,
                                                                      ulonglong2* __restrict__ visited,
                                                                      uint64_t n2, int odd, int zero_old,
                                                                      unsigned long long* count) {
    uint32_t c = 0;
    for (uint64_t i = blockIdx.x * uint64_t(kThreads) + threadIdx.x; i < n2; i += uint64_t(gridDim.x) * kThreads) {
        ulonglong2 n = nw[i];
        const ulonglong2 o = old[i];
        n.x &= ~o.x;
        n.y &= ~o.y;
        if (odd) {
            const ulonglong2 k = cur[i];
            n.x &= ~k.x;
            n.y &= ~k.y;
        }
        nw[i] = n;
        if (zero_old) old[i] = make_ulonglong2(0, 0);
        if (n.x | n.y) {
            ulonglong2 v = visited[i];
            v.x |= n.x;
            v.y |= n.y;
            visited[i] = v;
        }
        c += __popcll(n.x) + __popcll(n.y);
    }
    c = __reduce_add_sync(0xFFFFFFFFu, c);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(count, (unsigned long long)c);
}

// Three-bit level end of a sparse level, window by window: only windows
// flagged in new_flags can hold new states, and only windows flagged in
// old_flags (NULL: none) can hold old states, which are zeroed for reuse.
// Same result as finalize_three_bit(_visited) with zero_old = 1.
__global__ void __launch_bounds__(kThreads) finalize_three_bit_flagged(
    const ulonglong2* __restrict__ cur, ulonglong2* __restrict__ nw, ulonglong2* __restrict__ old,
    ulonglong2* __restrict__ visited, uint64_t n2, const uint8_t* __restrict__ new_flags,
    const uint8_t* __restrict__ old_flags, uint64_t n_windows, uint32_t per_window, int odd,
    unsigned long long* count) {
    uint32_t c = 0;
    for (uint64_t w = blockIdx.x; w < n_windows; w += gridDim.x) {
        const bool fn = new_flags[w] != 0;
        const bool fo = old_flags && old_flags[w] != 0;
        if (!fn && !fo) continue;
        const uint64_t i0 = w * per_window, i1 = i0 + per_window < n2 ? i0 + per_window : n2;
        for (uint64_t i = i0 + threadIdx.x; i < i1; i += kThreads) {
            if (fn) {
                ulonglong2 n = nw[i];
                const ulonglong2 o = old[i];
                n.x &= ~o.x;
                n.y &= ~o.y;
                if (odd) {
                    const ulonglong2 k = cur[i];
                    n.x &= ~k.x;
                    n.y &= ~k.y;
                }
                nw[i] = n;
                if (visited && (n.x | n.y)) {
                    ulonglong2 v = visited[i];
                    v.x |= n.x;
                    v.y |= n.y;
                    visited[i] = v;
                }
                c += __popcll(n.x) + __popcll(n.y);
            }
            if (fo) old[i] = make_ulonglong2(0, 0);
        }
    }
    c = __reduce_add_sync(0xFFFFFFFFu, c);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(count, (unsigned long long)c);
}

// Classic level end after a bottom-up level: as finalize_classic, plus the
// clearing of `open` that the top-down sweep does (BitArray::ScanBitsAndClear).
__global__ void __launch_bounds__(kThreads) finalize_classic_clear(ulonglong2* __restrict__ nw,
                                                                  ulonglong2* __restrict__ closed,
                                                                  ulonglong2* __restrict__ open, uint64_t n2,
                                                                  unsigned long long* count) {
    uint32_t c = 0;
    for (uint64_t i = blockIdx.x * uint64_t(kThreads) + threadIdx.x; i < n2; i += uint64_t(gridDim.x) * kThreads) {
        ulonglong2 n = nw[i];
        ulonglong2 k = closed[i];
        n.x &= ~k.x;
        n.y &= ~k.y;
        nw[i] = n;
        k.x |= n.x;
        k.y |= n.y;
        closed[i] = k;
        open[i] = make_ulonglong2(0, 0);
        c += __popcll(n.x) + __popcll(n.y);
    }
    c = __reduce_add_sync(0xFFFFFFFFu, c);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(count, (unsigned long long)c);
}

// Two-bit level end after a bottom-up level: every CUR code becomes OLD
// (the CUR -> OLD step of InMemoryTwoBitBFS.cpp:52-56, which the top-down
// sweep does in place), and the CUR states are counted (the depth's count).
__global__ void __launch_bounds__(kThreads) retire_two_bit(ulonglong2* __restrict__ codes, uint64_t n2,
                                                          uint32_t cur_code, unsigned long long* count) {
    uint32_t c = 0;
    auto retire = [&](unsigned long long& w) {
        const uint64_t hi = w & kEven, lo = (w >> 1) & kEven;
        const uint64_t cur = hi & (cur_code == 3 ? lo : ~lo);
        w ^= cur | (cur_code == 2 ? (cur << 1) : 0);
        c += __popcll(cur);
    };
    for (uint64_t i = blockIdx.x * uint64_t(kThreads) + threadIdx.x; i < n2; i += uint64_t(gridDim.x) * kThreads) {
        ulonglong2 w = codes[i];
        retire(w.x);
        retire(w.y);
        codes[i] = w;
    }
    c = __reduce_add_sync(0xFFFFFFFFu, c);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(count, (unsigned long long)c);
}

// Two-bit level end when the level's long-range marks went to the far
// bitmap (LevelArgs::far): a state whose far bit is set becomes NEXT if its
// code is UNVISITED (the `array.Get(child) == UNVISITED` test of
// InMemoryTwoBitBFS.cpp:44-49, applied once per state after the level instead
// of once per child), the bitmap is cleared for the next level, and the
// states that become NEXT are counted into `count` (the next frontier's
// size).  Far word j (32 states) pairs with code word j.  Each thread takes
// four far words and their four code words; `next_lo` is the low bit of the
// NEXT code (NEXT = 3: both bits, NEXT = 2: the high bit only).
__device__ __forceinline__ uint32_t fold_word(unsigned long long& w, uint32_t f, uint32_t next_lo) {
    if (!f) return 0;
    const uint64_t unvisited = ~(w | (w >> 1)) & kEven;
    const uint64_t m = spread_even(f) & unvisited;
    w |= m | (next_lo ? (m << 1) : 0);
    return uint32_t(__popcll(m));
}
__device__ __forceinline__ uint32_t fold_quad(ulonglong2* __restrict__ codes, uint4* __restrict__ far, uint64_t i,
                                              uint32_t next_lo) {
    const uint4 f = far[i];
    if (!(f.x | f.y | f.z | f.w)) return 0;
    ulonglong2 c0 = codes[2 * i], c1 = codes[2 * i + 1];
    uint32_t c = fold_word(c0.x, f.x, next_lo) + fold_word(c0.y, f.y, next_lo) + fold_word(c1.x, f.z, next_lo) +
                 fold_word(c1.y, f.w, next_lo);
    codes[2 * i] = c0;
    codes[2 * i + 1] = c1;
    far[i] = make_uint4(0, 0, 0, 0);
    return c;
}
__global__ void __launch_bounds__(kThreads) fold_two_bit(ulonglong2* __restrict__ codes, uint4* __restrict__ far,
                                                        uint64_t n4, uint32_t next_lo,
                                                        const unsigned long long* far_marks,
                                                        unsigned long long* count) {
    if (*far_marks == 0) return;  // the level made no far mark: the bitmap is clear
    uint32_t c = 0;
    for (uint64_t i = blockIdx.x * uint64_t(kThreads) + threadIdx.x; i < n4; i += uint64_t(gridDim.x) * kThreads)
        c += fold_quad(codes, far, i, next_lo);
    c = __reduce_add_sync(0xFFFFFFFFu, c);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(count, (unsigned long long)c);
}
// The same over the windows flagged this level only (a sparse level flags
// every window it marks, far marks included); `quads` far quads per window.
__global__ void __launch_bounds__(kThreads) fold_two_bit_flagged(ulonglong2* __restrict__ codes,
                                                                uint4* __restrict__ far, uint64_t n4,
                                                                const uint8_t* __restrict__ flags,
                                                                uint64_t n_windows, uint32_t quads,
                                                                uint32_t next_lo,
                                                                const unsigned long long* far_marks,
                                                                unsigned long long* count) {
    if (*far_marks == 0) return;
    uint32_t c = 0;
    for (uint64_t w = blockIdx.x; w < n_windows; w += gridDim.x) {
        if (!flags[w]) continue;
        for (uint32_t j = threadIdx.x; j < quads; j += kThreads) {
            const uint64_t i = w * quads + j;
            if (i < n4) c += fold_quad(codes, far, i, next_lo);
        }
    }
    c = __reduce_add_sync(0xFFFFFFFFu, c);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(count, (unsigned long long)c);
}

}  // namespace psb

namespace {

thread_local std::string g_error;

int fail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_error = buf;
    return code;
}

#define PSB_CUDA(call)                                                                              \
    do {                                                                                            \
        cudaError_t e_ = (call);                                                                    \
        if (e_ != cudaSuccess)                                                                      \
            return fail(e_ == cudaErrorMemoryAllocation ? PSB_ERR_NOMEM : PSB_ERR_CUDA, "%s: %s (%s:%d)", \
                        #call, cudaGetErrorString(e_), __FILE__, __LINE__);                        \
    } while (0)

uint64_t factorial(int n) {
    uint64_t r = 1;
    for (int i = 2; i <= n; i++) r *= uint64_t(i);
    return r;
}

// Permutation index of the reference (Puzzles/PermutationMap.cpp:39-58), host side.
uint64_t rank_host(const int* v, int n) {
    uint64_t index = 0;
    unsigned seen = 0;
    for (int i = 0; i < n; i++) {
        const int digit = v[i] - __builtin_popcount(seen & ((1u << v[i]) - 1u));
        seen |= 1u << v[i];
        index = index * uint64_t(n - i) + uint64_t(digit);
    }
    return index;
}

void unrank_host(uint64_t index, int* v, int n) {
    int d[16];
    for (int i = n - 1; i >= 0; i--) {
        d[i] = int(index % uint64_t(n - i));
        index /= uint64_t(n - i);
    }
    unsigned used = 0;
    for (int i = 0; i < n; i++) {
        int k = d[i], val = 0;
        for (;; val++) {
            if (used & (1u << val)) continue;
            if (k-- == 0) break;
        }
        v[i] = val;
        used |= 1u << val;
    }
}

// PancakeOptimized's index from the permutation rank and back (n >= 12;
// Puzzles/PancakeOptimized.cpp:26-77).
constexpr uint64_t kF12 = 479001600ull;
uint64_t opt_from_rank(uint64_t r) { return ((r / kF12) << 29) | (r % kF12); }
bool opt_to_rank(uint64_t i, uint64_t* r) {
    const uint64_t lo = i & ((uint64_t(1) << 29) - 1);
    if (lo >= kF12) return false;
    *r = (i >> 29) * kF12 + lo;
    return true;
}

// SlidingTilePuzzleOptimized's index (Puzzles/SlidingTilePuzzleOptimized.cpp:
// 12-26 sizes, 79-97 parity, 99-158 Pack / GetIndex, 160-187 FromIndex,
// 118-140 Unpack), host side: `tiles` are the board's tiles in board order,
// the blank left out, tile t held as t-1.
uint64_t sopt_indexes(int cells) {
    if (cells >= 14) return uint64_t(cells == 14 ? 0xC + 1 : cells == 15 ? 0xDC + 1 : 0xEDC + 1) << 32;
    uint64_t m = 16;
    for (int i = 3; i < cells; i++) m *= uint64_t(i);
    return m;
}
bool sopt_parity_ok(int width, const int* tiles, int ntiles, int blank) {
    int inv = 0;
    for (int i = 0; i < ntiles; i++)
        for (int j = 0; j < i; j++) inv += tiles[j] > tiles[i];
    return ((inv + (width % 2 == 0 ? blank / width : 0)) & 1) == 0;
}
uint64_t sopt_index(const int* tiles, int ntiles, int blank) {
    uint64_t low = 0, seg = 0;
    for (int i = std::min(ntiles - 1, 11); i >= 2; i--) {
        int d = 0;
        for (int j = 0; j < i; j++) d += tiles[j] < tiles[i];
        low = low * uint64_t(i + 1) + uint64_t(d);
    }
    for (int i = 12; i < ntiles; i++) {
        int d = 0;
        for (int j = 0; j < i; j++) d += tiles[j] < tiles[i];
        seg |= uint64_t(d) << (4 * (i - 12));
    }
    return (seg << 32) | (low * 16 + uint64_t(blank));
}
bool sopt_board(int width, int cells, uint64_t index, int* tiles, int* blank) {
    const int ntiles = cells - 1;
    int d[16] = {0};
    *blank = int(index & 15);
    if (*blank >= cells) return false;
    uint64_t low = (index & 0xFFFFFFFFull) >> 4;
    for (int i = 2; i <= 11; i++) {
        d[i] = int(low % uint64_t(i + 1));
        low /= uint64_t(i + 1);
    }
    uint64_t seg = index >> 32;
    for (int i = 12; i <= 14; i++, seg >>= 4) d[i] = int(seg & 15);
    if (low || seg) return false;
    for (int i = 0; i < 16; i++)
        if (d[i] > i || (i >= ntiles && d[i])) return false;
    unsigned used = 0;  // values placed so far, last tile first: d_i picks the d_i-th unused one
    for (int i = ntiles - 1; i >= 2; i--) {
        int k = d[i], val = 0;
        for (;; val++) {
            if (used & (1u << val)) continue;
            if (k-- == 0) break;
        }
        tiles[i] = val;
        used |= 1u << val;
    }
    int lo = 0;
    while (used & (1u << lo)) lo++;
    int hi = lo + 1;
    while (used & (1u << hi)) hi++;
    tiles[0] = hi;  // d_1 = 0; the other parity class swaps the first two
    tiles[1] = lo;
    if (!sopt_parity_ok(width, tiles, ntiles, *blank)) std::swap(tiles[0], tiles[1]);
    return true;
}

bool read_ints(const char* s, std::vector<int>& out) {
    std::istringstream in(s);
    std::string tok;
    while (in >> tok) {
        char* end = nullptr;
        long v = strtol(tok.c_str(), &end, 10);
        if (!end || *end) return false;
        out.push_back(int(v));
    }
    return true;
}

int ensure_device(int device) {
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0) return fail(PSB_ERR_NO_DEVICE, "no CUDA device visible");
    if (device >= 0) {
        if (device >= count) return fail(PSB_ERR_ARG, "device %d out of range (%d visible)", device, count);
        PSB_CUDA(cudaSetDevice(device));
    }
    return PSB_OK;
}

// Scratch device buffers of psb_expand, one set per host thread.
struct ExpandPool {
    int device = -1;
    uint64_t cap = 0, out_cap = 0;
    uint64_t* d_par = nullptr;
    uint32_t* d_ops_in = nullptr;
    uint64_t* d_out = nullptr;
    uint32_t* d_ops = nullptr;
    unsigned long long* d_err = nullptr;
    cudaStream_t stream = nullptr;
    void release() {
        cudaFree(d_par); cudaFree(d_ops_in); cudaFree(d_out); cudaFree(d_ops); cudaFree(d_err);
        if (stream) cudaStreamDestroy(stream);
        *this = ExpandPool();
    }
    ~ExpandPool() { if (device >= 0) release(); }
};
thread_local ExpandPool g_pool;

constexpr uint64_t kExpandChunk = 2 * 1024 * 1024;  // Puzzle::MAX_INDEXES_BUFFER, Common/Puzzle.h:18

int pool_reserve(int branching) {
    int dev = 0;
    PSB_CUDA(cudaGetDevice(&dev));
    const uint64_t out_cap = kExpandChunk * uint64_t(branching);
    if (g_pool.device == dev && g_pool.out_cap >= out_cap) return PSB_OK;
    if (g_pool.device >= 0) g_pool.release();
    g_pool.device = dev;
    PSB_CUDA(cudaMalloc(&g_pool.d_par, kExpandChunk * 8));
    PSB_CUDA(cudaMalloc(&g_pool.d_ops_in, kExpandChunk * 4));
    PSB_CUDA(cudaMalloc(&g_pool.d_out, out_cap * 8));
    PSB_CUDA(cudaMalloc(&g_pool.d_ops, out_cap * 4));
    PSB_CUDA(cudaMalloc(&g_pool.d_err, 8));
    PSB_CUDA(cudaStreamCreateWithFlags(&g_pool.stream, cudaStreamNonBlocking));
    g_pool.cap = kExpandChunk;
    g_pool.out_cap = out_cap;
    return PSB_OK;
}

int mode_of(int algo) {
    switch (algo) {
    case PSB_THREE_BIT: return psb::kThreeBit;
    case PSB_CLASSIC: return psb::kClassic;
    case PSB_TWO_BIT: return psb::kTwoBit;
    case PSB_FRONTIER: return psb::kFrontier;
    }
    return -1;
}

uint64_t words_for(uint64_t bits) { return (bits + 63) / 64; }
uint64_t padded(uint64_t words) { return (words + 31) / 32 * 32; }  // 256-byte multiples for 128-bit sweeps

}  // namespace

int psb_set_error(int code, const char* msg) { return fail(code, "%s", msg); }

extern "C" {

const char* psb_version(void) { return "puzzlesearch_b200 1.0 (sm_100a)"; }

int psb_last_error(char* buf, int cap) {
    if (!buf || cap <= 0) return PSB_ERR_ARG;
    snprintf(buf, size_t(cap), "%s", g_error.c_str());
    return PSB_OK;
}

int psb_device_count(int* count) {
    if (!count) return PSB_ERR_ARG;
    int c = 0;
    if (cudaGetDeviceCount(&c) != cudaSuccess) c = 0;
    *count = c;
    return PSB_OK;
}

int psb_device_name(int device, char* buf, int cap) {
    if (!buf || cap <= 0) return fail(PSB_ERR_ARG, "bad argument");
    if (int rc = ensure_device(device)) return rc;
    if (device < 0) PSB_CUDA(cudaGetDevice(&device));
    cudaDeviceProp prop{};
    PSB_CUDA(cudaGetDeviceProperties(&prop, device));
    snprintf(buf, size_t(cap), "%s (sm_%d%d, %d SMs)", prop.name, prop.major, prop.minor, prop.multiProcessorCount);
    return PSB_OK;
}

int psb_puzzle_create(int kind, int a, int b, psb_puzzle** out) {
    if (!out) return fail(PSB_ERR_ARG, "out is NULL");
    auto p = std::make_unique<psb_puzzle>();
    p->kind = kind; p->a = a; p->b = b;
    p->pz = PuzzleArgs{0, 0, 0};
    bool ok = false;
    switch (kind) {
    case PSB_SLIDING:  // SlidingTilePuzzleSimple.h:13-19, .cpp:35-39
        if (a < 1 || b < 1 || a * b < 2 || a * b > 16) return fail(PSB_ERR_ARG, "sliding tile %dx%d: need 2 <= w*h <= 16", a, b);
        p->cells = a * b; p->n_states = factorial(a * b); p->ops = 4; p->branching = 4; p->odd = 0;
        p->pz.width = a;
        ok = psb::sliding_kernels(a * b, &p->k);
        break;
    case PSB_PANCAKE:  // PancakeSimple.h:13-19, .cpp:26,36-40
        if (a < 2 || a > 16) return fail(PSB_ERR_ARG, "pancake size %d: need 2..16", a);
        p->cells = a; p->n_states = factorial(a); p->ops = a - 1; p->branching = a - 1; p->odd = 1;
        ok = psb::pancake_kernels(a, &p->k);
        break;
    case PSB_PANCAKE_OPT:  // PancakeOptimized.h:14-20, .cpp:81-105
        if (a < 2 || a > 16) return fail(PSB_ERR_ARG, "pancake size %d: need 2..16", a);
        p->cells = a; p->ops = a - 1; p->branching = a - 1; p->odd = 1;
        if (a < 12) {
            p->n_states = factorial(a);
            ok = psb::pancake_kernels(a, &p->k);
        } else {
            p->n_states = uint64_t(1) << 29;
            for (int k = 13; k <= a; k++) p->n_states *= uint64_t(k);
            ok = psb::pancake_opt_kernels(a, &p->k);
        }
        break;
    case PSB_SLIDING_OPT:  // SlidingTilePuzzleOptimized.h:13-24, .cpp:205-211
        if (a < 1 || b < 1 || a * b < 4 || a * b > 16)
            return fail(PSB_ERR_ARG, "sliding tile %dx%d: need 4 <= w*h <= 16", a, b);
        p->cells = a * b; p->n_states = sopt_indexes(a * b); p->ops = 4; p->branching = 4; p->odd = 0;
        p->pz.width = a;
        ok = psb::sliding_opt_kernels(a * b, &p->k);
        break;
    case PSB_HANOI4:      // FourPegHanoiSimple.h:14-20, .cpp:141-143
    case PSB_HANOI4_OPT:  // FourPegHanoiOptimized.h:8-20, .cpp:164-166: the same index space
        if (a < 1 || a > 31) return fail(PSB_ERR_ARG, "hanoi disks %d: need 1..31", a);
        p->cells = 0; p->n_states = uint64_t(1) << (2 * a); p->ops = 4; p->branching = 6; p->odd = 1;
        p->pz.disks = a; p->pz.sym = b ? (kind == PSB_HANOI4_OPT ? 2 : 1) : 0;
        ok = psb::hanoi_kernels(&p->k);
        break;
    default:
        return fail(PSB_ERR_ARG, "unknown puzzle kind %d", kind);
    }
    if (!ok) return fail(PSB_ERR_UNSUPPORTED, "no kernels for this puzzle");
    *out = p.release();
    return PSB_OK;
}

int psb_puzzle_destroy(psb_puzzle* p) {
    delete p;
    return PSB_OK;
}

int psb_puzzle_info(const psb_puzzle* p, uint64_t* indexes, int* operators, int* branching, int* odd) {
    if (!p) return fail(PSB_ERR_ARG, "puzzle is NULL");
    if (indexes) *indexes = p->n_states;
    if (operators) *operators = p->ops;
    if (branching) *branching = p->branching;
    if (odd) *odd = p->odd;
    return PSB_OK;
}

int psb_puzzle_name(const psb_puzzle* p, char* buf, int cap) {
    if (!p || !buf || cap <= 0) return fail(PSB_ERR_ARG, "bad argument");
    std::ostringstream s;
    switch (p->kind) {
    case PSB_SLIDING: s << "Sliding-Tile simple: " << p->a << " x " << p->b; break;   // SlidingTilePuzzleSimple.cpp:27-32
    case PSB_PANCAKE: s << "Pancake simple, size: " << p->a; break;                   // PancakeSimple.cpp:29-33
    case PSB_HANOI4: s << "Four-Peg Hanoi Towers, size=" << p->a << "; symmetry=" << (p->b ? 1 : 0); break;  // FourPegHanoiSimple.cpp:129-135
    case PSB_HANOI4_OPT:  // FourPegHanoiOptimized.cpp:151-157
        s << "Four-Peg Hanoi Towers Optimized, size=" << p->a << "; symmetry=" << (p->b ? 1 : 0);
        break;
    case PSB_PANCAKE_OPT:  // PancakeOptimized.cpp:88-92
        s << "Pancake optimized (29 bit segment), size: " << p->a << "; invIdx: " << (p->b ? 1 : 0);
        break;
    case PSB_SLIDING_OPT:  // SlidingTilePuzzleOptimized.cpp:196-202
        s << "Sliding-Tile GPU Optimized (for 32-bit segment): " << p->a << " x " << p->b;
        break;
    }
    const std::string str = s.str();
    if (int(str.size()) + 1 > cap) return fail(PSB_ERR_CAPACITY, "name buffer too small");
    memcpy(buf, str.c_str(), str.size() + 1);
    return int(str.size());
}

int psb_parse(const psb_puzzle* p, const char* state, uint64_t* index) {
    if (!p || !state || !index) return fail(PSB_ERR_ARG, "bad argument");
    std::vector<int> v;
    if (!read_ints(state, v)) return fail(PSB_ERR_ARG, "cannot parse state '%s'", state);
    if (p->kind == PSB_SLIDING_OPT) {
        // SlidingTilePuzzleOptimized.cpp:27-77, 224-236: a permutation of 0..n-1 (0 = blank) of the
        // solvable parity class (the reference's Parse stops the program on the other one).
        if (int(v.size()) != p->cells) return fail(PSB_ERR_ARG, "state '%s' needs %d values", state, p->cells);
        unsigned seen = 0;
        int tiles[16], k = 0, blank = -1;
        for (int i = 0; i < p->cells; i++) {
            const int x = v[i];
            if (x < 0 || x >= p->cells || (seen >> x) & 1u) return fail(PSB_ERR_ARG, "state '%s' is not a permutation", state);
            seen |= 1u << x;
            if (x == 0) blank = i;
            else tiles[k++] = x - 1;
        }
        if (!sopt_parity_ok(p->a, tiles, p->cells - 1, blank))
            return fail(PSB_ERR_ARG, "state '%s' is not solvable from the standard state", state);
        *index = sopt_index(tiles, p->cells - 1, blank);
        return PSB_OK;
    }
    if (p->kind != PSB_HANOI4 && p->kind != PSB_HANOI4_OPT) {
        // SlidingTilePuzzleSimple.cpp:52-59, PancakeSimple.cpp:53-60: a permutation of 0..n-1.
        if (int(v.size()) != p->cells) return fail(PSB_ERR_ARG, "state '%s' needs %d values", state, p->cells);
        unsigned seen = 0;
        for (int x : v) {
            if (x < 0 || x >= p->cells || (seen >> x) & 1u) return fail(PSB_ERR_ARG, "state '%s' is not a permutation", state);
            seen |= 1u << x;
        }
        *index = rank_host(v.data(), p->cells);
        if (p->kind == PSB_PANCAKE_OPT && p->cells >= 12) *index = opt_from_rank(*index);
        return PSB_OK;
    }
    // FourPegHanoiSimple.cpp:85-113: disks (1-based) listed peg by peg, a 0 between pegs.
    uint64_t idx = 0;
    int peg = 0;
    for (int x : v) {
        if (x == 0) { peg++; continue; }
        if (peg > 3 || x < 1 || x > p->a) return fail(PSB_ERR_ARG, "bad Hanoi state '%s'", state);
        idx |= uint64_t(peg) << (2 * (x - 1));
    }
    *index = idx;
    return PSB_OK;
}

int psb_to_string(const psb_puzzle* p, uint64_t index, char* buf, int cap) {
    if (!p || !buf || cap <= 0) return fail(PSB_ERR_ARG, "bad argument");
    if (index >= p->n_states) return fail(PSB_ERR_ARG, "index out of range");
    std::ostringstream s;
    if (p->kind == PSB_SLIDING_OPT) {
        // ToString via ToStandardState (SlidingTilePuzzleOptimized.cpp:46-59, 213-217).
        int tiles[16], blank, k = 0;
        if (!sopt_board(p->a, p->cells, index, tiles, &blank))
            return fail(PSB_ERR_ARG, "index %llu names no board", (unsigned long long)index);
        for (int i = 0; i < p->cells; i++) s << (i ? " " : "") << (i == blank ? 0 : tiles[k++] + 1);
    } else if (p->kind != PSB_HANOI4 && p->kind != PSB_HANOI4_OPT) {
        int v[16];
        if (p->kind == PSB_PANCAKE_OPT && p->cells >= 12) {
            if (!opt_to_rank(index, &index)) return fail(PSB_ERR_ARG, "offset %llu of its 2^29 block names no permutation",
                                                          (unsigned long long)(index & ((1ull << 29) - 1)));
        }
        unrank_host(index, v, p->cells);
        for (int i = 0; i < p->cells; i++) s << (i ? " " : "") << v[i];
    } else {
        // FourPegHanoiSimple.cpp:71-83: each peg top-down (1-based), then "0 ", last " 0 " dropped.
        std::string str;
        for (int peg = 0; peg < 4; peg++) {
            for (int d = 0; d < p->a; d++)
                if (int((index >> (2 * d)) & 3) == peg) str += std::to_string(d + 1) + " ";
            str += "0 ";
        }
        s << str.substr(0, str.size() - 3);
    }
    const std::string str = s.str();
    if (int(str.size()) + 1 > cap) return fail(PSB_ERR_CAPACITY, "string buffer too small");
    memcpy(buf, str.c_str(), str.size() + 1);
    return int(str.size());
}

int psb_expand(const psb_puzzle* p, const uint64_t* parents, const uint32_t* opbits, uint64_t n, uint64_t* children,
               uint32_t* child_ops, uint64_t cap, uint64_t* n_out, uint32_t flags, void* stream) {
    if (!p || !n_out || (n && (!parents || !children || !child_ops)))
        return fail(PSB_ERR_ARG, "bad argument");
    const bool host = flags & PSB_EXPAND_HOST_POINTERS;
    const bool compact = flags & PSB_EXPAND_COMPACT;
    const bool use_ob = (flags & PSB_EXPAND_USE_OPBITS) && opbits;
    const uint64_t br = uint64_t(p->branching);
    if (compact && !host) return fail(PSB_ERR_ARG, "PSB_EXPAND_COMPACT needs host pointers");
    if (!compact && cap < n * br) return fail(PSB_ERR_CAPACITY, "need %llu output slots", (unsigned long long)(n * br));
    *n_out = 0;
    if (n == 0) return PSB_OK;
    if (int rc = ensure_device(-1)) return rc;
    if (int rc = pool_reserve(p->branching)) return rc;
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : g_pool.stream;
    PSB_CUDA(cudaMemsetAsync(g_pool.d_err, 0, 8, s));
    if (!host) {
        // Device pointers: one launch per chunk, slots written in place.
        for (uint64_t off = 0; off < n; off += kExpandChunk) {
            const uint64_t m = std::min(kExpandChunk, n - off);
            PSB_CUDA(p->k.expand(parents + off, use_ob ? opbits + off : nullptr, m, p->n_states, children + off * br,
                                 child_ops + off * br, p->pz, g_pool.d_err, use_ob, s));
        }
        unsigned long long err = 0;
        PSB_CUDA(cudaMemcpyAsync(&err, g_pool.d_err, 8, cudaMemcpyDeviceToHost, s));
        PSB_CUDA(cudaStreamSynchronize(s));
        if (err) return fail(PSB_ERR_ARG, "a parent index is >= IndexesCount()");
        *n_out = n * br;
        return PSB_OK;
    }
    for (uint64_t i = 0; i < n; i++)
        if (parents[i] >= p->n_states) return fail(PSB_ERR_ARG, "parent %llu >= IndexesCount()", (unsigned long long)parents[i]);
    std::vector<uint64_t> hbuf;
    std::vector<uint32_t> obuf;
    uint64_t written = 0;
    for (uint64_t off = 0; off < n; off += kExpandChunk) {
        const uint64_t m = std::min(kExpandChunk, n - off);
        PSB_CUDA(cudaMemcpyAsync(g_pool.d_par, parents + off, m * 8, cudaMemcpyHostToDevice, s));
        if (use_ob) PSB_CUDA(cudaMemcpyAsync(g_pool.d_ops_in, opbits + off, m * 4, cudaMemcpyHostToDevice, s));
        PSB_CUDA(p->k.expand(g_pool.d_par, g_pool.d_ops_in, m, p->n_states, g_pool.d_out, g_pool.d_ops, p->pz,
                             g_pool.d_err, use_ob, s));
        uint64_t* dst = children + off * br;
        uint32_t* dop = child_ops + off * br;
        if (compact) {
            hbuf.resize(m * br);
            obuf.resize(m * br);
            dst = hbuf.data();
            dop = obuf.data();
        }
        PSB_CUDA(cudaMemcpyAsync(dst, g_pool.d_out, m * br * 8, cudaMemcpyDeviceToHost, s));
        PSB_CUDA(cudaMemcpyAsync(dop, g_pool.d_ops, m * br * 4, cudaMemcpyDeviceToHost, s));
        PSB_CUDA(cudaStreamSynchronize(s));
        if (compact) {
            for (uint64_t j = 0; j < m * br; j++) {
                if (hbuf[j] == PSB_INVALID_INDEX) continue;  // ExpandBuffer filters these (Common/Puzzle.h:98)
                if (written >= cap) return fail(PSB_ERR_CAPACITY, "compacted output exceeds cap");
                children[written] = hbuf[j];
                child_ops[written] = obuf[j];
                written++;
            }
        } else {
            written += m * br;
        }
    }
    *n_out = written;
    return PSB_OK;
}

int psb_final_words(const psb_puzzle* p, int algo, uint64_t* words) {
    if (!p || !words) return fail(PSB_ERR_ARG, "bad argument");
    const uint64_t N = p->n_states;
    switch (algo) {
    case PSB_TWO_BIT: *words = words_for(2 * N); return PSB_OK;
    case PSB_THREE_BIT: case PSB_CLASSIC: *words = 3 * words_for(N); return PSB_OK;
    case PSB_FRONTIER: *words = 2 * ((N + 15) / 16); return PSB_OK;
    }
    return fail(PSB_ERR_ARG, "unknown algorithm %d", algo);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// In-memory search session.
// ---------------------------------------------------------------------------
namespace {

// Search arrays come from one stream-ordered memory pool per device that keeps
// freed memory reserved (release threshold: everything), so back-to-back
// psb_bfs calls reuse their arrays.  Mapping and unmapping gigabytes per
// call is what cudaMalloc/cudaFree would do, and on B200 a cudaFree of a few
// GB took from 5 to 650 ms.  psb_release_cached_memory() returns the memory.
constexpr int kMaxPoolDevices = 64;
std::mutex g_pool_mu;
cudaMemPool_t g_pools[kMaxPoolDevices] = {};

int session_pool(int device, cudaMemPool_t* out) {
    if (device < 0 || device >= kMaxPoolDevices) return fail(PSB_ERR_ARG, "device %d out of range", device);
    std::lock_guard<std::mutex> lock(g_pool_mu);
    if (!g_pools[device]) {
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = device;
        cudaMemPool_t pool = nullptr;
        PSB_CUDA(cudaMemPoolCreate(&pool, &props));
        uint64_t keep = ~uint64_t(0);
        PSB_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
        g_pools[device] = pool;
    }
    *out = g_pools[device];
    return PSB_OK;
}

// Frontier spill resources: the segment encoder (its device scratch), one
// segment's extracted bitmap, an arena holding one depth's encoded segments
// back to back, a copy stream and two pinned host slots.  A depth is encoded
// into the arena before its level runs; while the level kernel runs, the
// calling thread moves the segments through the host slots (copy on the copy
// stream, then the callback) in order.  They are kept per device between
// searches (a search allocates them on first use);
// psb_release_cached_memory frees them.
struct SpillSeg {
    uint32_t depth, segment;
    uint64_t off, bytes, states;
};

struct SpillSlot {
    uint8_t* host = nullptr;
    uint64_t host_cap = 0;
    cudaEvent_t start = nullptr, done = nullptr;
};

struct SpillRes {
    int device = -1;
    psb::SegmentEncoder* enc = nullptr;
    uint64_t* bits = nullptr;
    uint64_t bits_cap = 0;  // bytes
    uint8_t* arena = nullptr;
    uint64_t arena_cap = 0;  // bytes
    std::vector<SpillSeg> segs;  // the depth in the arena
    std::vector<uint8_t> flags;  // host copy of the depth's active-window flags
    size_t issued = 0, delivered = 0;
    SpillSlot slot[2];  // segment i goes through slot i % 2
    cudaStream_t copy = nullptr;
    cudaEvent_t encoded = nullptr;

    ~SpillRes() {
        if (copy) cudaStreamSynchronize(copy);
        for (auto& sl : slot) {
            if (sl.host) cudaFreeHost(sl.host);
            if (sl.start) cudaEventDestroy(sl.start);
            if (sl.done) cudaEventDestroy(sl.done);
        }
        cudaFree(bits);
        cudaFree(arena);
        if (enc) psb::encoder_destroy(enc);
        if (encoded) cudaEventDestroy(encoded);
        if (copy) cudaStreamDestroy(copy);
    }

    // Waits for copies in flight and drops their segments (a search that
    // failed part-way leaves them behind).
    void reset() {
        if (copy) cudaStreamSynchronize(copy);
        segs.clear();
        issued = delivered = 0;
    }
};

std::mutex g_spill_mu;
std::vector<SpillRes*> g_spill_cache[kMaxPoolDevices];

int spill_acquire(int device, SpillRes** out) {
    {
        std::lock_guard<std::mutex> lock(g_spill_mu);
        if (device >= 0 && device < kMaxPoolDevices && !g_spill_cache[device].empty()) {
            *out = g_spill_cache[device].back();
            g_spill_cache[device].pop_back();
            return PSB_OK;
        }
    }
    std::unique_ptr<SpillRes> R(new (std::nothrow) SpillRes());
    if (!R || !(R->enc = psb::encoder_create())) return fail(PSB_ERR_NOMEM, "spill resources");
    R->device = device;
    PSB_CUDA(cudaStreamCreateWithFlags(&R->copy, cudaStreamNonBlocking));
    PSB_CUDA(cudaEventCreateWithFlags(&R->encoded, cudaEventDisableTiming));
    for (auto& sl : R->slot) {
        PSB_CUDA(cudaEventCreate(&sl.start));
        PSB_CUDA(cudaEventCreate(&sl.done));
    }
    *out = R.release();
    return PSB_OK;
}

void spill_return(SpillRes* R) {
    R->reset();
    std::lock_guard<std::mutex> lock(g_spill_mu);
    if (R->device >= 0 && R->device < kMaxPoolDevices) g_spill_cache[R->device].push_back(R);
    else delete R;
}

}  // namespace

struct psb_bfs_session {
    psb_puzzle p;
    int algo = 0, mode = 0, device = -1, window_bits = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    uint64_t* arr[4] = {nullptr, nullptr, nullptr, nullptr};
    uint64_t words[4] = {0, 0, 0, 0};  // padded sizes
    int n_arr = 0;
    uint64_t* visited = nullptr;  // three-bit searches that may run bottom-up: states at depth <= current
    uint32_t* far = nullptr;      // two-bit: long-range mark bitmap (1 bit per state), folded after each level
    uint64_t far_words = 0;       // its size in 64-bit words (padded)
    bool bottom_up = false;       // this search's algorithm and puzzle support bottom-up levels
    unsigned long long* d_stats = nullptr;
    unsigned long long* h_stats = nullptr;
    uint8_t* wflags[3] = {nullptr, nullptr, nullptr};  // active-window flags (1 byte per window), three levels
    uint64_t n_windows = 0;
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    uint64_t bytes = 0;
    cudaMemPool_t pool = nullptr;
    SpillRes* spill = nullptr;  // frontier spill resources, taken from the device's cache on first use

    int alloc(void** ptr, size_t size) {  // stream-ordered, from the device's session pool
        PSB_CUDA(cudaMallocFromPoolAsync(ptr, size, pool, stream));
        bytes += size;
        return PSB_OK;
    }

    ~psb_bfs_session() {
        for (auto* a : arr) if (a) cudaFreeAsync(a, stream);
        if (visited) cudaFreeAsync(visited, stream);
        if (far) cudaFreeAsync(far, stream);
        if (d_stats) cudaFreeAsync(d_stats, stream);
        for (auto* f : wflags) if (f) cudaFreeAsync(f, stream);
        if (spill) spill_return(spill);
        if (h_stats) cudaFreeHost(h_stats);
        for (auto& e : ev) if (e) cudaEventDestroy(e);
        if (own_stream && stream) cudaStreamDestroy(stream);
    }
};

namespace {

int layout(const psb_puzzle* p, int algo, uint64_t* words, int* n_arr) {
    const uint64_t N = p->n_states;
    switch (algo) {
    case PSB_THREE_BIT: case PSB_CLASSIC:
        *n_arr = 3;
        words[0] = words[1] = words[2] = padded(words_for(N));
        return PSB_OK;
    case PSB_TWO_BIT:
        *n_arr = 1;
        words[0] = padded(words_for(2 * N));
        return PSB_OK;
    case PSB_FRONTIER:
        if (p->ops > 4) return fail(PSB_ERR_UNSUPPORTED, "frontier search keeps 4 operator bits per state; this puzzle has %d operators", p->ops);
        *n_arr = p->odd ? 4 : 2;
        words[0] = words[1] = padded((N + 15) / 16);
        if (p->odd) words[2] = words[3] = padded(words_for(N));
        return PSB_OK;
    }
    return fail(PSB_ERR_ARG, "unknown algorithm %d", algo);
}

// Bottom-up levels need "v has a frontier neighbour" to equal "v is a child
// of a frontier state" on the states they scan.  That holds for the pancake,
// sliding-tile and plain Hanoi moves, which are undone by a move of the same
// puzzle, and it fails for Hanoi with symmetry, whose index space also holds
// non-canonical states that expand to canonical children.  Frontier search
// keeps no visited information.
// Default switch ratio of PSB_DIR_AUTO (unvisited < ratio x frontier).
constexpr double kBottomUpRatio = 1.0;

// PSB_FAR_AUTO's pick (measured on B200, two-bit, full searches):
//   13-pancake: ALL 241 ms, NEAR 254 ms, NONE 265 ms;
//   14-pancake: NEAR 4.18 s, NONE 4.45 s, ALL 4.73 s (its flips of 13 and 14
//   land anywhere in a 10.9 GB bitmap; read-first keeps them read-only);
//   18-disk Hanoi: NONE 1.58 s, ALL 1.84 s (0.3% of its marks are long-range).
int far_mode(const psb_puzzle* p, int algo, int requested) {
    if (algo != PSB_TWO_BIT) return PSB_FAR_NONE;
    if (requested >= PSB_FAR_NONE && requested <= PSB_FAR_ALL) return requested;
    if (p->kind == PSB_HANOI4 || p->kind == PSB_HANOI4_OPT) return PSB_FAR_NONE;
    return PSB_FAR_NEAR;
}

bool supports_bottom_up(const psb_puzzle* p, int algo) {
    if (algo != PSB_THREE_BIT && algo != PSB_TWO_BIT && algo != PSB_CLASSIC) return false;
    return !((p->kind == PSB_HANOI4 || p->kind == PSB_HANOI4_OPT) && p->pz.sym);
}

// Window of 2^16 states for the permutation puzzles and 2^17 for Hanoi
// (window sweeps on B200: 13-pancake three-bit 353 ms at 2^15..2^16 vs 374 ms
// at 2^17; 18-disk Hanoi two-bit 1.64 s at 2^17 vs 1.76 s at 2^16), smaller
// for small puzzles so that every SM gets windows.
int auto_window_bits(const psb_puzzle* p, int algo) {
    int lg = 0;
    while (lg < 63 && (uint64_t(1) << (lg + 1)) <= p->n_states) lg++;
    const int cap = (p->kind == PSB_HANOI4 || p->kind == PSB_HANOI4_OPT) ? 17 : 16;
    int wb = std::max(10, std::min(cap, lg - 10));
    if (algo == PSB_FRONTIER) wb = std::min(wb, 16);  // 4 mark bits per state
    return wb;
}

size_t smem_bytes(int mode, int wb, int threads = 0) {
    return psb::level_smem_bytes(mode, size_t(1) << wb, threads ? threads : psb::level_threads(mode));
}

// Shape variant of the top-down level kernel for psb_bfs_opts.threads.  With
// threads = 0, two-bit pancake and Hanoi searches of 2^32 states or more take
// 128-thread blocks, five per SM (B200 sweeps, whole search, far marks NEAR:
// 14-pancake 4.06 s at 128 threads vs 4.40 s at 256; 13-pancake 213 vs
// 219 ms; 18-disk Hanoi 1.58 vs 1.77 s).  Three-bit (13-pancake 195 vs
// 193 ms) and the sliding-tile puzzles (3x4 two-bit 45 vs 40 ms) keep 256.
int shape_variant(const psb_puzzle* p, int mode, int threads) {
    if (mode != psb::kTwoBit && mode != psb::kThreeBit) return 0;
    if (threads == 0 && mode == psb::kTwoBit && p->n_states >= (uint64_t(1) << 32) &&
        (p->kind == PSB_PANCAKE || p->kind == PSB_PANCAKE_OPT || p->kind == PSB_HANOI4 || p->kind == PSB_HANOI4_OPT))
        return 2;
    return threads == 512 ? 1 : threads == 128 ? 2 : 0;
}

int set_bit(uint64_t* d_word_base, uint64_t bit, cudaStream_t s) {
    // OR one bit into a freshly cleared array: the whole 64-bit word is written.
    static thread_local uint64_t word;  // pageable host source, copied before return
    word = uint64_t(1) << (bit & 63);
    PSB_CUDA(cudaMemcpyAsync(d_word_base + (bit >> 6), &word, 8, cudaMemcpyHostToDevice, s));
    PSB_CUDA(cudaStreamSynchronize(s));
    return PSB_OK;
}

// Where one depth's frontier lives when it is spilled: a one-bit array
// (three-bit `cur`, classic `open`), two-bit codes equal to `code`, the
// frontier search's operator nibbles less `excl`, or the single initial state.
struct SpillSource {
    const uint64_t* bitmap = nullptr;
    const uint64_t* codes = nullptr;
    uint32_t code = 0;
    const uint64_t* nibbles = nullptr;
    const uint64_t* excl = nullptr;
    uint64_t single = PSB_INVALID_INDEX;
    // Frontier search: the stream carries each state's operator bits, as
    // the reference's frontier-search segment files do (CompressedFrontierWriter).
    bool ops = false;
    // Active-window flags of this depth (one byte per 2^window_bits states,
    // a superset of the windows holding its states), or NULL: segments with
    // no flagged window are empty and skipped without touching the array.
    const uint8_t* flags = nullptr;
    int window_bits = 0;
    uint64_t n_windows = 0;
};

struct SpillTotals {
    double encode_ms = 0, drain_ms = 0, copy_ms = 0;
    uint64_t bytes = 0, segments = 0, launches = 0;
};

// Grows a device buffer to at least `need` bytes (*cap is its size in bytes).
template <class T>
int grow_device(T** p, uint64_t* cap, uint64_t need) {
    if (need <= *cap) return PSB_OK;
    PSB_CUDA(cudaFree(*p));
    *p = nullptr;
    *cap = 0;
    const uint64_t want = need + need / 4;
    PSB_CUDA(cudaMalloc(reinterpret_cast<void**>(p), want));
    *cap = want;
    return PSB_OK;
}

// Starts the copies of arena segments to free host slots (at most two in
// flight; segment i uses slot i % 2).
int spill_issue(SpillRes* R) {
    while (R->issued < R->segs.size() && R->issued < R->delivered + 2) {
        const SpillSeg& g = R->segs[R->issued];
        SpillSlot& sl = R->slot[R->issued & 1];
        if (sl.host_cap < g.bytes) {  // the slot is idle: its last segment was delivered
            if (sl.host) PSB_CUDA(cudaFreeHost(sl.host));
            sl.host = nullptr;
            sl.host_cap = 0;
            const uint64_t want = g.bytes + g.bytes / 4;
            PSB_CUDA(cudaHostAlloc(reinterpret_cast<void**>(&sl.host), want, cudaHostAllocDefault));
            sl.host_cap = want;
        }
        PSB_CUDA(cudaEventRecord(sl.start, R->copy));
        PSB_CUDA(cudaMemcpyAsync(sl.host, R->arena + g.off, g.bytes, cudaMemcpyDeviceToHost, R->copy));
        PSB_CUDA(cudaEventRecord(sl.done, R->copy));
        R->issued++;
    }
    return PSB_OK;
}

// Hands every segment of the arena's depth to the callback, in order, as its
// copy lands.  The search calls this right after launching a level, so the
// copies and callbacks run while that level is on the GPU.
int spill_drain(SpillRes* R, const psb_bfs_opts* o, SpillTotals* t) {
    const auto t0 = std::chrono::steady_clock::now();
    while (R->delivered < R->segs.size()) {
        if (int rc = spill_issue(R)) return rc;
        const SpillSeg& g = R->segs[R->delivered];
        SpillSlot& sl = R->slot[R->delivered & 1];
        PSB_CUDA(cudaEventSynchronize(sl.done));
        float ms = 0;
        PSB_CUDA(cudaEventElapsedTime(&ms, sl.start, sl.done));
        t->copy_ms += ms;
        R->delivered++;
        if (o->spill(o->spill_user, g.depth, g.segment, sl.host, g.bytes, g.states))
            return fail(PSB_ERR_ABORTED, "spill callback stopped the search at depth %u, segment %u", g.depth,
                        g.segment);
        t->bytes += g.bytes;
        t->segments++;
    }
    t->drain_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return PSB_OK;
}

// Encodes the states at `depth` into the arena, segment by segment (the
// segment's frontier bitmap is the array itself, or one extracted into the
// spill scratch), and starts the first copies.  The previous depth must be
// drained.  This takes SegmentWriter's place (Common/CompressedFrontier.cpp:
// 103-140 writes the same stream per segment).  The arrays may change as
// soon as this returns: the arena holds everything still to be copied.
int spill_depth(psb_bfs_session* S, const psb_bfs_opts* o, uint32_t depth, const SpillSource& src, SpillTotals* t) {
    const auto t0 = std::chrono::steady_clock::now();
    const uint64_t N = S->p.n_states;
    const uint64_t seg = uint64_t(1) << (o->segment_bits ? o->segment_bits : 32);
    cudaStream_t s = S->stream;
    SpillRes* R = S->spill;
    R->segs.clear();
    R->issued = R->delivered = 0;
    if (src.flags) {
        R->flags.resize(src.n_windows);
        PSB_CUDA(cudaMemcpyAsync(R->flags.data(), src.flags, src.n_windows, cudaMemcpyDeviceToHost, s));
        PSB_CUDA(cudaStreamSynchronize(s));
    }
    uint64_t off = 0;
    for (uint64_t g = 0; g * seg < N; g++) {
        const uint64_t first = g * seg, n = std::min(seg, N - first);
        if (src.flags) {
            const uint64_t w0 = first >> src.window_bits, w1 = std::min(src.n_windows, ((first + n - 1) >> src.window_bits) + 1);
            if (std::find_if(R->flags.begin() + w0, R->flags.begin() + w1, [](uint8_t f) { return f != 0; }) ==
                R->flags.begin() + w1)
                continue;
        }
        bool sums_ready = false;  // the extraction kernels also count
        if (!src.bitmap) {
            if (src.single != PSB_INVALID_INDEX && (src.single < first || src.single - first >= n)) continue;
            const uint64_t words = (n + 63) / 64;
            if (int rc = grow_device(&R->bits, &R->bits_cap, words * 8)) return rc;
            if (src.single != PSB_INVALID_INDEX) {
                PSB_CUDA(cudaMemsetAsync(R->bits, 0, words * 8, s));
                if (int rc = set_bit(R->bits, src.single - first, s)) return rc;
            } else {
                unsigned long long* sums = nullptr;
                if (int rc = psb::encoder_chunk_sums(R->enc, n, &sums)) return rc;
                t->launches++;
                const int rc =
                    src.codes ? psb::frontier_bits_two_bit(src.codes, first, n, src.code, R->bits, sums, src.flags,
                                                           src.window_bits, src.n_windows, s)
                              : psb::frontier_bits_nibbles(src.nibbles, src.excl, first, n, R->bits, sums, s);
                if (rc) return rc;
                sums_ready = true;
            }
        }
        const uint64_t* bits = src.bitmap ? src.bitmap + first / 64 : R->bits;  // after the scratch exists
        uint64_t bytes = 0, count = 0;
        psb::encoder_set_ops(R->enc, src.ops, src.nibbles, first);  // the initial state's nibble is 0
        const int prc = psb::encoder_plan(R->enc, bits, n, s, sums_ready, &bytes, &count);
        if (prc) {
            psb::encoder_set_ops(R->enc, false, nullptr, 0);
            return prc;
        }
        if (count == 0) continue;
        if (R->arena_cap < off + bytes) {  // grow, keeping this depth's segments written so far
            const uint64_t want = (off + bytes) + (off + bytes) / 4;
            uint8_t* bigger = nullptr;
            PSB_CUDA(cudaMalloc(reinterpret_cast<void**>(&bigger), want));
            if (off) PSB_CUDA(cudaMemcpyAsync(bigger, R->arena, off, cudaMemcpyDeviceToDevice, s));
            PSB_CUDA(cudaStreamSynchronize(s));
            PSB_CUDA(cudaFree(R->arena));
            R->arena = bigger;
            R->arena_cap = want;
        }
        const int wrc = psb::encoder_write(R->enc, R->arena + off, s);
        psb::encoder_set_ops(R->enc, false, nullptr, 0);
        if (wrc) return wrc;
        R->segs.push_back(SpillSeg{depth, uint32_t(g), off, bytes, count});
        off += bytes;
    }
    t->launches += psb::encoder_take_launches(R->enc);
    PSB_CUDA(cudaEventRecord(R->encoded, s));
    PSB_CUDA(cudaStreamWaitEvent(R->copy, R->encoded, 0));
    if (int rc = spill_issue(R)) return rc;
    t->encode_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return PSB_OK;
}

int session_run(psb_bfs_session* S, uint64_t initial, const psb_bfs_opts* opts, uint64_t* counts, uint32_t cap,
                uint32_t* n_depths, psb_bfs_stats* stats) {
    const psb_puzzle& P = S->p;
    const uint64_t N = P.n_states;
    if (initial >= N) return fail(PSB_ERR_ARG, "initial index %llu >= IndexesCount()", (unsigned long long)initial);
    if (!counts || !n_depths || cap == 0) return fail(PSB_ERR_ARG, "counts buffer missing");
    const uint32_t max_depth = opts ? opts->max_depth : 0;
    uint64_t* restored = opts ? opts->restored_counts : nullptr;
    const int far_marks = S->far ? far_mode(&P, S->algo, opts ? opts->far_marks : PSB_FAR_AUTO) : PSB_FAR_NONE;
    if (restored && !((P.kind == PSB_HANOI4 || P.kind == PSB_HANOI4_OPT) && P.pz.sym && S->algo == PSB_TWO_BIT))
        return fail(PSB_ERR_UNSUPPORTED, "restored_counts: 4-peg Hanoi with symmetry, two-bit searches only");
    const bool spill = opts && opts->spill;
    if (spill && opts->segment_bits && (opts->segment_bits < 6 || opts->segment_bits > 32))
        return fail(PSB_ERR_ARG, "segment_bits %d outside 6..32", opts->segment_bits);
    SpillTotals spilled;
    uint32_t spilled_depths = 0;
    cudaStream_t s = S->stream;
    if (spill) {
        if (!S->spill) if (int rc = spill_acquire(S->device, &S->spill)) return rc;
        S->spill->reset();
    }
    if (S->device >= 0) PSB_CUDA(cudaSetDevice(S->device));
    for (int i = 0; i < S->n_arr; i++) PSB_CUDA(cudaMemsetAsync(S->arr[i], 0, S->words[i] * 8, s));
    if (S->visited) PSB_CUDA(cudaMemsetAsync(S->visited, 0, S->words[0] * 8, s));
    if (S->far && far_marks != PSB_FAR_NONE) PSB_CUDA(cudaMemsetAsync(S->far, 0, S->far_words * 8, s));
    PSB_CUDA(cudaEventRecord(S->ev[0], s));
    const int direction = opts ? opts->direction : PSB_DIR_AUTO;
    const double bu_ratio = (opts && opts->bottom_up_ratio > 0) ? double(opts->bottom_up_ratio) : kBottomUpRatio;
    // Three-bit needs its visited array; classic (closed) and two-bit (codes) carry the information.
    const bool can_bu = S->bottom_up && direction != PSB_DIR_TOP_DOWN &&
                        (S->algo != PSB_THREE_BIT || S->visited != nullptr);

    const uint64_t W1 = words_for(N), W2 = words_for(2 * N), W4 = (N + 15) / 16;
    const unsigned grid = unsigned((N + (uint64_t(1) << S->window_bits) - 1) >> S->window_bits);
    const int threads_req = opts ? opts->threads : 0;
    if (threads_req != 0 && threads_req != 128 && threads_req != 256 && threads_req != 512)
        return fail(PSB_ERR_ARG, "threads must be 0, 128, 256 or 512");
    const int variant = shape_variant(&P, S->mode, threads_req);
    const size_t smem = smem_bytes(S->mode, S->window_bits, psb::variant_threads(variant));
    // Bottom-up levels use windows twice as large (fewer window-end barriers
    // per state; 13-pancake depth 12: 74 ms instead of 77 ms); top-down levels
    // keep the smaller windows, whose long-range marks stay closer together.
    const int wb_bu = std::max(S->window_bits, std::min(S->window_bits + 1, 18));
    const unsigned grid_bu = unsigned((N + (uint64_t(1) << wb_bu) - 1) >> wb_bu);
    const size_t smem_bu = smem_bytes(S->mode, wb_bu);
    LevelArgs a{};
    a.n_states = N;
    a.window_bits = S->window_bits;
    a.odd = P.odd;
    a.pz = P.pz;
    a.stats = S->d_stats;
    a.sym_mult = restored ? 1 : 0;

    uint64_t *old_ = S->arr[0], *cur = S->arr[1], *nw = S->arr[2];       // three-bit
    uint64_t *closed = S->arr[0], *open = S->arr[1], *nopen = S->arr[2]; // classic
    uint64_t *codes = S->arr[0];                                         // two-bit
    uint64_t *fcur = S->arr[0], *fnext = S->arr[1], *cex = S->arr[2], *nex = S->arr[3];  // frontier
    uint32_t cur_code = 2;

    switch (S->algo) {
    case PSB_THREE_BIT:
        if (int rc = set_bit(cur, initial, s)) return rc;
        if (S->visited) if (int rc = set_bit(S->visited, initial, s)) return rc;
        break;
    case PSB_CLASSIC:
        if (int rc = set_bit(open, initial, s)) return rc;
        if (int rc = set_bit(closed, initial, s)) return rc;
        break;
    case PSB_TWO_BIT: if (int rc = set_bit(codes, 2 * initial, s)) return rc; break;  // code CUR = 2: bit 2i
    default: break;
    }

    // Active-window flags: a level whose frontier is sparse (estimate below
    // N/64) records every window it marks; the next level then sweeps only
    // those windows.  Flags are a superset of the windows holding frontier
    // states, so skipping the others is exact.
    // Three flag arrays in rotation: the windows of this level's frontier
    // (flags_valid), of the previous level's states (flags_old; the three-bit
    // `old` array) and the ones this level marks.
    int flags_valid = -1;          // index of the flag array valid for this level, -1 = sweep every window
    int flags_old = -1;            // windows of the previous depth: -1 unknown, -2 none
    uint64_t estimate = 1;         // last known frontier size
    const uint64_t sparse_limit = N / 64;
    if (S->algo != PSB_FRONTIER) {
        // Level 0 sweeps only the window of the initial state.
        static thread_local uint8_t one;
        one = 1;
        PSB_CUDA(cudaMemsetAsync(S->wflags[0], 0, S->n_windows, s));
        PSB_CUDA(cudaMemcpyAsync(S->wflags[0] + (initial >> S->window_bits), &one, 1, cudaMemcpyHostToDevice, s));
        PSB_CUDA(cudaStreamSynchronize(s));
        flags_valid = 0;
        flags_old = -2;  // depth -1 is empty
    }

    std::vector<uint64_t> res;
    double expand_ms = 0, finalize_ms = 0;
    uint64_t expanded = 0, children = 0, local = 0, launches = 0, bu_levels = 0, others = 0;
    uint64_t seen = 0;       // states at depth < the frontier's depth
    uint64_t frontier = 1;   // states at the frontier's depth (two-bit: the kernel's estimate)
    const bool want_final = opts && opts->final_words;
    bool first = true;
    uint32_t iteration = 0;
    for (;;) {
        if (max_depth && res.size() >= size_t(max_depth) + 1) break;
        if (spill) {  // the states at depth `iteration`, before its level changes the arrays
            SpillSource src;
            switch (S->algo) {
            case PSB_THREE_BIT: src.bitmap = cur; break;
            case PSB_CLASSIC: src.bitmap = open; break;
            case PSB_TWO_BIT: src.codes = codes; src.code = cur_code; break;
            case PSB_FRONTIER:
                if (first) src.single = initial;
                else { src.nibbles = fcur; src.excl = P.odd ? cex : nullptr; }
                src.ops = true;
                break;
            }
            if (flags_valid >= 0) {
                src.flags = S->wflags[flags_valid];
                src.window_bits = S->window_bits;
                src.n_windows = S->n_windows;
            }
            if (int rc = spill_depth(S, opts, iteration, src, &spilled)) return rc;
            spilled_depths = iteration + 1;
        }
        PSB_CUDA(cudaMemsetAsync(S->d_stats, 0, 8 * sizeof(unsigned long long), s));
        // Direction of this level: bottom-up once the unvisited states are
        // fewer than ratio x the frontier (they probe until a round hits; the
        // frontier would generate every child).  Sparse frontiers stay
        // top-down: their levels sweep only the flagged windows, while a
        // bottom-up level sweeps every window.
        const uint64_t unvisited = N - std::min(N, seen + frontier);
        const bool bu = can_bu && (direction == PSB_DIR_BOTTOM_UP ||
                                   (frontier >= sparse_limit && double(unvisited) < bu_ratio * double(frontier)));
        // Window flags for the next level: a sparse top-down level records
        // the windows it marks; a two-bit bottom-up level records the
        // windows holding the states it found (in the top-down windows, half
        // the size of its own), so that the sparse tail after the last
        // bottom-up level sweeps only those (14-pancake depth 16: 35 ms of
        // full sweep otherwise).
        const bool produce = bu ? S->algo == PSB_TWO_BIT : estimate < sparse_limit;
        int flags_next = 0;
        while (flags_next == flags_valid || flags_next == flags_old) flags_next++;
        if (produce) PSB_CUDA(cudaMemsetAsync(S->wflags[flags_next], 0, S->n_windows, s));
        a.wflag_cur = flags_valid >= 0 ? S->wflags[flags_valid] : nullptr;
        a.wflag_next = produce ? S->wflags[flags_next] : nullptr;
        PSB_CUDA(cudaEventRecord(S->ev[1], s));
        uint64_t count = 0;
        if (bu) {
            a.wflag_cur = nullptr;
            a.cur_code = cur_code;
            switch (S->algo) {
            case PSB_THREE_BIT: a.front = S->visited; a.probe = cur; a.marks = nw; a.front_words = W1; a.mark_words = W1; break;
            case PSB_CLASSIC: a.front = closed; a.probe = open; a.marks = nopen; a.front_words = W1; a.mark_words = W1; break;
            case PSB_TWO_BIT: a.front = codes; a.probe = codes; a.marks = codes; a.front_words = W2; a.mark_words = W2; break;
            }
            a.window_bits = wb_bu;
            a.flag_bits = S->window_bits;
            PSB_CUDA(P.k.level_bu[S->mode](a, grid_bu, smem_bu, s));
            a.window_bits = S->window_bits;
            a.flag_bits = 0;
            launches++;
            bu_levels++;
        } else if (S->algo == PSB_FRONTIER && first) {
            a.marks = fnext; a.excl_next = nex; a.mark_words = W4;
            PSB_CUDA(P.k.seed(a, initial, s));
        } else {
            switch (S->algo) {
            case PSB_THREE_BIT: a.front = cur; a.marks = nw; a.front_words = W1; a.mark_words = W1; break;
            case PSB_CLASSIC: a.front = open; a.marks = nopen; a.front_words = W1; a.mark_words = W1; break;
            case PSB_TWO_BIT:
                a.front = codes; a.marks = codes; a.front_words = W2; a.mark_words = W2; a.cur_code = cur_code;
                a.far = far_marks != PSB_FAR_NONE ? S->far : nullptr;
                a.far_all = far_marks == PSB_FAR_ALL ? 1 : 0;
                break;
            case PSB_FRONTIER:
                a.front = fcur; a.marks = fnext; a.excl_cur = cex; a.excl_next = nex;
                a.front_words = W4; a.mark_words = W4;
                break;
            }
            PSB_CUDA((variant ? P.k.level_shape[variant][S->mode] : P.k.level[S->mode])(a, grid, smem, s));
            a.far = nullptr;
            launches++;
        }
        PSB_CUDA(cudaEventRecord(S->ev[2], s));
        const bool bu_three = bu && S->algo == PSB_THREE_BIT;
        if (bu_three) {
            // The bottom-up flush already ORed the found states into `visited`,
            // and they were all unvisited, so new &= ~old (& ~cur) changes
            // nothing: only `old` must be zeroed for reuse (as finalize does).
            if (!want_final) PSB_CUDA(cudaMemsetAsync(old_, 0, W1 * 8, s));
        } else if (S->algo == PSB_THREE_BIT || S->algo == PSB_CLASSIC) {
            const unsigned fgrid = 148 * 8;
            const uint64_t n2 = (W1 + 1) / 2;
            if (S->algo == PSB_THREE_BIT && produce && flags_old != -1 && !want_final)
                psb::finalize_three_bit_flagged<<<fgrid, psb::kThreads, 0, s>>>(
                    reinterpret_cast<const ulonglong2*>(cur), reinterpret_cast<ulonglong2*>(nw),
                    reinterpret_cast<ulonglong2*>(old_), reinterpret_cast<ulonglong2*>(S->visited), n2,
                    S->wflags[flags_next], flags_old >= 0 ? S->wflags[flags_old] : nullptr, S->n_windows,
                    uint32_t((uint64_t(1) << S->window_bits) / 128), P.odd, S->d_stats + 4);
            else if (S->algo == PSB_THREE_BIT && S->visited)
                psb::finalize_three_bit_visited<<<fgrid, psb::kThreads, 0, s>>>(
                    reinterpret_cast<const ulonglong2*>(cur), reinterpret_cast<ulonglong2*>(nw),
                    reinterpret_cast<ulonglong2*>(old_), reinterpret_cast<ulonglong2*>(S->visited), n2, P.odd,
                    want_final ? 0 : 1, S->d_stats + 4);
            else if (S->algo == PSB_THREE_BIT)
                psb::finalize_three_bit<<<fgrid, psb::kThreads, 0, s>>>(
                    reinterpret_cast<const ulonglong2*>(cur), reinterpret_cast<ulonglong2*>(nw),
                    reinterpret_cast<ulonglong2*>(old_), n2, P.odd, want_final ? 0 : 1, S->d_stats + 4);
            else if (bu)
                psb::finalize_classic_clear<<<fgrid, psb::kThreads, 0, s>>>(
                    reinterpret_cast<ulonglong2*>(nopen), reinterpret_cast<ulonglong2*>(closed),
                    reinterpret_cast<ulonglong2*>(open), n2, S->d_stats + 4);
            else
                psb::finalize_classic<<<fgrid, psb::kThreads, 0, s>>>(
                    reinterpret_cast<ulonglong2*>(nopen), reinterpret_cast<ulonglong2*>(closed), n2, S->d_stats + 4);
            PSB_CUDA(cudaGetLastError());
            others++;
        } else if (S->algo == PSB_TWO_BIT && bu) {
            psb::retire_two_bit<<<148 * 8, psb::kThreads, 0, s>>>(reinterpret_cast<ulonglong2*>(codes), (W2 + 1) / 2,
                                                                 cur_code, S->d_stats + 4);
            PSB_CUDA(cudaGetLastError());
            others++;
        } else if (S->algo == PSB_TWO_BIT && S->far && far_marks != PSB_FAR_NONE) {
            const uint64_t n4 = (W2 + 3) / 4;
            const uint32_t next_lo = cur_code == 2 ? 1u : 0u;  // NEXT = 5 - CUR
            if (produce)
                psb::fold_two_bit_flagged<<<148 * 8, psb::kThreads, 0, s>>>(
                    reinterpret_cast<ulonglong2*>(codes), reinterpret_cast<uint4*>(S->far), n4, S->wflags[flags_next],
                    S->n_windows, uint32_t((uint64_t(1) << S->window_bits) / 128), next_lo, S->d_stats + 6,
                    S->d_stats + 5);
            else
                psb::fold_two_bit<<<148 * 8, psb::kThreads, 0, s>>>(reinterpret_cast<ulonglong2*>(codes),
                                                                   reinterpret_cast<uint4*>(S->far), n4, next_lo,
                                                                   S->d_stats + 6, S->d_stats + 5);
            PSB_CUDA(cudaGetLastError());
            others++;
        }
        PSB_CUDA(cudaEventRecord(S->ev[3], s));
        if (spill) if (int rc = spill_drain(S->spill, opts, &spilled)) return rc;  // overlaps this level
        PSB_CUDA(cudaMemcpyAsync(S->h_stats, S->d_stats, 8 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
        PSB_CUDA(cudaStreamSynchronize(s));
        if (S->h_stats[3]) return fail(PSB_ERR_DEVICE, "level kernel produced a child index >= IndexesCount()");
        float t_exp = 0, t_fin = 0;
        PSB_CUDA(cudaEventElapsedTime(&t_exp, S->ev[1], S->ev[2]));
        PSB_CUDA(cudaEventElapsedTime(&t_fin, S->ev[2], S->ev[3]));
        expand_ms += t_exp;
        finalize_ms += t_fin;
        expanded += (S->algo == PSB_FRONTIER && first) ? 1 : S->h_stats[0];
        children += S->h_stats[1];
        local += S->h_stats[2];
        const size_t lvl = size_t(iteration++);  // the depth this level kernel expanded
        if (opts && opts->level_ms && lvl < cap) opts->level_ms[lvl] = t_exp + t_fin;
        if (opts && opts->level_children && lvl < cap) opts->level_children[lvl] = S->h_stats[1];

        switch (S->algo) {
        case PSB_THREE_BIT:
            count = bu_three ? S->h_stats[2] : S->h_stats[4];  // bottom-up: the states found
            if (first) { res.push_back(1); }
            if (count == 0) goto done;
            res.push_back(count);
            { uint64_t* t = old_; old_ = cur; cur = nw; nw = t; }  // old<-cur, cur<-new, new<-old
            if (want_final) PSB_CUDA(cudaMemsetAsync(nw, 0, W1 * 8, s));
            break;
        case PSB_CLASSIC:
            count = S->h_stats[4];
            if (first) { res.push_back(1); }
            if (count == 0) goto done;
            res.push_back(count);
            std::swap(open, nopen);
            break;
        case PSB_TWO_BIT:
            count = bu ? S->h_stats[4] : S->h_stats[0];  // states with code CUR = states at this depth
            if (count == 0) goto done;
            if (restored && res.size() < cap) restored[res.size()] = res.empty() ? 1 : S->h_stats[7];
            res.push_back(count);
            cur_code = 5 - cur_code;
            break;
        case PSB_FRONTIER:
            count = first ? 1 : S->h_stats[0];
            if (count == 0) goto done;
            res.push_back(count);
            std::swap(fcur, fnext);
            if (P.odd) {
                std::swap(cex, nex);
                PSB_CUDA(cudaMemsetAsync(nex, 0, W1 * 8, s));
            }
            break;
        }
        first = false;
        flags_old = flags_valid;
        flags_valid = produce ? flags_next : -1;
        estimate = count;
        if (S->algo == PSB_TWO_BIT) {  // res holds depths 0..d; the next frontier is only estimated
            seen += count;
            frontier = S->h_stats[5];
        } else {                       // res holds depths 0..d+1
            seen += res[res.size() - 2];
            frontier = res.back();
        }
        if (res.size() > cap) return fail(PSB_ERR_CAPACITY, "more than %u depths", cap);
        // Two-bit: h_stats[5] counts every UNVISITED -> NEXT move of the level
        // (some twice), so 0 means the next depth is empty.  The level that
        // would only sweep the array to find that out (a 14-pancake sweep is
        // 35 ms) is not launched: counts and arrays are the same without it.
        if (S->algo == PSB_TWO_BIT && frontier == 0) break;
    }
done:
    if (spill && spilled_depths < res.size()) {
        // Three-bit and classic searches stopped by max_depth hold their
        // last depth, which no level expanded, in cur / open.
        SpillSource src;
        src.bitmap = S->algo == PSB_THREE_BIT ? cur : open;
        if (int rc = spill_depth(S, opts, spilled_depths, src, &spilled)) return rc;
    }
    if (spill) if (int rc = spill_drain(S->spill, opts, &spilled)) return rc;
    PSB_CUDA(cudaEventRecord(S->ev[3], s));
    PSB_CUDA(cudaEventSynchronize(S->ev[3]));
    float total = 0;
    PSB_CUDA(cudaEventElapsedTime(&total, S->ev[0], S->ev[3]));
    if (res.size() > cap) return fail(PSB_ERR_CAPACITY, "more than %u depths", cap);
    std::copy(res.begin(), res.end(), counts);
    *n_depths = uint32_t(res.size());

    if (want_final) {
        uint64_t need = 0;
        psb_final_words(&P, S->algo, &need);
        if (opts->final_cap < need) return fail(PSB_ERR_CAPACITY, "final_words needs %llu words", (unsigned long long)need);
        uint64_t* out = opts->final_words;
        auto copy = [&](const uint64_t* src, uint64_t w) -> int {
            PSB_CUDA(cudaMemcpyAsync(out, src, w * 8, cudaMemcpyDeviceToHost, s));
            out += w;
            return PSB_OK;
        };
        int rc = PSB_OK;
        switch (S->algo) {
        case PSB_THREE_BIT: rc = copy(old_, W1); if (!rc) rc = copy(cur, W1); if (!rc) rc = copy(nw, W1); break;
        case PSB_CLASSIC: rc = copy(closed, W1); if (!rc) rc = copy(open, W1); if (!rc) rc = copy(nopen, W1); break;
        case PSB_TWO_BIT: rc = copy(codes, W2); break;
        case PSB_FRONTIER: rc = copy(fcur, W4); if (!rc) rc = copy(fnext, W4); break;
        }
        if (rc) return rc;
        PSB_CUDA(cudaStreamSynchronize(s));
    }
    if (stats && stats->struct_size >= sizeof(psb_bfs_stats)) {
        stats->levels = uint32_t(launches);
        stats->window_bits = uint32_t(S->window_bits);
        stats->threads = uint32_t(variant ? psb::variant_threads(variant) : psb::level_threads(S->mode));
        stats->total_ms = total;
        stats->expand_ms = expand_ms;
        stats->finalize_ms = finalize_ms;
        stats->expanded = expanded;
        stats->children = children;
        stats->local_children = local;
        stats->expand_launches = launches;
        stats->device_bytes = S->bytes;
        stats->bottom_up_levels = bu_levels;
        stats->spill_ms = spilled.encode_ms + spilled.drain_ms;
        stats->spill_encode_ms = spilled.encode_ms;
        stats->spill_copy_ms = spilled.copy_ms;
        stats->spill_bytes = spilled.bytes;
        stats->spill_segments = spilled.segments;
        stats->spill_launches = spilled.launches;
        stats->other_launches = others;
    }
    return PSB_OK;
}

}  // namespace

extern "C" {

int psb_bfs_footprint(const psb_puzzle* p, int algo, uint64_t* bytes) {
    if (!p || !bytes) return fail(PSB_ERR_ARG, "bad argument");
    uint64_t w[4] = {0, 0, 0, 0};
    int n = 0;
    if (int rc = layout(p, algo, w, &n)) return rc;
    *bytes = (w[0] + w[1] + w[2] + w[3]) * 8 + 64;
    if (algo == PSB_THREE_BIT && supports_bottom_up(p, algo)) *bytes += w[0] * 8;  // visited array
    if (far_mode(p, algo, PSB_FAR_AUTO) != PSB_FAR_NONE) *bytes += padded(words_for(p->n_states)) * 8;  // far bitmap
    return PSB_OK;
}

int psb_bfs_session_create(const psb_puzzle* p, int algo, const psb_bfs_opts* opts, psb_bfs_session** out) {
    if (!p || !out) return fail(PSB_ERR_ARG, "bad argument");
    if (opts && opts->struct_size != sizeof(psb_bfs_opts)) return fail(PSB_ERR_ARG, "psb_bfs_opts.struct_size mismatch");
    auto S = std::make_unique<psb_bfs_session>();
    S->p = *p;
    S->algo = algo;
    S->mode = mode_of(algo);
    if (S->mode < 0) return fail(PSB_ERR_ARG, "unknown algorithm %d", algo);
    if (int rc = layout(p, algo, S->words, &S->n_arr)) return rc;
    S->device = opts ? opts->device : -1;
    if (int rc = ensure_device(S->device)) return rc;
    if (S->device < 0) PSB_CUDA(cudaGetDevice(&S->device));
    S->window_bits = (opts && opts->window_bits) ? opts->window_bits : auto_window_bits(p, algo);
    if (S->window_bits < 10 || S->window_bits > 20 || (algo == PSB_FRONTIER && S->window_bits > 18))
        return fail(PSB_ERR_ARG, "window_bits %d out of range", S->window_bits);
    if (((p->n_states + (uint64_t(1) << S->window_bits) - 1) >> S->window_bits) > 0x7FFFFFFFull)
        return fail(PSB_ERR_ARG, "too many windows");
    if (opts && opts->stream) S->stream = static_cast<cudaStream_t>(opts->stream);
    else {
        PSB_CUDA(cudaStreamCreateWithFlags(&S->stream, cudaStreamNonBlocking));
        S->own_stream = true;
    }
    if (int rc = session_pool(S->device, &S->pool)) return rc;
    for (int i = 0; i < S->n_arr; i++)
        if (int rc = S->alloc(reinterpret_cast<void**>(&S->arr[i]), S->words[i] * 8)) return rc;
    S->bottom_up = supports_bottom_up(p, algo);
    if (S->bottom_up && algo == PSB_THREE_BIT && !(opts && opts->direction == PSB_DIR_TOP_DOWN)) {
        // Optional: without room for the visited array the search runs every
        // level top-down, in the reference's three arrays.
        void* v = nullptr;
        if (cudaMallocFromPoolAsync(&v, S->words[0] * 8, S->pool, S->stream) == cudaSuccess) {
            S->visited = static_cast<uint64_t*>(v);
            S->bytes += S->words[0] * 8;
        } else {
            cudaGetLastError();  // an allocation failure is not sticky; clear it
        }
    }
    if (far_mode(p, algo, opts ? opts->far_marks : PSB_FAR_AUTO) != PSB_FAR_NONE) {
        // Optional as well: without room for the far bitmap every long-range
        // mark reads the target's code first.
        void* v = nullptr;
        const uint64_t fw = padded(words_for(p->n_states));
        if (cudaMallocFromPoolAsync(&v, fw * 8, S->pool, S->stream) == cudaSuccess) {
            S->far = static_cast<uint32_t*>(v);
            S->far_words = fw;
            S->bytes += fw * 8;
        } else {
            cudaGetLastError();
        }
    }
    S->n_windows = (p->n_states + (uint64_t(1) << S->window_bits) - 1) >> S->window_bits;
    for (auto& f : S->wflags)
        if (int rc = S->alloc(reinterpret_cast<void**>(&f), S->n_windows)) return rc;
    if (int rc = S->alloc(reinterpret_cast<void**>(&S->d_stats), 8 * sizeof(unsigned long long))) return rc;
    PSB_CUDA(cudaMallocHost(&S->h_stats, 8 * sizeof(unsigned long long)));
    for (auto& e : S->ev) PSB_CUDA(cudaEventCreate(&e));
    *out = S.release();
    return PSB_OK;
}

int psb_bfs_session_run(psb_bfs_session* s, uint64_t initial, const psb_bfs_opts* opts, uint64_t* counts,
                        uint32_t cap, uint32_t* n_depths, psb_bfs_stats* stats) {
    if (!s) return fail(PSB_ERR_ARG, "session is NULL");
    if (opts && opts->struct_size != sizeof(psb_bfs_opts)) return fail(PSB_ERR_ARG, "psb_bfs_opts.struct_size mismatch");
    return session_run(s, initial, opts, counts, cap, n_depths, stats);
}

int psb_bfs_session_destroy(psb_bfs_session* s) {
    delete s;
    return PSB_OK;
}

int psb_release_cached_memory(int device) {
    if (int rc = ensure_device(device)) return rc;
    if (device < 0) PSB_CUDA(cudaGetDevice(&device));
    if (device >= kMaxPoolDevices) return PSB_OK;
    cudaMemPool_t pool = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_pool_mu);
        pool = g_pools[device];
    }
    std::vector<SpillRes*> cached;
    {
        std::lock_guard<std::mutex> lock(g_spill_mu);
        cached.swap(g_spill_cache[device]);
    }
    for (SpillRes* R : cached) delete R;
    if (!pool) return PSB_OK;
    PSB_CUDA(cudaDeviceSynchronize());  // frees still queued on streams return first
    PSB_CUDA(cudaMemPoolTrimTo(pool, 0));
    return PSB_OK;
}

int psb_bfs(const psb_puzzle* p, int algo, uint64_t initial, const psb_bfs_opts* opts, uint64_t* counts,
            uint32_t cap, uint32_t* n_depths, psb_bfs_stats* stats) {
    psb_bfs_session* s = nullptr;
    if (int rc = psb_bfs_session_create(p, algo, opts, &s)) return rc;
    std::unique_ptr<psb_bfs_session> guard(s);
    return session_run(s, initial, opts, counts, cap, n_depths, stats);
}

}  // extern "C"
