// psb_kernels.cuh -- sm_100a kernels of the complete-BFS hot path.
//
// One level of an in-memory search is ONE fused kernel: each thread block
// owns an aligned window of 2^window_bits states.  For each window it
//   1. sweeps the frontier words of the window (coalesced 64-bit loads, one
//      word per thread), applying the algorithm's sweep-side update
//      (three-bit: read only; classic: clear open; two-bit: CUR -> OLD with
//      an atomic XOR; frontier search: clear the 4-bit operator words and
//      apply the exclusion bitsets);
//   2. compacts the frontier states of each batch into a shared-memory list
//      with a block-wide prefix sum, so every thread expands a parent;
//   3. expands each parent (unrank -> each legal move -> rank) and marks each
//      child: children inside the block's own window go to a shared-memory
//      bitmap with shared atomics; the rest go straight to global memory
//      with fire-and-forget atomic ORs (RED);
//   4. flushes the shared-memory bitmap into global memory, one atomic OR per
//      non-zero 64-bit word.
// Puzzle moves are local in index space (a pancake flip of the last k values
// only changes the last k Lehmer digits; a Hanoi move of disk d only changes
// bits 2d..2d+1), so most children land in the block's own window and the
// scattered global traffic shrinks to the long-range moves.
//
// Array layouts follow the reference exactly (Common/BitArray.h:69-169 and
// Common/InMemory*.cpp), so final arrays can be compared bit for bit:
//   1-bit arrays:   state i -> word i/64, bit i%64
//   2-bit codes:    state i -> bit 2i = code/2, bit 2i+1 = code%2 (vector<bool>)
//   4-bit op bits:  state i -> word i/16, bits 4*(i%16) .. +3
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "psb_puzzles.cuh"

namespace psb {

constexpr int kThreads = 256;

enum Mode : int { kThreeBit = 0, kClassic = 1, kTwoBit = 2, kFrontier = 3 };

struct PuzzleArgs {
    int width;  // sliding tile: board width
    int disks;  // Hanoi: number of disks
    int sym;    // Hanoi: symmetry flag
};

// Adapters giving the three puzzles one device interface.
template <int N>
struct PancakeK {
    static constexpr int kBranch = N - 1;
    static constexpr int kOps = N - 1;
    template <bool kOpBits, class E>
    __device__ __forceinline__ static void expand(uint64_t i, uint32_t ob, const PuzzleArgs&, E& e) {
        Pancake<N>::template expand<kOpBits>(i, ob, e);
    }
};
template <int N>
struct SlidingK {
    static constexpr int kBranch = 4;
    static constexpr int kOps = 4;
    template <bool kOpBits, class E>
    __device__ __forceinline__ static void expand(uint64_t i, uint32_t ob, const PuzzleArgs& a, E& e) {
        Sliding<N>::template expand<kOpBits>(i, ob, a.width, e);
    }
};
struct HanoiK {
    static constexpr int kBranch = 6;
    static constexpr int kOps = 4;
    template <bool kOpBits, class E>
    __device__ __forceinline__ static void expand(uint64_t i, uint32_t ob, const PuzzleArgs& a, E& e) {
        Hanoi::template expand<kOpBits>(i, ob, a.disks, a.sym != 0, e);
    }
};

struct LevelArgs {
    uint64_t* front;           // frontier array (see the mode table above)
    uint64_t* marks;           // array the children are marked in
    const uint64_t* excl_cur;  // frontier search with odd cycles: states expanded last level
    uint64_t* excl_next;       // frontier search with odd cycles: states expanded this level
    uint64_t n_states;         // Puzzle::IndexesCount()
    uint64_t front_words;      // 64-bit words of `front`
    uint64_t mark_words;       // 64-bit words of `marks`
    int window_bits;           // log2 states per block window (>= 10)
    uint32_t cur_code;         // two-bit: code of the frontier (2 or 3); NEXT = 5 - CUR
    int odd;                   // frontier search: exclusion bitsets in use
    PuzzleArgs pz;
    unsigned long long* stats;  // [0] frontier states, [1] children, [2] local children, [3] error flag
};

constexpr uint64_t kEven = 0x5555555555555555ull;

// bits at even positions 2j -> bit j (32 bits)
__device__ __forceinline__ uint32_t gather_even(uint64_t t) {
    t &= kEven;
    t = (t | (t >> 1)) & 0x3333333333333333ull;
    t = (t | (t >> 2)) & 0x0F0F0F0F0F0F0F0Full;
    t = (t | (t >> 4)) & 0x00FF00FF00FF00FFull;
    t = (t | (t >> 8)) & 0x0000FFFF0000FFFFull;
    t = (t | (t >> 16)) & 0x00000000FFFFFFFFull;
    return uint32_t(t);
}
// bit j -> even position 2j
__device__ __forceinline__ uint64_t spread_even(uint32_t x32) {
    uint64_t x = x32;
    x = (x | (x << 16)) & 0x0000FFFF0000FFFFull;
    x = (x | (x << 8)) & 0x00FF00FF00FF00FFull;
    x = (x | (x << 4)) & 0x0F0F0F0F0F0F0F0Full;
    x = (x | (x << 2)) & 0x3333333333333333ull;
    x = (x | (x << 1)) & kEven;
    return x;
}
// non-zero nibble flags of a 16-nibble word -> 16-bit mask
__device__ __forceinline__ uint32_t nibble_flags(uint64_t x) {
    uint64_t t = x | (x >> 1);
    t |= t >> 2;
    t &= 0x1111111111111111ull;
    t = (t | (t >> 3)) & 0x0303030303030303ull;
    t = (t | (t >> 6)) & 0x000F000F000F000Full;
    t = (t | (t >> 12)) & 0x000000FF000000FFull;
    t = (t | (t >> 24)) & 0xFFFFull;
    return uint32_t(t);
}

// Block-wide exclusive prefix sum (kThreads threads); also returns the total.
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t x, uint32_t* s_warp, uint32_t& total) {
    constexpr int kWarps = kThreads / 32;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t incl = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
        if (lane >= o) incl += y;
    }
    if (lane == 31) s_warp[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < kWarps ? s_warp[lane] : 0;
#pragma unroll
        for (int o = 1; o < kWarps; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < kWarps) s_warp[lane] = w;
    }
    __syncthreads();
    total = s_warp[kWarps - 1];
    return (warp ? s_warp[warp - 1] : 0) + incl - x;
}

template <int MODE>
struct Emitter {
    uint64_t base;        // first state of the block's window
    uint32_t span;        // states in the window
    uint32_t* smarks;     // shared-memory window marks
    uint64_t* gmarks;     // global mark array
    uint64_t n_states;
    uint32_t next_pat;    // two-bit: bits of the NEXT code (hi at bit 0, lo at bit 1)
    uint32_t children = 0, local = 0, bad = 0;

    __device__ __forceinline__ void operator()(uint64_t c, uint32_t op) {
        if (c >= n_states) { bad = 1; return; }  // never expected: keeps a bad index off the memory system
        ++children;
        const uint64_t o = c - base;
        if (o < span) {
            ++local;
            if constexpr (MODE == kFrontier) atomicOr(&smarks[o >> 3], 1u << (4 * (uint32_t(o) & 7u) + op));
            else atomicOr(&smarks[o >> 5], 1u << (uint32_t(o) & 31u));
        } else if constexpr (MODE == kFrontier) {
            atomicOr(reinterpret_cast<unsigned int*>(gmarks) + (c >> 3), 1u << (4 * (uint32_t(c) & 7u) + op));
        } else if constexpr (MODE == kTwoBit) {
            unsigned long long* w = reinterpret_cast<unsigned long long*>(gmarks) + (c >> 5);
            const uint32_t sh = 2u * (uint32_t(c) & 31u);
            const uint64_t v = __ldcg(reinterpret_cast<const unsigned long long*>(w));
            if (((v >> sh) & 3u) == 0) atomicOr(w, (unsigned long long)next_pat << sh);  // UNVISITED -> NEXT
        } else {
            atomicOr(reinterpret_cast<unsigned int*>(gmarks) + (c >> 5), 1u << (uint32_t(c) & 31u));
        }
    }
};

template <class PZ, int MODE>
__global__ void __launch_bounds__(kThreads) level_kernel(LevelArgs a) {
    extern __shared__ __align__(16) unsigned long long smem64[];
    __shared__ uint32_t s_warp[kThreads / 32];
    const int tid = threadIdx.x;
    const uint32_t W = 1u << a.window_bits;
    const uint64_t base = uint64_t(blockIdx.x) << a.window_bits;
    if (base >= a.n_states) return;
    const uint64_t remaining = a.n_states - base;
    const uint32_t span = remaining < W ? uint32_t(remaining) : W;
    constexpr uint32_t kSPU = MODE == kTwoBit ? 32 : 64;  // states per thread unit
    const uint32_t units = (span + kSPU - 1) / kSPU;
    constexpr uint32_t kMarkBits = MODE == kFrontier ? 4 : 1;
    const uint32_t mark_u32 = (W * kMarkBits) / 32;
    uint32_t* smarks = reinterpret_cast<uint32_t*>(smem64);
    uint16_t* list16 = reinterpret_cast<uint16_t*>(smarks + mark_u32);
    uint32_t* list32 = smarks + mark_u32;

    for (uint32_t i = tid; i < mark_u32; i += kThreads) smarks[i] = 0;
    __syncthreads();

    Emitter<MODE> em{base, W, smarks, a.marks, a.n_states, 1u | (a.cur_code == 2 ? 2u : 0u)};
    uint32_t found = 0;

    for (uint32_t u0 = 0; u0 < units; u0 += kThreads) {
        const uint32_t u = u0 + tid;
        uint64_t pmask = 0;
        uint64_t nib0 = 0, nib1 = 0, nib2 = 0, nib3 = 0;
        if (u < units) {
            if constexpr (MODE == kThreeBit) {
                pmask = a.front[(base >> 6) + u];
            } else if constexpr (MODE == kClassic) {
                uint64_t* p = a.front + (base >> 6) + u;
                pmask = *p;
                if (pmask) *p = 0;  // BitArray::ScanBitsAndClear
            } else if constexpr (MODE == kTwoBit) {
                unsigned long long* p = reinterpret_cast<unsigned long long*>(a.front) + (base >> 5) + u;
                const uint64_t w = *p;
                const uint64_t hi = w & kEven, lo = (w >> 1) & kEven;
                const uint64_t cur = hi & (a.cur_code == 3 ? lo : ~lo);
                if (cur) atomicXor(p, (unsigned long long)(cur | (a.cur_code == 2 ? (cur << 1) : 0)));  // CUR -> OLD (1)
                pmask = gather_even(cur);
            } else {
                const uint64_t w0 = (base >> 4) + 4ull * u;
                uint64_t* p = a.front + w0;
                if (w0 + 0 < a.front_words) { nib0 = p[0]; if (nib0) p[0] = 0; }
                if (w0 + 1 < a.front_words) { nib1 = p[1]; if (nib1) p[1] = 0; }
                if (w0 + 2 < a.front_words) { nib2 = p[2]; if (nib2) p[2] = 0; }
                if (w0 + 3 < a.front_words) { nib3 = p[3]; if (nib3) p[3] = 0; }
                pmask = uint64_t(nibble_flags(nib0)) | (uint64_t(nibble_flags(nib1)) << 16) |
                        (uint64_t(nibble_flags(nib2)) << 32) | (uint64_t(nibble_flags(nib3)) << 48);
                if (a.odd) {
                    const uint64_t ex = a.excl_cur[(base >> 6) + u];
                    pmask &= ~ex;
                    a.excl_next[(base >> 6) + u] = pmask;
                }
            }
        }
        const uint32_t cnt = __popcll(pmask);
        found += cnt;
        uint32_t total;
        uint32_t off = block_exclusive_scan(cnt, s_warp, total);
        const uint32_t ub = uint32_t(tid) * kSPU;
        while (pmask) {
            const uint32_t j = __ffsll((long long)pmask) - 1;
            pmask &= pmask - 1;
            if constexpr (MODE == kFrontier) {
                const uint64_t nw = j < 16 ? nib0 : j < 32 ? nib1 : j < 48 ? nib2 : nib3;
                const uint32_t bits = uint32_t(nw >> (4 * (j & 15))) & 15u;
                list32[off++] = (ub + j) | (bits << 16);
            } else {
                list16[off++] = uint16_t(ub + j);
            }
        }
        __syncthreads();
        const uint64_t batch_base = base + uint64_t(u0) * kSPU;
        for (uint32_t k = tid; k < total; k += kThreads) {
            if constexpr (MODE == kFrontier) {
                const uint32_t e = list32[k];
                PZ::template expand<true>(batch_base + (e & 0xFFFFu), e >> 16, a.pz, em);
            } else {
                PZ::template expand<false>(batch_base + list16[k], 0u, a.pz, em);
            }
        }
        __syncthreads();
    }

    // Flush the window's shared-memory marks.
    if constexpr (MODE == kTwoBit) {
        const uint32_t next_pat = em.next_pat;
        unsigned long long* codes = reinterpret_cast<unsigned long long*>(a.marks) + (base >> 5);
        for (uint32_t i = tid; i < mark_u32; i += kThreads) {
            const uint32_t v = smarks[i];
            if (!v || (base >> 5) + i >= a.mark_words) continue;
            const uint64_t w = __ldcg(codes + i);
            const uint64_t unvisited = ~(w | (w >> 1)) & kEven;
            const uint64_t m = spread_even(v) & unvisited;
            if (m) atomicOr(codes + i, (unsigned long long)(m | ((next_pat & 2u) ? (m << 1) : 0)));
        }
    } else {
        constexpr uint32_t kShift = MODE == kFrontier ? 4 : 6;  // states per 64-bit word: 16 or 64
        unsigned long long* g = reinterpret_cast<unsigned long long*>(a.marks) + (base >> kShift);
        for (uint32_t i = tid; i < mark_u32 / 2; i += kThreads) {
            const unsigned long long v = smem64[i];
            if (v && (base >> kShift) + i < a.mark_words) atomicOr(g + i, v);
        }
    }

    // Counters: one atomic per block and counter.
    uint32_t c0 = __reduce_add_sync(0xFFFFFFFFu, found);
    uint32_t c1 = __reduce_add_sync(0xFFFFFFFFu, em.children);
    uint32_t c2 = __reduce_add_sync(0xFFFFFFFFu, em.local);
    uint32_t c3 = __reduce_or_sync(0xFFFFFFFFu, em.bad);
    if ((tid & 31) == 0) {
        if (c0) atomicAdd(&a.stats[0], (unsigned long long)c0);
        if (c1) atomicAdd(&a.stats[1], (unsigned long long)c1);
        if (c2) atomicAdd(&a.stats[2], (unsigned long long)c2);
        if (c3) atomicOr(&a.stats[3], 1ull);
    }
}

// Level 0 of frontier search (InMemoryFrontierSearch.cpp:81-88): expand the
// initial state with no used-operator bits.
template <class PZ>
__global__ void seed_kernel(LevelArgs a, uint64_t initial) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    Emitter<kFrontier> em{~uint64_t(0), 0, nullptr, a.marks, a.n_states, 0};
    PZ::template expand<true>(initial, 0u, a.pz, em);
    if (a.odd) a.excl_next[initial >> 6] |= 1ull << (initial & 63);
    a.stats[1] += em.children;
    if (em.bad) a.stats[3] = 1;
}

// Batched Expand (Puzzle::Expand; GPU twin of Puzzles/PuzzleGpu.cpp:53-82):
// one thread per parent, BranchingFactor slots per parent, valid children
// first in the reference order, unused slots INVALID_INDEX with operator
// (1 << OperatorsCount) - 1.
template <class PZ>
struct SlotEmitter {
    uint64_t* out;
    uint32_t* ops;
    int k = 0;
    __device__ __forceinline__ void operator()(uint64_t c, uint32_t op) {
        out[k] = c;
        ops[k] = op;
        ++k;
    }
};

template <class PZ, bool kOpBits>
__global__ void __launch_bounds__(kThreads) expand_batch_kernel(const uint64_t* __restrict__ parents,
                                                               const uint32_t* __restrict__ opbits, uint64_t n,
                                                               uint64_t n_states, uint64_t* __restrict__ children,
                                                               uint32_t* __restrict__ child_ops, PuzzleArgs pz,
                                                               unsigned long long* err) {
    const uint64_t i = blockIdx.x * uint64_t(kThreads) + threadIdx.x;
    if (i >= n) return;
    constexpr int kB = PZ::kBranch;
    uint64_t* out = children + i * kB;
    uint32_t* ops = child_ops + i * kB;
    const uint64_t p = parents[i];
    int k = 0;
    if (p < n_states) {
        SlotEmitter<PZ> em{out, ops};
        PZ::template expand<kOpBits>(p, kOpBits ? opbits[i] : 0u, pz, em);
        k = em.k;
    } else {
        atomicOr(err, 1ull);
    }
    const uint32_t inv_op = (1u << PZ::kOps) - 1u;
    for (; k < kB; ++k) {
        out[k] = kInvalidIndex;
        ops[k] = inv_op;
    }
}

// ---------------------------------------------------------------------------
// Launch helpers and per-puzzle dispatch tables.
// ---------------------------------------------------------------------------
using LevelLaunch = cudaError_t (*)(const LevelArgs&, unsigned grid, size_t smem, cudaStream_t);
using SeedLaunch = cudaError_t (*)(const LevelArgs&, uint64_t initial, cudaStream_t);
using ExpandLaunch = cudaError_t (*)(const uint64_t*, const uint32_t*, uint64_t, uint64_t, uint64_t*, uint32_t*,
                                     PuzzleArgs, unsigned long long*, bool, cudaStream_t);

struct PuzzleKernels {
    LevelLaunch level[4];  // indexed by Mode
    SeedLaunch seed;
    ExpandLaunch expand;
    int branching;
};

template <class PZ, int MODE>
cudaError_t launch_level(const LevelArgs& a, unsigned grid, size_t smem, cudaStream_t s) {
    cudaError_t e = cudaFuncSetAttribute(level_kernel<PZ, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         int(smem));
    if (e != cudaSuccess) return e;
    level_kernel<PZ, MODE><<<grid, kThreads, smem, s>>>(a);
    return cudaGetLastError();
}

template <class PZ>
cudaError_t launch_seed(const LevelArgs& a, uint64_t initial, cudaStream_t s) {
    seed_kernel<PZ><<<1, 32, 0, s>>>(a, initial);
    return cudaGetLastError();
}

template <class PZ>
cudaError_t launch_expand(const uint64_t* parents, const uint32_t* opbits, uint64_t n, uint64_t n_states,
                          uint64_t* children, uint32_t* child_ops, PuzzleArgs pz, unsigned long long* err,
                          bool use_opbits, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    const unsigned grid = unsigned((n + kThreads - 1) / kThreads);
    if (use_opbits)
        expand_batch_kernel<PZ, true><<<grid, kThreads, 0, s>>>(parents, opbits, n, n_states, children, child_ops,
                                                                pz, err);
    else
        expand_batch_kernel<PZ, false><<<grid, kThreads, 0, s>>>(parents, opbits, n, n_states, children, child_ops,
                                                                 pz, err);
    return cudaGetLastError();
}

template <class PZ>
PuzzleKernels make_kernels() {
    PuzzleKernels k;
    k.level[kThreeBit] = &launch_level<PZ, kThreeBit>;
    k.level[kClassic] = &launch_level<PZ, kClassic>;
    k.level[kTwoBit] = &launch_level<PZ, kTwoBit>;
    k.level[kFrontier] = &launch_level<PZ, kFrontier>;
    k.seed = &launch_seed<PZ>;
    k.expand = &launch_expand<PZ>;
    k.branching = PZ::kBranch;
    return k;
}

// Defined in psb_pancake.cu, psb_sliding.cu, psb_hanoi.cu.
bool pancake_kernels(int n, PuzzleKernels* out);
bool sliding_kernels(int cells, PuzzleKernels* out);
bool hanoi_kernels(PuzzleKernels* out);

}  // namespace psb
