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
#include <type_traits>

#include "psb_puzzles.cuh"

namespace psb {

constexpr int kThreads = 256;  // finalize and batched-expand kernels

enum Mode : int { kThreeBit = 0, kClassic = 1, kTwoBit = 2, kFrontier = 3 };

// Block shape of the level kernel per mode, chosen by a sweep on B200:
// two-bit top-down wants more resident warps (four 256-thread blocks per SM);
// three-bit's marks are fire-and-forget, and it runs fastest without a
// register cap.  Bottom-up levels wait on their probe loads, so they want
// resident warps too (four blocks per SM).
//
// Variants 1 and 2 of the top-down two-bit and three-bit kernels (the
// autotuner's threads-per-block dimension, psb_bfs_opts.threads): 512 and
// 128 threads per block.  For two-bit they also trade resident warps for
// registers: 128 per thread at 512 threads (one block per SM), 102 at 128
// threads (five blocks per SM; B200, whole searches: 13-pancake 213 ms
// against 226 ms with four blocks of 128 registers, 14-pancake 4.06 s
// against 4.15 s).  The 13- and 14-pancake kernels issue their far reads
// early and keep them in flight across the near children, which needs
// registers rather than warps (at 64 registers they spill).
template <int MODE, bool BU = false, int V = 0>
struct Shape {
    static constexpr int threads = V == 1 ? 512 : V == 2 ? 128 : 256;
    static constexpr int min_blocks = BU ? 4
                                    : MODE == kTwoBit ? (V == 1 ? 1 : V == 2 ? 5 : 4)
                                    : MODE == kFrontier ? 2
                                    : (V == 2 ? 2 : 1);
};
constexpr int kShapeVariants = 3;
__host__ __device__ constexpr int variant_threads(int v) { return v == 1 ? 512 : v == 2 ? 128 : 256; }

__host__ __device__ constexpr int level_threads(int mode) {
    return mode == kThreeBit ? Shape<kThreeBit>::threads
         : mode == kClassic  ? Shape<kClassic>::threads
         : mode == kTwoBit   ? Shape<kTwoBit>::threads
                             : Shape<kFrontier>::threads;
}

struct PuzzleArgs {
    int width;  // sliding tile: board width
    int disks;  // Hanoi: number of disks
    int sym;    // Hanoi: 0 no symmetry, 1 FourPegHanoiSimple's, 2 FourPegHanoiOptimized's (see Hanoi::expand)
};

// Adapters giving the three puzzles one device interface.  probe_range
// generates the children of one bottom-up probe round: the round starting at
// child `first` covers children first .. first+kProbeRound-1 in expansion order.
// kPairOp0: operator 0 maps state i to i ^ 1 (the pancake flip of the last
// two values only toggles the lowest Lehmer digit, of weight 1!), so a level
// kernel can mark those children for a whole frontier word at once and expand
// the rest with expand_from<1>.
// kChunkPrefix: the level kernel unranks the shared leading positions of a
// chunk's states once (make_prefix, two blocks of 7! indexes at most per
// chunk) and each state's remaining positions from index % 7!.
template <int N>
struct PancakeK {
    static constexpr int kBranch = N - 1;
    static constexpr int kOps = N - 1;
    static constexpr int kProbeRound = 4 < N - 1 ? 4 : N - 1;
    static constexpr bool kPairOp0 = true;
    static constexpr bool kFlip3Op1 = N >= 3;  // operator 1 permutes each aligned block of 6 (see flip3_push)
    static constexpr bool kFlip4Op2 = N >= 4;  // operator 2 permutes each aligned block of 24 (see flip4_pull)
    static constexpr bool kChunkPrefix = true;
    static constexpr bool kSymMult = false;
    static constexpr uint32_t kBlock = Pancake<N>::kBlock;
    using Prefix = typename Pancake<N>::Prefix;
    __device__ __forceinline__ static void make_prefix(uint32_t q, Prefix& P) { Pancake<N>::make_prefix(q, P); }
    template <int F, class E>
    __device__ __forceinline__ static void expand_from_prefixed(uint64_t i, const Prefix& P, uint32_t r, E& e) {
        Pancake<N>::template expand_prefixed<false>(i, P, r, 0u, F, N - 1, e);
    }
    template <class E>
    __device__ __forceinline__ static void probe_prefixed(uint64_t i, const Prefix& P, uint32_t r, int first,
                                                          int last, E& e) {
        Pancake<N>::template expand_prefixed<false>(i, P, r, 0u, first, last, e);
    }
    template <bool kOpBits, class E>
    __device__ __forceinline__ static void expand(uint64_t i, uint32_t ob, const PuzzleArgs&, E& e) {
        Pancake<N>::template expand<kOpBits>(i, ob, e);
    }
    template <int F, class E>
    __device__ __forceinline__ static void expand_from(uint64_t i, const PuzzleArgs&, E& e) {
        Pancake<N>::template expand_range<false>(i, 0u, F, N - 1, e);
    }
    template <class E>
    __device__ __forceinline__ static void probe_range(uint64_t i, int first, int last, const PuzzleArgs&, E& e) {
        Pancake<N>::template expand_range<false>(i, 0u, first, last, e);
    }
};
// PancakeOptimized (Puzzles/PancakeOptimized.cpp:26-139): the pancake moves
// in the reference's GPU pancake index, for n >= 12: (rank / 12!) << 29 |
// (rank % 12!), where rank is PancakeSimple's index; offsets >= 12! inside a
// 2^29 block name no permutation and have no children.  The level kernel
// runs it through the generic per-state path (no per-word flip tricks:
// their residue classes are those of the plain rank).
template <int N>
struct PancakeOptK {
    static constexpr int kBranch = N - 1;
    static constexpr int kOps = N - 1;
    static constexpr int kProbeRound = 4 < N - 1 ? 4 : N - 1;
    static constexpr bool kPairOp0 = false;
    static constexpr bool kFlip3Op1 = false;
    static constexpr bool kFlip4Op2 = false;
    static constexpr bool kChunkPrefix = false;
    static constexpr bool kSymMult = false;
    static constexpr uint32_t kBlock = 1;
    struct Prefix { uint32_t unused; };
    static constexpr uint64_t kF12 = 479001600ull;  // 12!
    __device__ __forceinline__ static bool to_rank(uint64_t i, uint64_t& r) {
        const uint64_t lo = i & ((uint64_t(1) << 29) - 1);
        if (lo >= kF12) return false;
        r = (i >> 29) * kF12 + lo;
        return true;
    }
    __device__ __forceinline__ static uint64_t from_rank(uint64_t r) { return ((r / kF12) << 29) | (r % kF12); }
    template <class E>
    struct Wrap {  // children come out as plain ranks; emit them in this index
        E& e;
        __device__ __forceinline__ void operator()(uint64_t c, uint32_t op) { e(from_rank(c), op); }
    };
    template <bool kOpBits, class E>
    __device__ __forceinline__ static void expand(uint64_t i, uint32_t ob, const PuzzleArgs&, E& e) {
        uint64_t r;
        if (!to_rank(i, r)) return;
        Wrap<E> w{e};
        Pancake<N>::template expand<kOpBits>(r, ob, w);
    }
    template <class E>
    __device__ __forceinline__ static void probe_range(uint64_t i, int first, int last, const PuzzleArgs&, E& e) {
        uint64_t r;
        if (!to_rank(i, r)) return;
        Wrap<E> w{e};
        Pancake<N>::template expand_range<false>(r, 0u, first, last, w);
    }
};

// SlidingTilePuzzleOptimized's index (see SlidingOpt); its moves have no
// per-word structure, so the level kernel runs the generic per-state path.
template <int N>
struct SlidingOptK {
    static constexpr int kBranch = 4;
    static constexpr int kOps = 4;
    static constexpr int kProbeRound = 4;  // one round: four cheap children
    static constexpr bool kPairOp0 = false;
    static constexpr bool kFlip3Op1 = false;
    static constexpr bool kFlip4Op2 = false;
    static constexpr bool kChunkPrefix = false;
    static constexpr bool kSymMult = false;
    static constexpr uint32_t kBlock = 1;
    struct Prefix { uint32_t unused; };
    template <bool kOpBits, class E>
    __device__ __forceinline__ static void expand(uint64_t i, uint32_t ob, const PuzzleArgs& a, E& e) {
        SlidingOpt<N>::template expand<kOpBits>(i, ob, a.width, e);
    }
    template <class E>
    __device__ __forceinline__ static void probe_range(uint64_t i, int, int, const PuzzleArgs& a, E& e) {
        SlidingOpt<N>::template expand<false>(i, 0u, a.width, e);
    }
};

template <int N>
struct SlidingK {
    static constexpr int kBranch = 4;
    static constexpr int kOps = 4;
    static constexpr int kProbeRound = 4;  // one round: four cheap children
    static constexpr bool kPairOp0 = false;
    static constexpr bool kFlip3Op1 = false;
    static constexpr bool kFlip4Op2 = false;
    static constexpr bool kChunkPrefix = false;
    static constexpr bool kSymMult = false;
    static constexpr uint32_t kBlock = 1;
    struct Prefix { uint32_t unused; };
    template <bool kOpBits, class E>
    __device__ __forceinline__ static void expand(uint64_t i, uint32_t ob, const PuzzleArgs& a, E& e) {
        Sliding<N>::template expand<kOpBits>(i, ob, a.width, e);
    }
    template <class E>
    __device__ __forceinline__ static void probe_range(uint64_t i, int, int, const PuzzleArgs& a, E& e) {
        Sliding<N>::template expand<false>(i, 0u, a.width, e);
    }
};
struct HanoiK {
    static constexpr int kBranch = 6;
    static constexpr int kOps = 4;
    static constexpr int kProbeRound = 6;  // one round: six cheap children
    static constexpr bool kPairOp0 = false;
    static constexpr bool kFlip3Op1 = false;
    static constexpr bool kFlip4Op2 = false;
    static constexpr bool kChunkPrefix = false;
    // With symmetry the index space holds one state per class of peg 1-3
    // permutations (pegs 1..3 ordered by their bottom disk).  The class size
    // is HanoiTowers::PegsMult (HanoiTowers/HanoiTowers.h:48-55): 6 when
    // pegs 1 and 2 hold disks, 3 when only peg 1 does (peg 1 empty leaves
    // only the all-on-peg-0 state, whose depth 0 the search counts as 1).
    static constexpr bool kSymMult = true;
    __device__ __forceinline__ static uint32_t sym_mult(uint64_t i) {
        const uint64_t hi = i >> 1, lo = i;
        const uint64_t peg1 = ~hi & lo & kEvenBits, peg2 = hi & ~lo & kEvenBits;
        return 6u - 3u * uint32_t(peg2 == 0) - uint32_t(peg1 == 0);
    }
    static constexpr uint64_t kEvenBits = 0x5555555555555555ull;
    static constexpr uint32_t kBlock = 1;
    struct Prefix { uint32_t unused; };
    template <bool kOpBits, class E>
    __device__ __forceinline__ static void expand(uint64_t i, uint32_t ob, const PuzzleArgs& a, E& e) {
        Hanoi::template expand<kOpBits>(i, ob, a.disks, a.sym, e);
    }
    template <class E>
    __device__ __forceinline__ static void probe_range(uint64_t i, int, int, const PuzzleArgs& a, E& e) {
        Hanoi::template expand<false>(i, 0u, a.disks, a.sym, e);
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
    unsigned long long* stats;  // [0] frontier (bottom-up: unvisited) states, [1] children (probes),
                                // [2] local children (bottom-up: found), [3] error flag, [5] two-bit next-frontier size,
                                // [6] two-bit far-bitmap marks, [7] class sizes of the frontier (sym_mult)
    const uint8_t* wflag_cur;   // optional: 1 byte per window, non-zero if the window may hold frontier states
    uint8_t* wflag_next;        // optional: set for every window that receives a mark this level
    const uint64_t* probe;      // bottom-up levels: the frontier array the unvisited states probe
    uint32_t* far;              // two-bit top-down, optional: 1 bit per state for long-range marks (see Emitter)
    int far_all;                // far != NULL: the far-reaching marks (Emitter::far) use it too
    int sym_mult;               // Hanoi with symmetry: add each frontier state's class size to stats[7]
    int flag_bits;              // non-zero: wflag_next has one byte per 2^flag_bits states (a bottom-up level's
                                // windows are larger than the top-down windows its flags serve); 0: window_bits
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

// L2 eviction-priority hints (PTX createpolicy / .L2::cache_hint, sm_80+).
// Far children (pancake flips of more than 12) land anywhere in the array and
// are never reused, so they are marked evict-first: they no longer displace
// the region that the flips of 9..12 keep hitting (a flip of m stays inside
// its aligned block of m! states).  13-pancake depth 11: 79 -> 72 ms.
__device__ __forceinline__ uint64_t l2_evict_first() {
    uint64_t p;
    asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
}
__device__ __forceinline__ void red_or_far(unsigned int* a, unsigned int v) {
    asm volatile("red.global.or.b32.L2::cache_hint [%0], %1, %2;" ::"l"(a), "r"(v), "l"(l2_evict_first())
                 : "memory");
}
__device__ __forceinline__ uint64_t ld_cg_far(const unsigned long long* a) {
    uint64_t v;
    asm volatile("ld.global.cg.L2::cache_hint.b64 %0, [%1], %2;" : "=l"(v) : "l"(a), "l"(l2_evict_first()));
    return v;
}
__device__ __forceinline__ uint64_t ld_nc_far(const uint64_t* a) {
    uint64_t v;
    asm("ld.global.nc.L2::cache_hint.b64 %0, [%1], %2;" : "=l"(v) : "l"(a), "l"(l2_evict_first()));
    return v;
}
__device__ __forceinline__ uint64_t ld_far(const uint64_t* a) {
    uint64_t v;
    asm volatile("ld.global.L2::cache_hint.b64 %0, [%1], %2;" : "=l"(v) : "l"(a), "l"(l2_evict_first()));
    return v;
}

// Shared-memory marks: one bit per state (1-bit modes) or four operator bits
// per state (frontier search).
__host__ __device__ constexpr size_t mark_bytes(int mode, size_t window_states) {
    return mode == kFrontier ? window_states / 2 : window_states / 8;
}

// Warp chunk: 32 lanes x one unit each (64 states; 32 for two-bit codes).
__host__ __device__ constexpr uint32_t states_per_unit(int mode) { return mode == kTwoBit ? 32 : 64; }
__host__ __device__ constexpr size_t list_entry_bytes(int mode) { return mode == kFrontier ? 4 : 2; }
constexpr size_t kWarpScratch = 256;  // per warp: the chunk's two unranking prefixes (kChunkPrefix)

// Dynamic shared memory of a level_window pass: window marks, then one list
// of a chunk's states per warp, then each warp's scratch.
__host__ __device__ constexpr size_t level_smem_bytes(int mode, size_t window_states, int threads) {
    return mark_bytes(mode, window_states) +
           size_t(threads / 32) * (32 * states_per_unit(mode) * list_entry_bytes(mode) + kWarpScratch);
}

// Pancake operator 1 (flip of the last three values) only changes the two
// lowest Lehmer digits: it maps index 6q + r to 6q + pi3(r) with
// pi3 = (5 3 4 1 2 0), an involution, and n! is a multiple of 6.  So for a
// unit of UW consecutive states (UW = 64 or 32, first state g*UW) the
// children of a frontier mask F are shifts of F by +5 (r = 0), +2 (r = 1, 2),
// -2 (r = 3, 4) and -5 (r = 5) under residue masks; bits shifted out of the
// unit belong to the neighbouring units.
__host__ __device__ constexpr uint64_t res6_mask(int phase, int r0, int r1, int width) {
    uint64_t m = 0;
    for (int b = 0; b < width; ++b)
        if ((phase + b) % 6 == r0 || (phase + b) % 6 == r1) m |= uint64_t(1) << b;
    return m;
}
template <int UW>
struct Res6 {  // residue masks of a unit whose first state is phase (mod 6)
    uint64_t m0, m12, m34, m5;
    __device__ __forceinline__ explicit Res6(uint64_t g) {  // g = global unit index
        // phase = (g * UW) mod 6, which depends on g mod 3 only
        constexpr int p1 = (UW % 6), p2 = (2 * UW) % 6;
        const uint32_t k = uint32_t(g % 3u);
        m0 = k == 0 ? res6_mask(0, 0, 0, UW) : k == 1 ? res6_mask(p1, 0, 0, UW) : res6_mask(p2, 0, 0, UW);
        m12 = k == 0 ? res6_mask(0, 1, 2, UW) : k == 1 ? res6_mask(p1, 1, 2, UW) : res6_mask(p2, 1, 2, UW);
        m34 = k == 0 ? res6_mask(0, 3, 4, UW) : k == 1 ? res6_mask(p1, 3, 4, UW) : res6_mask(p2, 3, 4, UW);
        m5 = k == 0 ? res6_mask(0, 5, 5, UW) : k == 1 ? res6_mask(p1, 5, 5, UW) : res6_mask(p2, 5, 5, UW);
    }
};
// Top-down: the operator-1 children of frontier mask F of unit g, split into
// the unit itself, the previous unit and the next one.
template <int UW>
__device__ __forceinline__ void flip3_push(uint64_t F, uint64_t g, uint64_t& prev, uint64_t& own, uint64_t& next) {
    const Res6<UW> m(g);
    const uint64_t p0 = F & m.m0, p12 = F & m.m12, p34 = F & m.m34, p5 = F & m.m5;
    constexpr uint64_t kLow = UW == 64 ? ~uint64_t(0) : 0xFFFFFFFFull;
    const uint64_t up = (p0 << 5) | (p12 << 2);  // UW = 32: bits above 31 overflow into the next unit
    own = (up | (p34 >> 2) | (p5 >> 5)) & kLow;
    if constexpr (UW == 64) {
        next = (p0 >> 59) | (p12 >> 62);
        prev = (p34 << 62) | (p5 << 59);
    } else {
        next = up >> 32;
        prev = ((p34 << 30) | (p5 << 27)) & kLow;
    }
}
// Bottom-up: the states of unit g whose operator-1 partner is in the
// frontier, from the frontier masks of units g-1, g and g+1.
template <int UW>
__device__ __forceinline__ uint64_t flip3_pull(uint64_t prevF, uint64_t F, uint64_t nextF, uint64_t g) {
    const Res6<UW> m(g);
    uint64_t up5, up2, dn2, dn5;  // bit b: frontier bit of state b+5, b+2, b-2, b-5
    if constexpr (UW == 64) {
        up5 = (F >> 5) | (nextF << 59);
        up2 = (F >> 2) | (nextF << 62);
        dn2 = (F << 2) | (prevF >> 62);
        dn5 = (F << 5) | (prevF >> 59);
    } else {
        const uint64_t x = (nextF << 32) | F, y = (F << 32) | prevF;
        up5 = (x >> 5) & 0xFFFFFFFFull;
        up2 = (x >> 2) & 0xFFFFFFFFull;
        dn2 = (y << 2) >> 32;
        dn5 = (y << 5) >> 32;
    }
    return (m.m0 & up5) | (m.m12 & up2) | (m.m34 & dn2) | (m.m5 & dn5);
}

// Pancake operator 2 (flip of the last four values) changes the three lowest
// Lehmer digits only: it maps index 24q + r to 24q + pi4(r), an involution
// (pi4 below is the Lehmer rank of the reversed arrangement of rank r), and
// n! is a multiple of 24 for n >= 4.  Bottom-up: the states of unit g whose
// operator-2 partner is in the frontier.  The residue masks are bits
// {0, 24, 48} of the unit shifted by (r - phase) mod 24.
// pi4 = (23 17 21 11 15 9 22 16 19 5 13 3 20 10 18 4 7 1 14 8 12 2 6 0), five bits per entry.
__host__ __device__ constexpr int pi4(int r) {
    return int(((r < 12 ? 0x1b4b38592f5d637ull >> (5 * r) : 0x184c4382724954ull >> (5 * (r - 12)))) & 31u);
}
template <int UW>
__device__ __forceinline__ uint64_t flip4_pull(uint64_t prevF, uint64_t F, uint64_t nextF, uint64_t g) {
    // phase = (g * UW) mod 24 depends on g mod 3 only
    constexpr int p1 = UW % 24, p2 = (2 * UW) % 24;
    const uint32_t k = uint32_t(g % 3u);
    const int phase = k == 0 ? 0 : k == 1 ? p1 : p2;
    const int t = phase == 0 ? 0 : 24 - phase;
    constexpr uint64_t kBase = UW == 64 ? 0x0001000001000001ull : 0x01000001ull;
    constexpr uint64_t kLow = UW == 64 ? ~uint64_t(0) : 0xFFFFFFFFull;
    uint64_t hit = 0;
#pragma unroll
    for (int r = 0; r < 24; ++r) {
        const int d = pi4(r) - r;  // partner offset, compile-time after unrolling
        int x = r + t;
        if (x >= 24) x -= 24;
        const uint64_t m = (kBase << x) & kLow;
        uint64_t sh;  // bit b: frontier bit of state b + d
        if constexpr (UW == 64) {
            sh = d > 0 ? (F >> d) | (nextF << ((64 - d) & 63)) : (F << -d) | (prevF >> ((64 + d) & 63));
        } else {
            sh = d > 0 ? (((nextF << 32) | F) >> d) & kLow : ((((F << 32) | prevF) << -d) >> 32);
        }
        hit |= m & sh;
    }
    return hit;
}

template <int MODE>
struct Emitter {
    uint64_t base;        // first state of the block's window
    uint32_t span;        // states of the window below n_states
    uint32_t* smarks;     // shared-memory window marks
    uint64_t* gmarks;     // global mark array
    uint64_t n_states;
    uint32_t next_pat;    // two-bit: bits of the NEXT code (hi at bit 0, lo at bit 1)
    uint8_t* wflag_next;  // optional active-window flags of the next level
    int window_bits;
    uint32_t* farbits;    // two-bit: long-range mark bitmap (NULL: read the target's code, then mark it)
    int far_all;          // the far-reaching marks (far()) go to farbits too; else they read first
    uint32_t children = 0, local = 0, bad = 0;
    uint32_t marked = 0;      // two-bit: long-range UNVISITED -> NEXT marks issued (two lanes may mark one state)
    uint32_t farmarks = 0;    // two-bit: marks set in the far bitmap
    uint32_t parent_off = 0;  // offset of the parent being expanded in the window (rel)

    // Records that window c >> window_bits receives a mark.  Most long-range
    // children land in windows already flagged, so the flag is read first:
    // storing every time made all SMs write the same few lines of a small
    // array (13-pancake depth 8: 2e8 stores, 11.7 ms).
    __device__ __forceinline__ void flag_window(uint64_t c) {
        if (!wflag_next) return;
        uint8_t* f = wflag_next + (c >> window_bits);
        if (!*f) *f = 1;
    }

    __device__ __forceinline__ void mark_local(uint32_t o, uint32_t op) {
        ++children;
        ++local;
        if constexpr (MODE == kFrontier) {
            atomicOr(&smarks[o >> 3], 1u << (4 * (o & 7u) + op));
        } else {
            atomicOr(&smarks[o >> 5], 1u << (o & 31u));
        }
    }

    template <bool kFar = false>
    __device__ __forceinline__ void mark_remote(uint64_t c, uint32_t op) {
        if (c >= n_states) { bad = 1; return; }  // never expected: keeps a bad index off the memory system
        ++children;
        if constexpr (MODE == kFrontier) {
            flag_window(c);
            atomicOr(reinterpret_cast<unsigned int*>(gmarks) + (c >> 3), 1u << (4 * (uint32_t(c) & 7u) + op));
        } else if constexpr (MODE == kTwoBit) {
            if (farbits && (!kFar || far_all)) {
                // Fire-and-forget: set the child's bit in the long-range
                // bitmap; fold_two_bit turns the UNVISITED ones into NEXT
                // after the level.  No dependent read of the target's code.
                flag_window(c);
                ++farmarks;
                if constexpr (kFar) red_or_far(farbits + (c >> 5), 1u << (uint32_t(c) & 31u));
                else atomicOr(farbits + (c >> 5), 1u << (uint32_t(c) & 31u));
                return;
            }
            unsigned long long* w = reinterpret_cast<unsigned long long*>(gmarks) + (c >> 5);
            const uint32_t sh = 2u * (uint32_t(c) & 31u);
            const uint64_t v = kFar ? ld_cg_far(w) : __ldcg(reinterpret_cast<const unsigned long long*>(w));
            if (((v >> sh) & 3u) == 0) {  // UNVISITED -> NEXT
                flag_window(c);
                atomicOr(w, (unsigned long long)next_pat << sh);
                ++marked;
            }
        } else {
            flag_window(c);
            unsigned int* w = reinterpret_cast<unsigned int*>(gmarks) + (c >> 5);
            if constexpr (kFar) red_or_far(w, 1u << (uint32_t(c) & 31u));
            else atomicOr(w, 1u << (uint32_t(c) & 31u));
        }
    }

    __device__ __forceinline__ void operator()(uint64_t c, uint32_t op) {
        const uint64_t o = c - base;
        if (o < span) mark_local(uint32_t(o), op);
        else mark_remote(c, op);
    }

    // A child anywhere in the index space (see EmitFar).
    __device__ __forceinline__ void far(uint64_t c, uint32_t op) {
        const uint64_t o = c - base;
        if (o < span) mark_local(uint32_t(o), op);
        else mark_remote<true>(c, op);
    }

    // The same in two steps (see EmitSplitFar): a two-bit mark that must
    // read its target first issues the read here and completes in
    // far_finish, after the parent's near children; every other mark is
    // made at once.
    __device__ __forceinline__ FarTicket far_issue(uint64_t c, uint32_t op) {
        const uint64_t o = c - base;
        if constexpr (MODE == kTwoBit) {
            if (o >= span && c < n_states && !(farbits && far_all))
                return FarTicket{ld_cg_far(reinterpret_cast<const unsigned long long*>(gmarks) + (c >> 5)), true};
        }
        far(c, op);
        return FarTicket{0, false};
    }
    __device__ __forceinline__ void far_finish(uint64_t c, uint32_t, const FarTicket& t) {
        if constexpr (MODE == kTwoBit) {
            if (!t.pending) return;
            ++children;
            if (((t.word >> (2u * (uint32_t(c) & 31u))) & 3u) == 0) {  // UNVISITED -> NEXT
                flag_window(c);
                atomicOr(reinterpret_cast<unsigned long long*>(gmarks) + (c >> 5),
                         (unsigned long long)next_pat << (2u * (uint32_t(c) & 31u)));
                ++marked;
            }
        }
    }

    // Child = parent + delta, with the parent at parent_off in the window.
    __device__ __forceinline__ void rel(uint64_t parent, int32_t delta, uint32_t op) {
        const uint32_t o = parent_off + uint32_t(delta);
        if (o < span) mark_local(o, op);
        else mark_remote(parent + int64_t(delta), op);
    }
};

// Bottom-up probe of one round: each child of an unvisited state that is in
// the frontier (three-bit `cur`, classic `open`: one bit per state; two-bit:
// code CUR) is a hit.  The probes of a round are independent loads, issued
// back to back; the state leaves the rounds at its first round with a hit.
// All three puzzles have symmetric moves (a flip, a slide or a disk move is
// undone by a move of the same puzzle), so "v has a frontier neighbour"
// equals "v is a child of a frontier state".
template <int MODE>
struct Probe {
    const uint64_t* front;
    uint64_t n_states;
    uint32_t cur_pat;  // two-bit: bits of the CUR code (hi at bit 0, lo at bit 1)
    bool hit = false;
    uint32_t probes = 0, bad = 0;

    template <bool kFar = false>
    __device__ __forceinline__ void probe(uint64_t c) {
        if (c >= n_states) { bad = 1; return; }
        ++probes;
        if constexpr (MODE == kTwoBit) {
            // Plain load: other blocks set NEXT bits in these words meanwhile,
            // which never changes a CUR code.
            const uint64_t w = kFar ? ld_far(front + (c >> 5)) : front[c >> 5];
            hit |= ((w >> (2u * (uint32_t(c) & 31u))) & 3u) == cur_pat;
        } else {
            // read-only during a bottom-up level
            const uint64_t w = kFar ? ld_nc_far(front + (c >> 6)) : __ldg(front + (c >> 6));
            hit |= ((w >> (uint32_t(c) & 63u)) & 1u) != 0;
        }
    }
    __device__ __forceinline__ void operator()(uint64_t c, uint32_t) { probe<false>(c); }
    __device__ __forceinline__ void far(uint64_t c, uint32_t) { probe<true>(c); }
};

// Shared variables of one window pass (a kernel's static shared memory).
struct WindowShared {
    uint32_t any;         // some warp found a frontier state in the window
    uint32_t next_chunk;  // chunks are handed out dynamically so warps finish together
    unsigned long long cnt[8];  // the window's counters (stats[0..7]), added to stats once per block
};

// One window of one level (see the top of this file).  KTHREADS threads of
// the block take part; smem64 is the block's dynamic shared memory.  The
// function ends with a block barrier, so a persistent kernel can call it for
// window after window.
//
// Bottom-up levels (BU = true; three-bit, classic and two-bit) turn the
// roles around: the sweep reads the visited information (three-bit: its
// visited array, classic: `closed`, two-bit: codes != UNVISITED), the list
// holds the window's UNVISITED states, and each probes its neighbours for a
// frontier state (Probe).  Found states are marked in the shared bitmap of
// their own window and flushed exactly as top-down marks are.  The probed
// arrays do not change during the level: two-bit's CUR -> OLD step runs
// afterwards (retire_two_bit), classic's clearing of `open` in
// finalize_classic_clear.
template <class PZ, int MODE, int KTHREADS, bool BU = false>
__device__ __forceinline__ void level_window(const LevelArgs& a, uint64_t window, unsigned long long* smem64,
                                             WindowShared& sh) {
    static_assert(!BU || MODE != kFrontier, "frontier search keeps no visited information");
    // Operator-0 children marked per frontier word in the sweep (see PancakeK);
    // bottom-up: unvisited states whose operator-0 neighbour is in the
    // frontier, found per word before any probing.
    constexpr bool kPairs = PZ::kPairOp0 && MODE != kFrontier && !BU;
    constexpr bool kBuPairs = PZ::kPairOp0 && BU;
    // three-bit / classic bottom-up pairs also read the unit's frontier word
    constexpr bool kProbeWord = kBuPairs && MODE != kTwoBit;
    // Operator-1 children (top-down) and hits (bottom-up) per unit as well
    // (flip3_push / flip3_pull); per-state expansion then starts at operator 2.
    constexpr bool kFlip3 = kPairs && PZ::kFlip3Op1;
    constexpr bool kBuFlip3 = kBuPairs && PZ::kFlip3Op1;
    // Bottom-up also finds operator-2 hits per unit (flip4_pull).
    constexpr bool kBuFlip4 = kBuFlip3 && PZ::kFlip4Op2;
    constexpr int kThreads = KTHREADS;
    constexpr int kWarps = kThreads / 32;
    constexpr uint32_t kSPU = states_per_unit(MODE);
    constexpr uint32_t kChunk = 32 * kSPU;           // states per warp chunk
    constexpr int kWPU = MODE == kFrontier ? 4 : 1;  // 64-bit frontier words per unit
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t W = 1u << a.window_bits;
    const uint64_t base = window << a.window_bits;
    if (base >= a.n_states) return;
    if (!BU && a.wflag_cur && !a.wflag_cur[window]) return;  // no frontier state can be in this window
    const uint64_t remaining = a.n_states - base;
    const uint32_t span = remaining < W ? uint32_t(remaining) : W;
    const uint32_t units = (span + kSPU - 1) / kSPU;
    const uint32_t chunks = (units + 31) / 32;
    const uint32_t mbytes = uint32_t(mark_bytes(MODE, W));
    uint32_t* smarks = reinterpret_cast<uint32_t*>(smem64);
    using Entry = typename std::conditional<MODE == kFrontier, uint32_t, uint16_t>::type;
    Entry* wlist = reinterpret_cast<Entry*>(reinterpret_cast<char*>(smem64) + mbytes) + size_t(warp) * kChunk;
    // Unranking prefixes of the chunk's (at most two) blocks of PZ::kBlock indexes.
    constexpr bool kPrefixed = PZ::kChunkPrefix && MODE != kFrontier;
    using Prefix = typename PZ::Prefix;
    static_assert(2 * sizeof(Prefix) <= kWarpScratch, "prefix scratch");
    Prefix* pref = reinterpret_cast<Prefix*>(reinterpret_cast<char*>(smem64) + mbytes +
                                             size_t(kWarps) * kChunk * sizeof(Entry) + size_t(warp) * kWarpScratch);

    for (uint32_t i = tid; i < mbytes / 16; i += kThreads) reinterpret_cast<uint4*>(smem64)[i] = make_uint4(0, 0, 0, 0);
    if (tid == 0) {
        sh.any = 0;
        sh.next_chunk = kWarps;  // chunks 0 .. kWarps-1 go to warps 0 .. kWarps-1
        for (int i = 0; i < 8; ++i) sh.cnt[i] = 0;
    }
    __syncthreads();

    Emitter<MODE> em{base, span, smarks, a.marks, a.n_states, 1u | (a.cur_code == 2 ? 2u : 0u), a.wflag_next,
                     a.window_bits, MODE == kTwoBit ? a.far : nullptr, a.far_all};
    uint32_t found = 0;
    // ORs a mask of unit x's states into the window's shared marks.
    auto mark_unit = [&](uint32_t x, uint64_t m) {
        if constexpr (kSPU == 64) {
            if (uint32_t(m)) atomicOr(&smarks[2 * x], uint32_t(m));
            if (uint32_t(m >> 32)) atomicOr(&smarks[2 * x + 1], uint32_t(m >> 32));
        } else {
            atomicOr(&smarks[x], uint32_t(m));
        }
    };
    // The CUR states of two-bit code word x (one bit per state).
    auto cur_states = [&](uint64_t x) -> uint64_t {
        const uint64_t hi = x & kEven, lo = (x >> 1) & kEven;
        return gather_even(hi & (a.cur_code == 3 ? lo : ~lo));
    };
    uint32_t probes = 0, hits = 0, pbad = 0;  // bottom-up counters
    uint32_t mult = 0;                         // sum of the frontier states' class sizes (sym_mult)

    // Each warp takes chunks on its own (its first chunk is its warp index,
    // later ones come from a shared counter): lane l sweeps unit 32*chunk + l,
    // the warp compacts the frontier states into its shared-memory list with a
    // shuffle scan and expands them, while the next chunk's words are already
    // in flight.  No block barrier until the flush.
    auto load = [&](uint32_t ch, uint64_t (&w)[kWPU]) {
        const uint32_t u = ch * 32 + uint32_t(lane);
#pragma unroll
        for (int q = 0; q < kWPU; ++q) {
            const uint64_t wi = MODE == kFrontier ? (base >> 4) + 4ull * u + q
                              : MODE == kTwoBit   ? (base >> 5) + u
                                                  : (base >> 6) + u;
            w[q] = (ch < chunks && u < units && wi < a.front_words) ? a.front[wi] : 0;
        }
    };
    auto load_probe = [&](uint32_t ch) -> uint64_t {
        const uint32_t u = ch * 32 + uint32_t(lane);
        return (kProbeWord && ch < chunks && u < units) ? __ldg(a.probe + (base >> 6) + u) : 0;
    };
    uint64_t cw[kWPU], nw[kWPU];
    uint32_t ch = uint32_t(warp);
    load(ch, cw);
    uint64_t cp = load_probe(ch), np = 0;
    while (ch < chunks) {  // uniform within the warp
        uint32_t nch = 0;
        if (lane == 0) nch = atomicAdd(&sh.next_chunk, 1u);
        nch = __shfl_sync(0xFFFFFFFFu, nch, 0);
        load(nch, nw);
        if constexpr (kProbeWord) np = load_probe(nch);
        const uint32_t u = ch * 32 + uint32_t(lane);
        uint64_t pmask = 0;
        if (BU && u < units) {
            // Unvisited states of the unit, restricted to indexes < n_states.
            const uint32_t left = span - u * kSPU;  // >= 1
            if constexpr (MODE == kTwoBit) {
                const uint64_t w = cw[0];
                pmask = gather_even(~(w | (w >> 1)) & kEven);
            } else {
                pmask = ~cw[0];
            }
            if (left < kSPU) pmask &= (uint64_t(1) << left) - 1u;
            if constexpr (kBuPairs) {
                uint64_t fw;  // the unit's frontier states
                if constexpr (MODE == kTwoBit) {
                    const uint64_t w = cw[0], hi = w & kEven, lo = (w >> 1) & kEven;
                    fw = gather_even(hi & (a.cur_code == 3 ? lo : ~lo));
                } else {
                    fw = cp;
                }
                const uint64_t hit2 = pmask & (((fw & kEven) << 1) | ((fw >> 1) & kEven));
                if (hit2) {
                    if constexpr (kSPU == 64) {
                        if (uint32_t(hit2)) atomicOr(&smarks[2 * u], uint32_t(hit2));
                        if (uint32_t(hit2 >> 32)) atomicOr(&smarks[2 * u + 1], uint32_t(hit2 >> 32));
                    } else {
                        atomicOr(&smarks[u], uint32_t(hit2));
                    }
                    hits += __popcll(hit2);
                    pmask &= ~hit2;
                }
                if (kBuFlip3 && pmask) {
                    // neighbouring units' frontier states (stable during a bottom-up level)
                    const uint64_t g = (MODE == kTwoBit ? (base >> 5) : (base >> 6)) + u;
                    uint64_t pf = 0, nf = 0;
                    if constexpr (MODE == kTwoBit) {
                        if (g > 0) pf = cur_states(a.front[g - 1]);
                        if (g + 1 < a.front_words) nf = cur_states(a.front[g + 1]);
                    } else {
                        if (g > 0) pf = __ldg(a.probe + g - 1);
                        if (g + 1 < a.front_words) nf = __ldg(a.probe + g + 1);
                    }
                    uint64_t hit3 = flip3_pull<kSPU>(pf, fw, nf, g);
                    if constexpr (kBuFlip4) hit3 |= flip4_pull<kSPU>(pf, fw, nf, g);
                    hit3 &= pmask;
                    if (hit3) {
                        mark_unit(u, hit3);
                        hits += __popcll(hit3);
                        pmask &= ~hit3;
                    }
                }
            }
        } else if (u < units) {
            if constexpr (MODE == kThreeBit) {
                pmask = cw[0];
            } else if constexpr (MODE == kClassic) {
                pmask = cw[0];
                if (pmask) a.front[(base >> 6) + u] = 0;  // BitArray::ScanBitsAndClear
            } else if constexpr (MODE == kTwoBit) {
                const uint64_t w = cw[0];
                const uint64_t hi = w & kEven, lo = (w >> 1) & kEven;
                const uint64_t cur = hi & (a.cur_code == 3 ? lo : ~lo);
                if (cur)  // CUR -> OLD (code 1); only this block changes this window's CUR codes
                    atomicXor(reinterpret_cast<unsigned long long*>(a.front) + (base >> 5) + u,
                              (unsigned long long)(cur | (a.cur_code == 2 ? (cur << 1) : 0)));
                pmask = gather_even(cur);
            } else {
                const uint64_t w0 = (base >> 4) + 4ull * u;
#pragma unroll
                for (int q = 0; q < kWPU; ++q) {
                    if (cw[q]) a.front[w0 + q] = 0;  // FourBitArray::ScanAndClear
                    pmask |= uint64_t(nibble_flags(cw[q])) << (16 * q);
                }
                if (a.odd) {
                    const uint64_t ex = a.excl_cur[(base >> 6) + u];
                    pmask &= ~ex;
                    a.excl_next[(base >> 6) + u] = pmask;
                }
            }
        }
        if constexpr (kPairs) {
            // children i ^ 1 of the unit's frontier states: swap adjacent bits
            const uint64_t pairs = ((pmask & kEven) << 1) | ((pmask >> 1) & kEven);
            if (pairs) {
                if constexpr (kSPU == 64) {
                    if (uint32_t(pairs)) atomicOr(&smarks[2 * u], uint32_t(pairs));
                    if (uint32_t(pairs >> 32)) atomicOr(&smarks[2 * u + 1], uint32_t(pairs >> 32));
                } else {
                    atomicOr(&smarks[u], uint32_t(pairs));
                }
                const uint32_t np = __popcll(pairs);
                em.children += np;
                em.local += np;
            }
        }
        if constexpr (kFlip3) {
            uint64_t pv, own, nx;
            flip3_push<kSPU>(pmask, (MODE == kTwoBit ? (base >> 5) : (base >> 6)) + u, pv, own, nx);
            if (own) {
                mark_unit(u, own);
                em.children += __popcll(own);
                em.local += __popcll(own);
            }
            // children in the neighbouring units: shared marks inside the
            // window, the emitter's long-range path outside it
            auto side = [&](uint64_t m, int64_t x) {
                if (!m) return;
                if (x >= 0 && x < int64_t(W / kSPU)) {
                    mark_unit(uint32_t(x), m);
                    em.children += __popcll(m);
                    em.local += __popcll(m);
                } else {
                    while (m) {
                        const uint32_t bit = __ffsll((long long)m) - 1;
                        m &= m - 1;
                        em(uint64_t(int64_t(base) + x * int64_t(kSPU) + bit), 1u);
                    }
                }
            };
            side(pv, int64_t(u) - 1);
            side(nx, int64_t(u) + 1);
        }
        const uint32_t cnt = __popcll(pmask);
        found += cnt;
        auto entry_of = [&](uint32_t j) -> Entry {
            const uint32_t ub = uint32_t(lane) * kSPU;
            if constexpr (MODE == kFrontier) {
                const uint64_t word = j < 16 ? cw[0 % kWPU] : j < 32 ? cw[1 % kWPU] : j < 48 ? cw[2 % kWPU] : cw[3 % kWPU];
                const uint32_t bits = uint32_t(word >> (4 * (j & 15))) & 15u;
                return Entry((ub + j) | (bits << 16));
            } else {
                return Entry(ub + j);
            }
        };
        uint32_t incl = cnt;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
            if (lane >= o) incl += y;
        }
        const uint32_t total = __shfl_sync(0xFFFFFFFFu, incl, 31);
        if (total) {
            uint32_t off = incl - cnt;
            while (pmask) {
                const uint32_t j = __ffsll((long long)pmask) - 1;
                pmask &= pmask - 1;
                wlist[off++] = entry_of(j);
            }
            __syncwarp();
            const uint64_t cbase = base + uint64_t(ch) * kChunk;
            uint32_t q0 = 0;  // block of the chunk's first state
            if constexpr (kPrefixed) {
                q0 = uint32_t(cbase / PZ::kBlock);
                if (lane < 2) PZ::make_prefix(q0 + uint32_t(lane), pref[lane]);
                __syncwarp();
            }
            // state p = q*kBlock + r with q = q0 or q0 + 1 (a chunk is shorter than a block)
            auto split = [&](uint64_t p, uint32_t& var) -> uint32_t {
                const uint32_t r0 = uint32_t(p - uint64_t(q0) * PZ::kBlock);
                var = r0 >= PZ::kBlock ? 1u : 0u;
                return r0 - var * PZ::kBlock;
            };
            if constexpr (BU) {
                // Probe rounds: the round starting at child `first` probes
                // children first .. first+R-1 of every state still listed;
                // states with a hit are marked, the rest are compacted in
                // place (ballot) for the next round, so every round keeps all
                // lanes busy whatever the hit pattern.
                // Pancake: the children left after the word-level flips in two
                // rounds (each round re-unranks the states still listed; 13-pancake
                // depth 12: 58 ms in 2 rounds of 5 against 65 ms in 3 rounds of 4).
                constexpr int kLeftChildren = PZ::kBranch - (kBuFlip4 ? 3 : kBuFlip3 ? 2 : kBuPairs ? 1 : 0);
                constexpr int R = PZ::kPairOp0 ? (kLeftChildren > 1 ? (kLeftChildren + 1) / 2 : 1) : PZ::kProbeRound;
                const uint32_t cur_pat = a.cur_code == 2 ? 1u : 3u;
                uint32_t left = total;
                constexpr int kFirst = kBuFlip4 ? 3 : kBuFlip3 ? 2 : kBuPairs ? 1 : 0;
                constexpr int kRounds = (PZ::kBranch - kFirst + R - 1) / R;
                for (int round = 0; round < kRounds && left; ++round) {
                    // children [lo, hi) of this round, ascending from kFirst
                    const int lo = kFirst + round * R;
                    const int hi = lo + R < PZ::kBranch ? lo + R : PZ::kBranch;
                    uint32_t kept = 0;
                    for (uint32_t e0 = 0; e0 < left; e0 += 32) {
                        const uint32_t e = e0 + uint32_t(lane);
                        bool miss = false;
                        Entry entry = 0;
                        if (e < left) {
                            entry = wlist[e];
                            const uint32_t o = uint32_t(ch) * kChunk + entry;  // offset in the window
                            Probe<MODE> pr{a.probe, a.n_states, cur_pat};
                            if constexpr (kPrefixed) {
                                uint32_t var;
                                const uint32_t r = split(base + o, var);
                                PZ::probe_prefixed(base + o, pref[var], r, lo, hi, pr);
                            } else {
                                PZ::probe_range(base + o, lo, hi, a.pz, pr);
                            }
                            probes += pr.probes;
                            pbad |= pr.bad;
                            if (pr.hit) {
                                ++hits;
                                atomicOr(&smarks[o >> 5], 1u << (o & 31u));
                            } else {
                                miss = true;
                            }
                        }
                        const uint32_t bal = __ballot_sync(0xFFFFFFFFu, miss);
                        // kept <= e0: the writes only reach entries this step has read
                        if (miss) wlist[kept + __popc(bal & ((1u << lane) - 1u))] = entry;
                        kept += __popc(bal);
                        __syncwarp();
                    }
                    left = kept;
                }
            } else
            for (uint32_t e = uint32_t(lane); e < total; e += 32) {
                if constexpr (MODE == kFrontier) {
                    const uint32_t v = wlist[e];
                    em.parent_off = ch * kChunk + (v & 0xFFFFu);
                    PZ::template expand<true>(cbase + (v & 0xFFFFu), v >> 16, a.pz, em);
                } else {
                    em.parent_off = ch * kChunk + wlist[e];
                    const uint64_t p = cbase + wlist[e];
                    if constexpr (PZ::kSymMult) {
                        if (a.sym_mult) mult += PZ::sym_mult(p);
                    }
                    if constexpr (kPrefixed) {
                        uint32_t var;
                        const uint32_t r = split(p, var);
                        PZ::template expand_from_prefixed<kFlip3 ? 2 : kPairs ? 1 : 0>(p, pref[var], r, em);
                    } else if constexpr (kPairs) {
                        PZ::template expand_from<kFlip3 ? 2 : 1>(p, a.pz, em);
                    } else {
                        PZ::template expand<false>(p, 0u, a.pz, em);
                    }
                }
            }
            __syncwarp();
        }
#pragma unroll
        for (int q = 0; q < kWPU; ++q) cw[q] = nw[q];
        cp = np;
        ch = nch;
    }
    if (BU ? hits != 0 : found != 0) sh.any = 1;
    __syncthreads();

    // Flush the window's shared-memory marks (only if it had frontier states).
    uint32_t fresh = 0;  // two-bit: states this flush moves from UNVISITED to NEXT
    if (sh.any) {
        if (a.wflag_next && tid == 0) {
            if (a.flag_bits) {  // every flag window this window overlaps (base + span <= n_states)
                for (uint64_t f = base >> a.flag_bits; f <= (base + span - 1) >> a.flag_bits; ++f) a.wflag_next[f] = 1;
            } else {
                a.wflag_next[window] = 1;
            }
        }
        if constexpr (MODE == kTwoBit) {
            const uint32_t next_pat = em.next_pat;
            unsigned long long* codes = reinterpret_cast<unsigned long long*>(a.marks) + (base >> 5);
            for (uint32_t i = tid; i < W / 32; i += kThreads) {
                const uint32_t v = smarks[i];
                if (!v || (base >> 5) + i >= a.mark_words) continue;
                const uint64_t w = __ldcg(codes + i);
                const uint64_t unvisited = ~(w | (w >> 1)) & kEven;
                const uint64_t m = spread_even(v) & unvisited;
                if (m) {
                    atomicOr(codes + i, (unsigned long long)(m | ((next_pat & 2u) ? (m << 1) : 0)));
                    fresh += __popcll(m);
                }
            }
        } else {
            constexpr uint32_t kShift = MODE == kFrontier ? 4 : 6;  // states per 64-bit word: 16 or 64
            unsigned long long* g = reinterpret_cast<unsigned long long*>(a.marks) + (base >> kShift);
            const uint32_t words = MODE == kFrontier ? W / 16 : W / 64;
            for (uint32_t i = tid; i < words; i += kThreads) {
                const unsigned long long v = smem64[i];
                if (v && (base >> kShift) + i < a.mark_words) {
                    atomicOr(g + i, v);
                    // three-bit bottom-up: the found states join the visited
                    // array here (only this block writes this window's words),
                    // so the level needs no finalize sweep
                    if constexpr (BU && MODE == kThreeBit) a.front[(base >> kShift) + i] |= v;
                }
            }
        }
    }

    // Counters: per warp into shared memory, then one global atomic per
    // block and counter (every warp of every window adding to the same few
    // global addresses would serialise at L2).
    uint32_t c0 = __reduce_add_sync(0xFFFFFFFFu, found);
    uint32_t c1 = __reduce_add_sync(0xFFFFFFFFu, BU ? probes : em.children);
    uint32_t c2 = __reduce_add_sync(0xFFFFFFFFu, BU ? hits : em.local);
    uint32_t c3 = __reduce_or_sync(0xFFFFFFFFu, BU ? pbad : em.bad);
    // Two-bit: size of the next frontier (exact for bottom-up levels, an
    // upper estimate otherwise); steers the choice of the next direction.
    uint32_t c5 = 0;
    uint32_t c6 = 0;  // two-bit: far-bitmap marks (the fold after the level has work only if some were made)
    if constexpr (MODE == kTwoBit) c5 = __reduce_add_sync(0xFFFFFFFFu, BU ? hits : em.marked + fresh);
    if constexpr (MODE == kTwoBit && !BU) c6 = __reduce_add_sync(0xFFFFFFFFu, em.farmarks);
    uint32_t c7 = 0;
    if constexpr (PZ::kSymMult && !BU) c7 = __reduce_add_sync(0xFFFFFFFFu, mult);
    if (lane == 0) {
        if (c5) atomicAdd(&sh.cnt[5], (unsigned long long)c5);
        if (c6) atomicAdd(&sh.cnt[6], (unsigned long long)c6);
        if (c7) atomicAdd(&sh.cnt[7], (unsigned long long)c7);
        if (c0) atomicAdd(&sh.cnt[0], (unsigned long long)c0);
        if (c1) atomicAdd(&sh.cnt[1], (unsigned long long)c1);
        if (c2) atomicAdd(&sh.cnt[2], (unsigned long long)c2);
        if (c3) atomicOr(&sh.cnt[3], 1ull);
    }
    __syncthreads();  // the shared marks and lists may be reused for another window
    if (tid == 0) {
        for (int i = 0; i < 8; ++i) {
            if (!sh.cnt[i] || i == 4) continue;
            if (i == 3) atomicOr(&a.stats[3], 1ull);
            else atomicAdd(&a.stats[i], sh.cnt[i]);
        }
    }
}

template <class PZ, int MODE, bool BU = false, int V = 0>
__global__ void __launch_bounds__(Shape<MODE, BU, V>::threads, Shape<MODE, BU, V>::min_blocks)
    level_kernel(LevelArgs a) {
    extern __shared__ __align__(16) unsigned long long smem64[];
    __shared__ WindowShared sh;
    level_window<PZ, MODE, Shape<MODE, BU, V>::threads, BU>(a, blockIdx.x, smem64, sh);
}

// Level 0 of frontier search (InMemoryFrontierSearch.cpp:81-88): expand the
// initial state with no used-operator bits.
template <class PZ>
__global__ void seed_kernel(LevelArgs a, uint64_t initial) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    Emitter<kFrontier> em{~uint64_t(0), 0, nullptr, a.marks, a.n_states, 0, a.wflag_next, a.window_bits, nullptr, 0};
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
// Segmented (out-of-core) search: expansion of one segment's states with a
// segment filter (the two halves of DB_Opt3BitBFS_Solver::Expand,
// Common/DiskBasedOptThreeBitBFS.cpp:73-137).  The states are the set bits
// of `bits` (segment-relative, words word_lo .. word_hi).
//   cross == 0: children inside the segment are ORed into `next` (RED);
//   cross == 1: children outside it are appended, as global indexes, to
//               `out` (warp-aggregated: one atomicAdd per converged group).
// ---------------------------------------------------------------------------
struct SegExpandArgs {
    const uint64_t* bits;  // the segment's states (bit i = state seg_base + i)
    uint64_t seg_base, seg_states;
    uint64_t word_lo, word_hi;
    uint64_t* next;             // cross == 0: the segment's next bitmap
    uint64_t* out;              // cross == 1: children outside the segment
    unsigned long long* out_n;  // cross == 1: entries appended (may exceed out_cap: overflow)
    uint64_t out_cap;
    uint64_t n_states;
    int cross;
    PuzzleArgs pz;
    unsigned long long* err;  // set when a child index is >= n_states
};

struct SegEmitter {
    const SegExpandArgs* a;
    uint32_t bad = 0;
    __device__ __forceinline__ void operator()(uint64_t c, uint32_t) {
        if (c >= a->n_states) { bad = 1; return; }
        const uint64_t o = c - a->seg_base;
        const bool inside = o < a->seg_states;
        if (!a->cross) {
            if (inside) atomicOr(reinterpret_cast<unsigned int*>(a->next) + (o >> 5), 1u << (uint32_t(o) & 31u));
            return;
        }
        if (inside) return;
        // the lanes that reach this point together share one atomicAdd
        const uint32_t mask = __activemask();
        const int lane = int(threadIdx.x & 31);
        const int leader = __ffs(mask) - 1;
        const uint32_t rank = __popc(mask & ((1u << lane) - 1u));
        unsigned long long base = 0;
        if (lane == leader) base = atomicAdd(a->out_n, (unsigned long long)__popc(mask));
        base = __shfl_sync(mask, base, leader);
        if (base + rank < a->out_cap) a->out[base + rank] = c;
    }
};

// Position of the k-th (0-based) set bit of v (k < popc(v)).
__device__ __forceinline__ uint32_t select_bit(uint64_t v, uint32_t k) {
    uint32_t pos = 0, w = uint32_t(v), c = __popc(w);
    if (k >= c) { k -= c; w = uint32_t(v >> 32); pos = 32; }
    c = __popc(w & 0xFFFFu); if (k >= c) { k -= c; w >>= 16; pos += 16; }
    c = __popc(w & 0xFFu);   if (k >= c) { k -= c; w >>= 8;  pos += 8; }
    c = __popc(w & 0xFu);    if (k >= c) { k -= c; w >>= 4;  pos += 4; }
    c = __popc(w & 0x3u);    if (k >= c) { k -= c; w >>= 2;  pos += 2; }
    return pos + ((k >= (w & 1u)) ? 1u : 0u);
}

// Each warp takes 32 consecutive words of the segment bitmap and expands
// their set bits 32 at a time, one state per lane: the lanes of a dense word
// share its states instead of one thread walking all 64.
template <class PZ>
__global__ void __launch_bounds__(kThreads) segment_expand_kernel(SegExpandArgs a) {
    SegEmitter em{&a};
    const uint32_t lane = threadIdx.x & 31u;
    const uint64_t warp = (uint64_t(blockIdx.x) * kThreads + threadIdx.x) >> 5;
    const uint64_t warps = (uint64_t(gridDim.x) * kThreads) >> 5;
    for (uint64_t w0 = a.word_lo + warp * 32; w0 < a.word_hi; w0 += warps * 32) {
        const uint64_t w = w0 + lane;
        const uint64_t v = w < a.word_hi ? a.bits[w] : 0;
        const uint32_t c = __popcll(v);
        uint32_t incl = c;  // inclusive prefix of the lanes' set bits
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
            if (lane >= uint32_t(o)) incl += y;
        }
        const uint32_t total = __shfl_sync(0xFFFFFFFFu, incl, 31);
        for (uint32_t base = 0; base < total; base += 32) {
            const uint32_t k = base + lane;
            // source lane: the first whose inclusive prefix exceeds k
            uint32_t lo = 0, hi = 31;
#pragma unroll
            for (int step = 0; step < 5; ++step) {
                const uint32_t mid = (lo + hi) >> 1;
                const uint32_t im = __shfl_sync(0xFFFFFFFFu, incl, int(mid));
                if (im > k) hi = mid;
                else lo = mid + 1;
            }
            const uint32_t before = __shfl_sync(0xFFFFFFFFu, incl - c, int(lo));
            const uint64_t word = __shfl_sync(0xFFFFFFFFu, v, int(lo));
            if (k < total) {
                const uint64_t i = (w0 + lo) * 64 + select_bit(word, k - before);
                if (i < a.seg_states) PZ::template expand<false>(a.seg_base + i, 0u, a.pz, em);
            }
        }
    }
    if (em.bad) atomicOr(a.err, 1ull);
}

// ---------------------------------------------------------------------------
// Launch helpers and per-puzzle dispatch tables.
// ---------------------------------------------------------------------------
using LevelLaunch = cudaError_t (*)(const LevelArgs&, unsigned grid, size_t smem, cudaStream_t);
using SeedLaunch = cudaError_t (*)(const LevelArgs&, uint64_t initial, cudaStream_t);
using ExpandLaunch = cudaError_t (*)(const uint64_t*, const uint32_t*, uint64_t, uint64_t, uint64_t*, uint32_t*,
                                     PuzzleArgs, unsigned long long*, bool, cudaStream_t);

using SegExpandLaunch = cudaError_t (*)(const SegExpandArgs&, unsigned grid, cudaStream_t);

struct PuzzleKernels {
    LevelLaunch level[4];     // indexed by Mode
    LevelLaunch level_bu[4];  // bottom-up levels, indexed by Mode (none for frontier search)
    LevelLaunch level_shape[kShapeVariants][4];  // top-down levels in shape variant v (two-bit, three-bit)
    SeedLaunch seed;
    ExpandLaunch expand;
    SegExpandLaunch segment_expand;
    int branching;
};

template <class PZ>
cudaError_t launch_segment_expand(const SegExpandArgs& a, unsigned grid, cudaStream_t s) {
    segment_expand_kernel<PZ><<<grid, kThreads, 0, s>>>(a);
    return cudaGetLastError();
}

template <class PZ, int MODE, bool BU = false, int V = 0>
cudaError_t launch_level(const LevelArgs& a, unsigned grid, size_t smem, cudaStream_t s) {
    cudaError_t e = cudaFuncSetAttribute(level_kernel<PZ, MODE, BU, V>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    if (e != cudaSuccess) return e;
    level_kernel<PZ, MODE, BU, V><<<grid, Shape<MODE, BU, V>::threads, smem, s>>>(a);
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
    k.level_bu[kThreeBit] = &launch_level<PZ, kThreeBit, true>;
    k.level_bu[kClassic] = &launch_level<PZ, kClassic, true>;
    k.level_bu[kTwoBit] = &launch_level<PZ, kTwoBit, true>;
    k.level_bu[kFrontier] = nullptr;
    for (auto& row : k.level_shape)
        for (auto& f : row) f = nullptr;
    k.level_shape[0][kThreeBit] = &launch_level<PZ, kThreeBit>;
    k.level_shape[0][kTwoBit] = &launch_level<PZ, kTwoBit>;
    k.level_shape[1][kThreeBit] = &launch_level<PZ, kThreeBit, false, 1>;
    k.level_shape[1][kTwoBit] = &launch_level<PZ, kTwoBit, false, 1>;
    k.level_shape[2][kThreeBit] = &launch_level<PZ, kThreeBit, false, 2>;
    k.level_shape[2][kTwoBit] = &launch_level<PZ, kTwoBit, false, 2>;
    k.seed = &launch_seed<PZ>;
    k.expand = &launch_expand<PZ>;
    k.segment_expand = &launch_segment_expand<PZ>;
    k.branching = PZ::kBranch;
    return k;
}

// Defined in psb_pancake.cu, psb_sliding.cu, psb_hanoi.cu.
bool pancake_kernels(int n, PuzzleKernels* out);
bool pancake_opt_kernels(int n, PuzzleKernels* out);  // psb_pancake_opt.cu, n = 12..16
bool sliding_kernels(int cells, PuzzleKernels* out);
bool sliding_opt_kernels(int cells, PuzzleKernels* out);  // psb_sliding_opt.cu: 4, 6, 8, 9, 10, 12, 14, 15, 16 cells
bool hanoi_kernels(PuzzleKernels* out);

}  // namespace psb
