// psb_puzzles.cuh -- device-side state codecs and expanders for the three
// puzzles of the reference (lightln2/PuzzleSearch), in the index spaces of its
// *Simple classes, so that every index, child and operator code is identical
// to the reference's CPU path.
//
//   sliding tile : Puzzles/SlidingTilePuzzleSimple.cpp  (n! permutation index)
//   pancake      : Puzzles/PancakeSimple.cpp            (n! permutation index, suffix reversal)
//   4-peg Hanoi  : Puzzles/FourPegHanoiSimple.cpp       (2 bits per disk)
//
// Permutation index (Puzzles/PermutationMap.cpp:39-58): position 0 is the
// most significant digit; digit i equals the number of later values smaller
// than the value at i; index = sum_i d_i * (n-1-i)!.  Everything is
// templated on n so all radices and factorial weights are compile-time
// constants: divisions become multiply-high sequences and the value arrays
// stay in registers.
#pragma once

#include <cstdint>
#include <type_traits>

namespace psb {

constexpr uint64_t kInvalidIndex = ~uint64_t(0);  // Common/Puzzle.h:19

// Emitters with a member rel(parent, delta, op) take a child given as its
// parent's index plus a signed 32-bit delta (see Pancake); others get the
// child's index.
template <class E, class = void>
struct EmitRel : std::false_type {};
template <class E>
struct EmitRel<E, decltype(void(&E::rel))> : std::true_type {};

// Emitters with a member far(child, op) take children that can land anywhere
// in a large index space (pancake flips of more than 12) there, so they can
// mark them without displacing cached data that nearer children reuse.
template <class E, class = void>
struct EmitFar : std::false_type {};
template <class E>
struct EmitFar<E, decltype(void(&E::far))> : std::true_type {};

// Emitters with members far_issue(child, op) and far_finish(child, op, ticket)
// take the far children in two steps: the first starts whatever the mark
// has to read and returns a ticket, the second completes the mark.  The
// expander issues the far children first and finishes them after the near
// ones, so the reads overlap the near children's arithmetic.
template <class E, class = void>
struct EmitSplitFar : std::false_type {};
template <class E>
struct EmitSplitFar<E, decltype(void(&E::far_issue))> : std::true_type {};

struct FarTicket {
    uint64_t word;  // the target's code word, when `pending`
    bool pending;
};

__host__ __device__ constexpr uint64_t fact(int k) { return k <= 1 ? 1 : uint64_t(k) * fact(k - 1); }
constexpr uint32_t kF12 = 479001600u;  // 12!

// Lehmer digits of a permutation index.  Digits with weight < 12! come from
// the low 32-bit part; the (at most four) top digits of n > 12 from the quotient.
template <int N>
__device__ __forceinline__ void perm_digits(uint64_t index, uint32_t (&d)[N]) {
    uint32_t lo, hi = 0;
    if constexpr (N <= 12) {
        lo = uint32_t(index);
    } else {
        hi = uint32_t(index / kF12);
        lo = uint32_t(index - uint64_t(hi) * kF12);
    }
#pragma unroll
    for (int i = N - 1; i >= 0; --i) {
        const uint32_t radix = uint32_t(N - i);
        if (N - 1 - i < 12) {
            d[i] = lo % radix;
            lo /= radix;
        } else {
            d[i] = hi % radix;
            hi /= radix;
        }
    }
}

// PermutationUncompact (PermutationMap.cpp:21-37): digit k picks the k-th
// unused value from a nibble list.
template <int N>
__device__ __forceinline__ void perm_values(const uint32_t (&d)[N], uint32_t (&v)[N]) {
    uint64_t tiles = 0xFEDCBA9876543210ull;
#pragma unroll
    for (int i = 0; i < N; ++i) {
        const uint32_t s = 4u * d[i];
        v[i] = uint32_t(tiles >> s) & 15u;
        const uint64_t lo = tiles & ((uint64_t(1) << s) - 1);
        const uint64_t hi = ((tiles >> s) >> 4) << s;
        tiles = hi | lo;
    }
}

// PermutationRank via "smaller values to the right" counts.
template <int N>
__device__ __forceinline__ uint64_t perm_rank(const uint32_t (&v)[N]) {
    uint32_t seen = 0, lo = 0, hi = 0;
#pragma unroll
    for (int i = N - 1; i >= 0; --i) {
        const uint32_t dig = __popc(seen & ((1u << v[i]) - 1u));
        seen |= 1u << v[i];
        const int w = N - 1 - i;
        if (w < 12) lo += dig * uint32_t(fact(w));
        else hi += dig * uint32_t(fact(w) / kF12);
    }
    return uint64_t(hi) * kF12 + lo;
}

// Rank of a nibble-packed permutation (nibble i = value at position i).
template <int N>
__device__ __forceinline__ uint64_t perm_rank_packed(uint64_t p) {
    uint32_t v[N];
#pragma unroll
    for (int i = 0; i < N; ++i) v[i] = uint32_t(p >> (4 * i)) & 15u;
    return perm_rank<N>(v);
}

// --------------------------------------------------------------------------
// Pancake (PancakeSimple.cpp:12-20,62-73): operator k reverses the LAST k+2
// values; the child's operator code is k.  Only the last m = k+2 Lehmer
// digits change, so child = parent - low_m(parent) + low_m(child), where
// low_m(child) = sum_{q<m} q! * #(earlier values of the parent suffix that
// are smaller than the parent value at position n-m+q).
// --------------------------------------------------------------------------
template <int N>
struct Pancake {
    static constexpr int kBranch = N - 1;
    static constexpr int kOps = N - 1;

    // Chunk-shared unranking.  Digit i has weight (n-1-i)!, so the first
    // kL = n-7 positions of an index depend only on index / 7!: every index
    // of a block of 7! = 5040 consecutive indexes shares them.  A Prefix holds
    // those positions (digits, pre, pb) and the other 7 values as a 32-bit
    // nibble list; unrank_suffix completes a state from index % 7!.
    static constexpr int kL = N > 7 ? N - 7 : 0;
    static constexpr uint32_t kBlock = 5040;  // 7!
    struct Prefix {
        uint32_t d[kL > 0 ? kL : 1], pre[kL > 0 ? kL : 1], pb[kL > 0 ? kL : 1];
        uint32_t acc;     // values at positions < kL, one bit each
        uint32_t tiles7;  // the other 7 values, ascending, one nibble each
    };

    // Lehmer digits d, and for each position j: pre[j] = values left of j,
    // pb[j] = those of them smaller than v[j] (one bit per value).
    __device__ __forceinline__ static void unrank(uint64_t index, uint32_t (&d)[N], uint32_t (&pre)[N],
                                                  uint32_t (&pb)[N]) {
        uint32_t v[N];
        perm_digits<N>(index, d);
        perm_values<N>(d, v);
        uint32_t acc = 0;
#pragma unroll
        for (int i = 0; i < N; ++i) {
            pre[i] = acc;
            pb[i] = acc & ((1u << v[i]) - 1u);
            acc |= 1u << v[i];
        }
    }

    // Prefix of the indexes in [q*7!, (q+1)*7!); q < n!/7! <= 16!/7! < 2^32.
    __device__ __forceinline__ static void make_prefix(uint32_t q, Prefix& P) {
        if constexpr (kL > 0) {
            uint32_t d[kL];
#pragma unroll
            for (int i = kL - 1; i >= 0; --i) {
                d[i] = q % uint32_t(N - i);
                q /= uint32_t(N - i);
            }
            uint64_t tiles = 0xFEDCBA9876543210ull;
            uint32_t acc = 0;
#pragma unroll
            for (int i = 0; i < kL; ++i) {
                const uint32_t s = 4u * d[i];
                const uint32_t v = uint32_t(tiles >> s) & 15u;
                tiles = (((tiles >> s) >> 4) << s) | (tiles & ((uint64_t(1) << s) - 1));
                P.d[i] = d[i];
                P.pre[i] = acc;
                P.pb[i] = acc & ((1u << v) - 1u);
                acc |= 1u << v;
            }
            P.acc = acc;
            P.tiles7 = uint32_t(tiles) & 0x0FFFFFFFu;
        } else {
            P.acc = 0;
            P.tiles7 = 0x06543210u;
        }
    }

    // State of index q*7! + r from its block's prefix (r < 7!).
    __device__ __forceinline__ static void unrank_suffix(const Prefix& P, uint32_t r, uint32_t (&d)[N],
                                                         uint32_t (&pre)[N], uint32_t (&pb)[N]) {
#pragma unroll
        for (int i = 0; i < kL; ++i) {
            d[i] = P.d[i];
            pre[i] = P.pre[i];
            pb[i] = P.pb[i];
        }
#pragma unroll
        for (int i = N - 1; i >= kL; --i) {
            d[i] = r % uint32_t(N - i);
            r /= uint32_t(N - i);
        }
        uint32_t t = P.tiles7, acc = P.acc;
#pragma unroll
        for (int i = kL; i < N; ++i) {
            const uint32_t s = 4u * d[i];
            const uint32_t v = (t >> s) & 15u;
            t = ((t >> s) >> 4 << s) | (t & ((1u << s) - 1u));
            pre[i] = acc;
            pb[i] = acc & ((1u << v) - 1u);
            acc |= 1u << v;
        }
    }

    template <bool kOpBits, class Emit>
    __device__ __forceinline__ static void expand(uint64_t index, uint32_t opbits, Emit& emit) {
        expand_range<kOpBits>(index, opbits, 0, N - 1, emit);
    }

    // Only the children with operator in [first, last) (bottom-up probe rounds).
    template <bool kOpBits, class Emit>
    __device__ __forceinline__ static void expand_range(uint64_t index, uint32_t opbits, int first, int last,
                                                        Emit& emit) {
        uint32_t d[N], pre[N], pb[N];
        unrank(index, d, pre, pb);
        children<kOpBits>(index, d, pre, pb, opbits, first, last, emit);
    }

    // expand_range for index = q*7! + r, with P = make_prefix(q).
    template <bool kOpBits, class Emit>
    __device__ __forceinline__ static void expand_prefixed(uint64_t index, const Prefix& P, uint32_t r,
                                                           uint32_t opbits, int first, int last, Emit& emit) {
        uint32_t d[N], pre[N], pb[N];
        unrank_suffix(P, r, d, pre, pb);
        children<kOpBits>(index, d, pre, pb, opbits, first, last, emit);
    }

    // Rank of the child of flip m: with pre = the values left of the suffix
    // (positions < n-m) and pb[j] = the values left of position j that are
    // smaller than v[j], the count above is popc(pb[j] & ~pre).  For m <= 12
    // every quantity is below 12! < 2^31, so the child is passed to emitters
    // that take it (EmitRel) as the parent plus a 32-bit signed delta.
    template <bool kOpBits, class Emit>
    __device__ __forceinline__ static void children(uint64_t index, const uint32_t (&d)[N], const uint32_t (&pre)[N],
                                                    const uint32_t (&pb)[N], uint32_t opbits, int first, int last,
                                                    Emit& emit) {
        // Far children first, for emitters that take them in two steps.
        constexpr bool kSplit = EmitSplitFar<Emit>::value && (N > 12);
        constexpr int kFarN = N > 12 ? N - 12 : 1;
        uint64_t far_child[kFarN];
        FarTicket far_ticket[kFarN];
        if constexpr (kSplit) {
            uint64_t low = 0;
#pragma unroll
            for (int m = 2; m <= N; ++m) {
                low += uint64_t(d[N - m]) * fact(m - 1);
                if (m <= 12) continue;
                const int op = m - 2, k = m - 13;
                far_ticket[k].pending = false;
                if (op < first || op >= last || (kOpBits && (opbits >> op) & 1u)) {
                    far_child[k] = kInvalidIndex;
                    continue;
                }
                const uint32_t excl = pre[N - m];
                uint32_t s32 = 0, t = 0;
#pragma unroll
                for (int q = 1; q < m; ++q) {
                    const uint32_t c = __popc(pb[N - m + q] & ~excl);
                    if (q < 12) s32 += uint32_t(fact(q)) * c;
                    else t += uint32_t(fact(q) / kF12) * c;
                }
                far_child[k] = index - low + (uint64_t(t) * kF12 + s32);
                far_ticket[k] = emit.far_issue(far_child[k], uint32_t(op));
            }
        }
        uint32_t low32 = 0;  // low_m for m <= 12 (d[n-1] is always 0)
        uint64_t low64 = 0;  // low_m for m > 12
#pragma unroll
        for (int m = 2; m <= N; ++m) {
            if (kSplit && m > 12) break;
            if (m <= 12) low32 += d[N - m] * uint32_t(fact(m - 1));
            else low64 = (m == 13 ? uint64_t(low32) : low64) + uint64_t(d[N - m]) * fact(m - 1);
            const int op = m - 2;
            if (op >= last) break;
            if (op < first || (kOpBits && (opbits >> op) & 1u)) continue;
            const uint32_t excl = pre[N - m];
            if (m <= 12) {  // m is a compile-time constant after unrolling
                uint32_t s32 = 0;
#pragma unroll
                for (int q = 1; q < m; ++q) s32 += uint32_t(fact(q)) * __popc(pb[N - m + q] & ~excl);
                const int32_t delta = int32_t(s32 - low32);
                if constexpr (EmitRel<Emit>::value) emit.rel(index, delta, uint32_t(op));
                else emit(index + int64_t(delta), uint32_t(op));
            } else {
                uint32_t s32 = 0, t = 0;
#pragma unroll
                for (int q = 1; q < m; ++q) {
                    const uint32_t c = __popc(pb[N - m + q] & ~excl);
                    if (q < 12) s32 += uint32_t(fact(q)) * c;
                    else t += uint32_t(fact(q) / kF12) * c;
                }
                const uint64_t child = index - low64 + (uint64_t(t) * kF12 + s32);
                if constexpr (EmitFar<Emit>::value) emit.far(child, uint32_t(op));
                else emit(child, uint32_t(op));
            }
        }
        if constexpr (kSplit) {
#pragma unroll
            for (int k = 0; k < N - 12; ++k)
                if (far_child[k] != kInvalidIndex) emit.far_finish(far_child[k], uint32_t(k + 11), far_ticket[k]);
        }
    }
};

// --------------------------------------------------------------------------
// Sliding tile (SlidingTilePuzzleSimple.cpp:8,61-99): operators UP=0, LEFT=1,
// RIGHT=2, DOWN=3; children in the order up, down, left, right; each child
// carries the operator that moves the blank back.
// --------------------------------------------------------------------------
template <int N>
struct Sliding {
    static constexpr int kBranch = 4;
    static constexpr int kOps = 4;

    template <bool kOpBits, class Emit>
    __device__ __forceinline__ static void expand(uint64_t index, uint32_t opbits, int width, Emit& emit) {
        uint32_t d[N], v[N];
        perm_digits<N>(index, d);
        perm_values<N>(d, v);
        uint64_t packed = 0;
        int blank = 0;
#pragma unroll
        for (int i = 0; i < N; ++i) {
            packed |= uint64_t(v[i]) << (4 * i);
            if (v[i] == 0) blank = i;
        }
        const int col = blank % width;
        auto child = [&](int t) -> uint64_t {
            const uint64_t tile = (packed >> (4 * t)) & 15u;
            const uint64_t p = packed + (tile << (4 * blank)) - (tile << (4 * t));
            return perm_rank_packed<N>(p);
        };
        if (blank >= width && !(kOpBits && (opbits & 1u))) emit(child(blank - width), 3u);
        if (blank < N - width && !(kOpBits && (opbits & 8u))) emit(child(blank + width), 0u);
        if (col > 0 && !(kOpBits && (opbits & 2u))) emit(child(blank - 1), 2u);
        if (col < width - 1 && !(kOpBits && (opbits & 4u))) emit(child(blank + 1), 1u);
    }
};

// --------------------------------------------------------------------------
// Sliding tile in SlidingTilePuzzleOptimized's index
// (Puzzles/SlidingTilePuzzleOptimized.cpp:99-236; GPU expand
// kernel_sliding_tile_optimized, Puzzles/SlidingPuzzleGpu.cu:211-269).  The
// board's T = N-1 tiles in board order, the blank left out; digit i of tile
// i (i >= 2) = how many earlier tiles are smaller.  Digit 0 is always 0 and
// digit 1 follows from the parity rule (:79-97), so neither is stored.  Low
// 32 bits: blank + 16 * sum_{i=2..11} d_i * i!/2; bits 32 and up (14..16
// cells): d_12 | d_13 << 4 | d_14 << 8.  Moving the blank up or down rotates
// the tiles between the two blank positions by one place; moving it left or
// right only changes the blank digit (index -+ 1).
// --------------------------------------------------------------------------
template <int N>
struct SlidingOpt {
    static constexpr int kBranch = 4;
    static constexpr int kOps = 4;
    static constexpr int T = N - 1;                    // tiles
    static constexpr int kTop = T - 1 < 11 ? T - 1 : 11;  // last digit of the low word
    static_assert(N >= 4 && N <= 16, "2x2 .. 4x4 boards");

    // The tiles (values 0..T-1, list position i in nibble i) and blank of an
    // index; false when the index names no board.
    __device__ __forceinline__ static bool board(uint64_t index, int width, uint64_t& tiles, uint32_t& blank) {
        blank = uint32_t(index) & 15u;
        if (blank >= uint32_t(N)) return false;
        uint32_t d[16];
        uint32_t low = uint32_t(index) >> 4;
#pragma unroll
        for (int i = 2; i <= kTop; ++i) {
            d[i] = low % uint32_t(i + 1);
            low /= uint32_t(i + 1);
        }
        if (low) return false;
        uint64_t seg = index >> 32;
#pragma unroll
        for (int i = 12; i < T; ++i) {
            d[i] = uint32_t(seg) & 15u;
            seg >>= 4;
            if (d[i] > uint32_t(i)) return false;
        }
        if (seg) return false;
        // Values, last tile first: d_i picks among the values still unused
        // (ascending in a nibble list; the first i+1 entries are the unused ones).
        uint64_t left = 0xFEDCBA9876543210ull;
        uint32_t odd = 1;  // inversions of the tile list with d_1 = 0: sum (i - d_i) + 1
        tiles = 0;
#pragma unroll
        for (int i = T - 1; i >= 2; --i) {
            const uint32_t s = 4u * d[i];
            tiles |= ((left >> s) & 15u) << (4 * i);
            left = (((left >> s) >> 4) << s) | (left & ((uint64_t(1) << s) - 1));
            odd += uint32_t(i) - d[i];
        }
        const uint32_t lo = uint32_t(left) & 15u, hi = (uint32_t(left) >> 4) & 15u;
        if (width % 2 == 0) odd += blank / uint32_t(width);
        // d_1 = 0 puts the larger of the last two values first; the other
        // parity class swaps them (Unpack, :133-137)
        tiles |= (odd & 1u) ? uint64_t(lo | (hi << 4)) : uint64_t(hi | (lo << 4));
        return true;
    }

    // Index of tiles / blank (Pack + GetIndex, :99-158).
    __device__ __forceinline__ static uint64_t index_of(uint64_t tiles, uint32_t blank) {
        uint32_t seen = (1u << (tiles & 15u)) | (1u << ((tiles >> 4) & 15u));
        uint32_t low = 0;
        uint64_t seg = 0;
#pragma unroll
        for (int i = 2; i < T; ++i) {
            const uint32_t v = uint32_t(tiles >> (4 * i)) & 15u;
            const uint32_t d = __popc(seen & ((1u << v) - 1u));
            seen |= 1u << v;
            if (i <= 11) low += d * uint32_t(fact(i) / 2);
            else seg |= uint64_t(d) << (4 * (i - 12));
        }
        return (seg << 32) | (uint64_t(low) * 16u + blank);
    }

    template <bool kOpBits, class Emit>
    __device__ __forceinline__ static void expand(uint64_t index, uint32_t opbits, int width, Emit& emit) {
        uint64_t tiles;
        uint32_t z;
        if (!board(index, width, tiles, z)) return;
        const uint32_t w = uint32_t(width);
        const uint64_t mask = (uint64_t(1) << (4 * w)) - 1;  // w <= 8 tiles
        if (z >= w && !(kOpBits && (opbits & 1u))) {  // blank up: tiles z-w .. z-1 rotate left
            const uint32_t a = 4u * (z - w);
            const uint64_t seg = (tiles >> a) & mask;
            const uint64_t rot = (seg >> 4) | ((seg & 15u) << (4 * (w - 1)));
            emit(index_of((tiles & ~(mask << a)) | (rot << a), z - w), 3u);
        }
        if (z + w < uint32_t(N) && !(kOpBits && (opbits & 8u))) {  // blank down: tiles z .. z+w-1 rotate right
            const uint32_t a = 4u * z;
            const uint64_t seg = (tiles >> a) & mask;
            const uint64_t rot = ((seg << 4) & mask) | (seg >> (4 * (w - 1)));
            emit(index_of((tiles & ~(mask << a)) | (rot << a), z + w), 0u);
        }
        if (z % w > 0 && !(kOpBits && (opbits & 2u))) emit(index - 1, 2u);
        if (z % w < w - 1 && !(kOpBits && (opbits & 4u))) emit(index + 1, 1u);
    }
};

// --------------------------------------------------------------------------
// Four-peg Towers of Hanoi (FourPegHanoiSimple.cpp:104-124,156-174): disk d
// (0 = smallest) sits on peg (index >> 2d) & 3.  For each peg pair a<b the
// smaller of the two top disks moves; the operator bit tested is the source
// peg and the child's operator is the destination peg.  With symmetry on,
// pegs 1..3 are relabelled after the move so that their bottom disks are in
// descending order, using the compare-exchange sequence (2,3),(1,2),(2,3)
// of FourPegHanoiSimple.cpp:51-69, and the child's operator is the
// destination's new label.
// --------------------------------------------------------------------------
struct Hanoi {
    static constexpr int kBranch = 6;
    static constexpr int kOps = 4;

    template <bool kOpBits, class Emit>
    // sym: 0 none; 1 FourPegHanoiSimple (restore after every move); 2
    // FourPegHanoiOptimized (restore only when the move empties the source
    // peg or lands on an empty one, FourPegHanoiOptimized.cpp:190-197; the
    // same children for canonical states, different ones for the others).
    __device__ __forceinline__ static void expand(uint64_t index, uint32_t opbits, int disks, int sym,
                                                  Emit& emit) {
        const uint64_t even = disks >= 32 ? 0x5555555555555555ull
                                          : (0x5555555555555555ull & ((uint64_t(1) << (2 * disks)) - 1));
        const uint64_t L = index & even, H = (index >> 1) & even;
        uint64_t m[4];
        m[0] = ~H & ~L & even;
        m[1] = ~H & L;
        m[2] = H & ~L;
        m[3] = H & L;
        int top[4];
#pragma unroll
        for (int p = 0; p < 4; ++p) top[p] = m[p] ? __ffsll((long long)m[p]) - 1 : 64;  // even bit position
#pragma unroll
        for (int a = 0; a < 4; ++a) {
#pragma unroll
            for (int b = a + 1; b < 4; ++b) {
                if (top[a] == 64 && top[b] == 64) continue;
                const bool a_src = top[a] < top[b];
                const int src = a_src ? a : b, dst = a_src ? b : a;
                const int pos = a_src ? top[a] : top[b];
                if (kOpBits && ((opbits >> src) & 1u)) continue;
                uint64_t child = index ^ (uint64_t(src ^ dst) << pos);
                uint32_t op = uint32_t(dst);
                if (sym == 1 || (sym == 2 && (top[dst] == 64 || m[src] == (uint64_t(1) << pos)))) {
                    const uint64_t bitpos = uint64_t(1) << pos;
                    uint64_t mm[4];
#pragma unroll
                    for (int q = 0; q < 4; ++q) mm[q] = m[q] ^ ((q == src || q == dst) ? bitpos : 0);
                    int bottom[4], lab[4] = {0, 1, 2, 3};
#pragma unroll
                    for (int p = 0; p < 4; ++p) bottom[p] = mm[p] ? 63 - __clzll((long long)mm[p]) : -1;
                    // compare-exchange (2,3), (1,2), (2,3): swap when bottom[i] < bottom[j]
                    auto cx = [&](int i, int j) {
                        if (bottom[i] < bottom[j]) {
                            int t = bottom[i]; bottom[i] = bottom[j]; bottom[j] = t;
                            uint64_t u = mm[i]; mm[i] = mm[j]; mm[j] = u;
                            t = lab[i]; lab[i] = lab[j]; lab[j] = t;
                        }
                    };
                    cx(2, 3); cx(1, 2); cx(2, 3);
                    // position k now holds original peg lab[k]: index bits of disks on it = k
                    const uint64_t nl = mm[1] | mm[3], nh = mm[2] | mm[3];
                    child = nl | (nh << 1);
                    uint32_t inv = 0;
#pragma unroll
                    for (int k = 0; k < 4; ++k) if (lab[k] == dst) inv = uint32_t(k);
                    op = inv;
                }
                emit(child, op);
            }
        }
    }
};

}  // namespace psb
