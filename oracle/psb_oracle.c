/*
 * psb_oracle.c -- CPU oracle (test infrastructure only; see psb_oracle.h).
 *
 * Plain-C restatement of the reference's CPU path.  Each function names the
 * reference file:line it follows (paths relative to the reference project).
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load
 * this library; the product library never does.
 */
#include "psb_oracle.h"

#include <ctype.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------- */
/* Permutation index: Puzzles/PermutationMap.cpp:7-58                          */
/* ------------------------------------------------------------------------- */

/* PermutationMap.cpp:7-19: arr[i] -= number of earlier values smaller than it. */
void orc_perm_compact(int* arr, int size) {
    unsigned seen = 0;
    for (int i = 0; i < size; i++) {
        int v = arr[i];
        arr[i] -= __builtin_popcount(seen & ((1u << v) - 1u));
        seen |= 1u << v;
    }
}

/* PermutationMap.cpp:21-37: digit d selects the d-th unused value, via a
 * nibble list of the values still available. */
void orc_perm_uncompact(int* arr, int size) {
    uint64_t tiles = 0xFEDCBA9876543210ull;
    for (int i = 0; i < size; i++) {
        int k = arr[i];
        arr[i] = (int)((tiles >> (4 * k)) & 15);
        uint64_t lo = k == 0 ? 0 : (tiles & ((1ull << (4 * k)) - 1));
        uint64_t hi = (4 * k + 4) >= 64 ? 0 : ((tiles >> (4 * k + 4)) << (4 * k));
        tiles = hi | lo;
    }
}

/* PermutationMap.cpp:39-49: mixed radix, position 0 most significant. */
uint64_t orc_perm_rank(int* arr, int size) {
    orc_perm_compact(arr, size);
    uint64_t index = 0;
    for (int i = 0; i < size; i++) {
        index *= (uint64_t)(size - i);
        index += (uint64_t)arr[i];
    }
    return index;
}

/* PermutationMap.cpp:51-58 */
void orc_perm_unrank(uint64_t index, int* arr, int size) {
    for (int i = size - 1; i >= 0; i--) {
        arr[i] = (int)(index % (uint64_t)(size - i));
        index /= (uint64_t)(size - i);
    }
    orc_perm_uncompact(arr, size);
}

/* ------------------------------------------------------------------------- */
/* Puzzle descriptions                                                         */
/* ------------------------------------------------------------------------- */

static uint64_t factorial(int n) {
    uint64_t r = 1;
    for (int i = 2; i <= n; i++) r *= (uint64_t)i;
    return r;
}

/* PancakeOptimized's index (Puzzles/PancakeOptimized.cpp:26-77): for n <= 12
 * the permutation rank; above, the rank of the first n-12 Lehmer digits
 * (radices n .. 13) times 2^29 plus the rank of the last 12 (radices 12 .. 1),
 * i.e. (rank / 12!) << 29 | rank % 12!.  Offsets >= 12! in a 2^29 block
 * name no permutation. */
#define ORC_F12 479001600ull
static uint64_t popt_from_rank(int n, uint64_t r) { return n <= 12 ? r : ((r / ORC_F12) << 29) | (r % ORC_F12); }
static int popt_to_rank(int n, uint64_t i, uint64_t* r) {
    if (n <= 12) { *r = i; return 1; }
    uint64_t lo = i & ((1ull << 29) - 1);
    if (lo >= ORC_F12) return 0;
    *r = (i >> 29) * ORC_F12 + lo;
    return 1;
}

/* SlidingTilePuzzleOptimized's index (Puzzles/SlidingTilePuzzleOptimized.cpp).
 * The board's tiles in board order with the blank left out, tile t held as
 * t-1 (ParseState, :64-77); slot 15 holds the blank's position.  Pack
 * (:99-116) turns tile i into digit d_i = number of earlier tiles smaller
 * than it (0 <= d_i <= i) and drops d_0 and d_1: d_0 is always 0 and the
 * parity rule (:79-97) decides d_1.  GetIndex (:142-158): the low 32 bits are
 * blank + 16 * (d_2 + 3 * (d_3 + 4 * (d_4 + ... + 11 * d_11))), the segment
 * (bits 32 and up) is d_12 | d_13 << 4 | d_14 << 8. */
static uint64_t sopt_states(int size) {  /* IndexesCount (:205-211), MaxSegments / MaxIndexesPerSegment (:12-26) */
    if (size >= 14) return (uint64_t)(size == 14 ? 0xC + 1 : size == 15 ? 0xDC + 1 : 0xEDC + 1) << 32;
    uint64_t m = 16;
    for (int i = 3; i < size; i++) m *= (uint64_t)i;
    return m;
}

/* Parity (:79-97): the tile list's inversions, plus the blank's row when the
 * width is even, must be even. */
static int sopt_parity_ok(int w, int ntiles, const int* t, int blank) {
    int inv = 0;
    for (int i = 0; i < ntiles; i++)
        for (int j = 0; j < i; j++) inv += t[j] > t[i];
    return ((inv + (w % 2 == 0 ? blank / w : 0)) & 1) == 0;
}

static uint64_t sopt_index(int ntiles, const int* t, int blank) {  /* Pack + GetIndex */
    int d[16] = { 0 };
    for (int i = 2; i < ntiles; i++)
        for (int j = 0; j < i; j++) d[i] += t[j] < t[i];
    uint64_t low = 0;
    for (int i = (ntiles - 1 < 11 ? ntiles - 1 : 11); i >= 2; i--) low = low * (uint64_t)(i + 1) + (uint64_t)d[i];
    uint64_t seg = 0;
    for (int i = 12; i < ntiles; i++) seg |= (uint64_t)d[i] << (4 * (i - 12));
    return (seg << 32) | (low * 16 + (uint64_t)blank);
}

/* FromIndex (:160-187) + Unpack (:118-140): 0 when the index names no board. */
static int sopt_board(int w, int size, uint64_t index, int* t, int* blank) {
    const int ntiles = size - 1;
    int d[16] = { 0 };
    *blank = (int)(index & 15);
    if (*blank >= size) return 0;
    uint64_t low = (index & 0xFFFFFFFFull) >> 4;
    for (int i = 2; i <= 11; i++) {
        d[i] = (int)(low % (uint64_t)(i + 1));
        low /= (uint64_t)(i + 1);
    }
    if (low) return 0;
    uint64_t seg = index >> 32;
    for (int i = 12; i <= 14; i++) { d[i] = (int)(seg & 15); seg >>= 4; }
    if (seg) return 0;
    for (int i = 0; i < 16; i++) if (d[i] > i || (i >= ntiles && d[i])) return 0;
    /* values from the digits, last tile first: d_i selects among the unused values */
    uint64_t left = 0xFEDCBA9876543210ull;
    for (int i = ntiles - 1; i >= 2; i--) {
        t[i] = (int)((left >> (4 * d[i])) & 15);
        uint64_t lo = d[i] == 0 ? 0 : (left & ((1ull << (4 * d[i])) - 1));
        left = ((left >> (4 * d[i] + 4)) << (4 * d[i])) | lo;
    }
    t[0] = (int)((left >> 4) & 15); /* d_1 = 0: tile 1 below tile 0 */
    t[1] = (int)(left & 15);
    if (!sopt_parity_ok(w, ntiles, t, *blank)) { int x = t[0]; t[0] = t[1]; t[1] = x; }
    return 1;
}

static int valid(const orc_puzzle* p) {
    if (!p) return 0;
    switch (p->kind) {
    case ORC_SLIDING: return p->a >= 1 && p->b >= 1 && p->a * p->b >= 2 && p->a * p->b <= 16;
    case ORC_PANCAKE: return p->a >= 2 && p->a <= 16;   /* PancakeSimple.cpp:26 */
    case ORC_PANCAKE_OPT: return p->a >= 2 && p->a <= 16;  /* PancakeOptimized.cpp:81-86 */
    case ORC_HANOI4: case ORC_HANOI4_OPT: return p->a >= 1 && p->a <= 31;
    case ORC_SLIDING_OPT: return p->a >= 1 && p->b >= 1 && p->a * p->b >= 4 && p->a * p->b <= 16;
    }
    return 0;
}

int orc_info(const orc_puzzle* p, uint64_t* indexes, int* ops, int* branching, int* odd) {
    if (!valid(p)) return -1;
    uint64_t n = 0; int o = 0, br = 0, od = 0;
    switch (p->kind) {
    case ORC_SLIDING: /* SlidingTilePuzzleSimple.h:13-19, .cpp:35-39 */
        n = factorial(p->a * p->b); o = 4; br = 4; od = 0; break;
    case ORC_PANCAKE: /* PancakeSimple.h:13-19, .cpp:36-40 */
        n = factorial(p->a); o = p->a - 1; br = p->a - 1; od = 1; break;
    case ORC_HANOI4: case ORC_HANOI4_OPT: /* FourPegHanoiSimple.h:14-20, .cpp:141-143; FourPegHanoiOptimized.cpp:164-166 */
        n = 1ull << (2 * p->a); o = 4; br = 6; od = 1; break;
    case ORC_PANCAKE_OPT: /* PancakeOptimized.h:14-20, .cpp:94-105: n! below 12, else prod(13..n) << 29 */
        if (p->a < 12) n = factorial(p->a);
        else { n = 1; for (int k = 13; k <= p->a; k++) n *= (uint64_t)k; n <<= 29; }
        o = p->a - 1; br = p->a - 1; od = 1; break;
    case ORC_SLIDING_OPT: /* SlidingTilePuzzleOptimized.h:14-24 */
        n = sopt_states(p->a * p->b); o = 4; br = 4; od = 0; break;
    }
    if (indexes) *indexes = n;
    if (ops) *ops = o;
    if (branching) *branching = br;
    if (odd) *odd = od;
    return 0;
}

static int read_ints(const char* s, int* out, int cap) {
    int n = 0;
    while (*s) {
        while (*s && isspace((unsigned char)*s)) s++;
        if (!*s) break;
        char* end;
        long v = strtol(s, &end, 10);
        if (end == s) return -1;
        if (n >= cap) return -1;
        out[n++] = (int)v;
        s = end;
    }
    return n;
}

/* Hanoi: disk d sits on peg (index >> 2d) & 3; disk 0 is the smallest
 * (FourPegHanoiSimple.cpp:104-124).  A state is kept as one disk mask per peg. */
typedef struct { uint64_t m[4]; } hstate;

static hstate hanoi_from_index(int n, uint64_t index) {
    hstate s; memset(&s, 0, sizeof s);
    for (int d = 0; d < n; d++) s.m[(index >> (2 * d)) & 3] |= 1ull << d;
    return s;
}

static uint64_t hanoi_to_index(const hstate* s) {
    uint64_t index = 0;
    for (int p = 0; p < 4; p++)
        for (uint64_t m = s->m[p]; m; m &= m - 1) index |= (uint64_t)p << (2 * __builtin_ctzll(m));
    return index;
}

static int hanoi_top(const hstate* s, int p) { return s->m[p] ? __builtin_ctzll(s->m[p]) : -1; }
static int hanoi_bottom(const hstate* s, int p) { return s->m[p] ? 63 - __builtin_clzll(s->m[p]) : -1; }

int orc_parse(const orc_puzzle* p, const char* state, uint64_t* index) {
    if (!valid(p) || !state || !index) return -1;
    int vals[64];
    int cnt = read_ints(state, vals, 64);
    if (cnt < 0) return -1;
    if (p->kind == ORC_SLIDING || p->kind == ORC_PANCAKE || p->kind == ORC_PANCAKE_OPT) {
        /* SlidingTilePuzzleSimple.cpp:52-59, PancakeSimple.cpp:53-60, PancakeOptimized.cpp:118-125 */
        int size = p->kind == ORC_SLIDING ? p->a * p->b : p->a;
        if (cnt != size) return -1;
        unsigned seen = 0;
        for (int i = 0; i < size; i++) {
            if (vals[i] < 0 || vals[i] >= size || (seen >> vals[i]) & 1) return -1;
            seen |= 1u << vals[i];
        }
        *index = orc_perm_rank(vals, size);
        if (p->kind == ORC_PANCAKE_OPT) *index = popt_from_rank(size, *index);
        return 0;
    }
    if (p->kind == ORC_SLIDING_OPT) {
        /* SlidingTilePuzzleOptimized.cpp:27-77 (ParseStandardState, ParseState)
         * and :224-236 (Parse): a board of an unsolvable parity is rejected. */
        const int size = p->a * p->b;
        if (cnt != size) return -1;
        int t[16], k = 0, blank = -1;
        unsigned seen = 0;
        for (int i = 0; i < size; i++) {
            if (vals[i] < 0 || vals[i] >= size || (seen >> vals[i]) & 1) return -1;
            seen |= 1u << vals[i];
            if (vals[i] == 0) blank = i;
            else t[k++] = vals[i] - 1;
        }
        if (!sopt_parity_ok(p->a, size - 1, t, blank)) return -1;
        *index = sopt_index(size - 1, t, blank);
        return 0;
    }
    /* FourPegHanoiSimple.cpp:85-102 (ParseState) + :104-113 (StateToIndex):
     * tokens are disk numbers starting at 1; a 0 moves to the next peg. */
    hstate s; memset(&s, 0, sizeof s);
    int peg = 0;
    for (int i = 0; i < cnt; i++) {
        if (vals[i] == 0) { peg++; continue; }
        if (peg > 3 || vals[i] < 1 || vals[i] > p->a) return -1;
        s.m[peg] |= 1ull << (vals[i] - 1);
    }
    *index = hanoi_to_index(&s);
    return 0;
}

int orc_to_string(const orc_puzzle* p, uint64_t index, char* buf, int cap) {
    if (!valid(p) || !buf || cap <= 0) return -1;
    char tmp[512]; int pos = 0;
    if (p->kind == ORC_SLIDING || p->kind == ORC_PANCAKE || p->kind == ORC_PANCAKE_OPT) {
        int size = p->kind == ORC_SLIDING ? p->a * p->b : p->a;
        int arr[16];
        if (p->kind == ORC_PANCAKE_OPT && !popt_to_rank(size, index, &index)) return -1;
        orc_perm_unrank(index, arr, size);
        for (int i = 0; i < size; i++) pos += snprintf(tmp + pos, sizeof tmp - pos, i ? " %d" : "%d", arr[i]);
    } else if (p->kind == ORC_SLIDING_OPT) {
        /* ToString (:213-217) via ToStandardState (:46-59): the blank as 0, tile t as t+1 */
        const int size = p->a * p->b;
        int t[16], blank, k = 0;
        if (!sopt_board(p->a, size, index, t, &blank)) return -1;
        for (int i = 0; i < size; i++)
            pos += snprintf(tmp + pos, sizeof tmp - pos, i ? " %d" : "%d", i == blank ? 0 : t[k++] + 1);
    } else {
        /* FourPegHanoiSimple.cpp:71-83: disks top-down (1-based) then a 0 per peg,
         * trailing " 0 " removed. */
        hstate s = hanoi_from_index(p->a, index);
        for (int pg = 0; pg < 4; pg++) {
            for (uint64_t m = s.m[pg]; m; m &= m - 1)
                pos += snprintf(tmp + pos, sizeof tmp - pos, "%d ", __builtin_ctzll(m) + 1);
            pos += snprintf(tmp + pos, sizeof tmp - pos, "0 ");
        }
        pos -= 3;
        tmp[pos] = 0;
    }
    if (pos + 1 > cap) return -1;
    memcpy(buf, tmp, (size_t)pos + 1);
    return pos;
}

/* ------------------------------------------------------------------------- */
/* Expand                                                                      */
/* ------------------------------------------------------------------------- */

typedef struct {
    uint64_t* children; uint32_t* ops; uint64_t cap; uint64_t n; int overflow;
} emitter;

static void emit(emitter* e, uint64_t child, uint32_t op) {
    if (e->n >= e->cap) { e->overflow = 1; return; }
    e->children[e->n] = child;
    e->ops[e->n] = op;
    e->n++;
}

/* SlidingTilePuzzleSimple.cpp:8 (op codes) and :61-99 (expand order). */
static void sliding_expand(int w, int h, uint64_t index, uint32_t op, emitter* e) {
    enum { UP = 0, LEFT = 1, RIGHT = 2, DOWN = 3 };
    int size = w * h, arr[16], tmp[16];
    orc_perm_unrank(index, arr, size);
    int blank = -1;
    for (int i = 0; i < size; i++) if (arr[i] == 0) { blank = i; break; }
    const int nb[4] = { blank - w, blank + w, blank - 1, blank + 1 };
    const int ok[4] = { blank >= w && !(op & (1u << UP)),
                        blank < size - w && !(op & (1u << DOWN)),
                        blank % w > 0 && !(op & (1u << LEFT)),
                        blank % w < w - 1 && !(op & (1u << RIGHT)) };
    const uint32_t back[4] = { DOWN, UP, RIGHT, LEFT };
    for (int k = 0; k < 4; k++) {
        if (!ok[k]) continue;
        memcpy(tmp, arr, sizeof arr);
        tmp[blank] = arr[nb[k]];
        tmp[nb[k]] = arr[blank];
        emit(e, orc_perm_rank(tmp, size), back[k]);
    }
}

/* PancakeSimple.cpp:12-20 (Move reverses the LAST count elements) and :62-73. */
static void pancake_expand(int n, uint64_t index, uint32_t opbits, emitter* e) {
    int arr[16], tmp[16];
    orc_perm_unrank(index, arr, n);
    for (int op = 0; op < n - 1; op++) {
        if (opbits & (1u << op)) continue;
        memcpy(tmp, arr, sizeof arr);
        for (int s = n - (op + 2), t = n - 1; s < t; s++, t--) { int x = tmp[s]; tmp[s] = tmp[t]; tmp[t] = x; }
        emit(e, orc_perm_rank(tmp, n), (uint32_t)op);
    }
}

/* FourPegHanoiSimple.cpp:51-69: pegs 1..3 sorted by their bottom (largest)
 * disk, descending, with the compare-exchange sequence (2,3),(1,2),(2,3).
 * Returns the new label of peg dst. */
static int hanoi_restore_symmetry(hstate* s, int dst) {
    int pegs[4] = { 0, 1, 2, 3 };
    static const int pairs[3][2] = { { 2, 3 }, { 1, 2 }, { 2, 3 } };
    for (int k = 0; k < 3; k++) {
        int i = pairs[k][0], j = pairs[k][1];
        if (hanoi_bottom(s, i) < hanoi_bottom(s, j)) {
            uint64_t t = s->m[i]; s->m[i] = s->m[j]; s->m[j] = t;
            int q = pegs[i]; pegs[i] = pegs[j]; pegs[j] = q;
        }
    }
    int inv[4];
    for (int k = 0; k < 4; k++) inv[pegs[k]] = k;
    return inv[dst];
}

/* FourPegHanoiSimple.cpp:156-174: for each peg pair (p1<p2) move the smaller
 * top disk; the operator bit tested is the source peg, the child's operator is
 * the destination peg (relabelled when symmetry is on).  sym 2 is
 * FourPegHanoiOptimized (.cpp:180-204): the order is restored only when the
 * move lands on an empty peg or empties its source. */
static void hanoi_expand(int n, int sym, uint64_t index, uint32_t op, emitter* e) {
    hstate st = hanoi_from_index(n, index);
    for (int a = 0; a < 4; a++) {
        for (int b = a + 1; b < 4; b++) {
            int ta = hanoi_top(&st, a), tb = hanoi_top(&st, b);
            int src, dst;
            if (ta >= 0 && (tb < 0 || tb > ta)) { src = a; dst = b; }
            else if (tb >= 0 && (ta < 0 || ta > tb)) { src = b; dst = a; }
            else continue; /* both pegs empty */
            hstate s2 = st;
            int disk = hanoi_top(&s2, src);
            s2.m[src] &= ~(1ull << disk);
            s2.m[dst] |= 1ull << disk;
            int childOp = dst;
            const int dst_was_empty = st.m[dst] == 0, src_now_empty = s2.m[src] == 0;
            if (sym == 1 || (sym == 2 && (dst_was_empty || src_now_empty))) childOp = hanoi_restore_symmetry(&s2, dst);
            if (!(op & (1u << src))) emit(e, hanoi_to_index(&s2), (uint32_t)childOp);
        }
    }
}

/* GPU expand kernel_sliding_tile_optimized (Puzzles/SlidingPuzzleGpu.cu:211-269):
 * blank up / down rotate the tiles between the old and the new blank
 * position; left / right only change the blank digit (index -+ 1).  The
 * op codes are SlidingTilePuzzleSimple's (UP 0, LEFT 1, RIGHT 2, DOWN 3). */
static void sliding_opt_expand(int w, int h, uint64_t index, uint32_t op, emitter* e) {
    enum { UP = 0, LEFT = 1, RIGHT = 2, DOWN = 3 };
    const int size = w * h, ntiles = size - 1;
    int t[16], u[16], z;
    if (!sopt_board(w, size, index, t, &z)) return;
    if (z >= w && !(op & (1u << UP))) {  /* RotateUp (:190-197) */
        memcpy(u, t, sizeof t);
        int x = u[z - w];
        for (int i = z - w; i < z - 1; i++) u[i] = u[i + 1];
        u[z - 1] = x;
        emit(e, sopt_index(ntiles, u, z - w), DOWN);
    }
    if (z < size - w && !(op & (1u << DOWN))) {  /* RotateDn (:199-206) */
        memcpy(u, t, sizeof t);
        int x = u[z + w - 1];
        for (int i = z + w - 1; i > z; i--) u[i] = u[i - 1];
        u[z] = x;
        emit(e, sopt_index(ntiles, u, z + w), UP);
    }
    if (z % w > 0 && !(op & (1u << LEFT))) emit(e, index - 1, RIGHT);
    if (z % w < w - 1 && !(op & (1u << RIGHT))) emit(e, index + 1, LEFT);
}

/* PancakeOptimized::Expand (.cpp:128-139): PancakeSimple's moves in its own
 * index; an offset that names no permutation has no children. */
static void pancake_opt_expand(int n, uint64_t index, uint32_t opbits, emitter* e) {
    uint64_t r;
    if (!popt_to_rank(n, index, &r)) return;
    uint64_t first = e->n;
    pancake_expand(n, r, opbits, e);
    for (uint64_t k = first; k < e->n; k++) e->children[k] = popt_from_rank(n, e->children[k]);
}

static void expand_one(const orc_puzzle* p, uint64_t index, uint32_t op, emitter* e) {
    switch (p->kind) {
    case ORC_SLIDING: sliding_expand(p->a, p->b, index, op, e); break;
    case ORC_PANCAKE: pancake_expand(p->a, index, op, e); break;
    case ORC_HANOI4: hanoi_expand(p->a, p->b ? 1 : 0, index, op, e); break;
    case ORC_HANOI4_OPT: hanoi_expand(p->a, p->b ? 2 : 0, index, op, e); break;
    case ORC_PANCAKE_OPT: pancake_opt_expand(p->a, index, op, e); break;
    case ORC_SLIDING_OPT: sliding_opt_expand(p->a, p->b, index, op, e); break;
    }
}

int64_t orc_expand(const orc_puzzle* p, const uint64_t* parents, const uint32_t* opbits,
                   uint64_t n, uint64_t* children, uint32_t* child_ops, uint64_t cap) {
    if (!valid(p)) return -2;
    emitter e = { children, child_ops, cap, 0, 0 };
    for (uint64_t i = 0; i < n; i++) expand_one(p, parents[i], opbits ? opbits[i] : 0, &e);
    return e.overflow ? -1 : (int64_t)e.n;
}

/* ------------------------------------------------------------------------- */
/* In-memory BFS drivers                                                       */
/* ------------------------------------------------------------------------- */

/* Children of one parent go through a small buffer (at most 15 children). */
#define ORC_MAXBR 16

static uint64_t words64(uint64_t bits) { return (bits + 63) / 64; }

uint64_t orc_final_words(const orc_puzzle* p, int algo) {
    uint64_t n;
    if (orc_info(p, &n, 0, 0, 0)) return 0;
    switch (algo) {
    case ORC_TWO_BIT: return words64(2 * n);
    case ORC_THREE_BIT: case ORC_CLASSIC: return 3 * words64(n);
    case ORC_FRONTIER: return 2 * ((n + 15) / 16);
    }
    return 0;
}

/* 2-bit array in the reference's vector<bool> layout
 * (InMemoryTwoBitBFS.cpp:6-20): bit 2i = code/2, bit 2i+1 = code%2. */
static inline int tb_get(const uint64_t* a, uint64_t i) {
    uint64_t b = 2 * i;
    int hi = (a[b >> 6] >> (b & 63)) & 1;
    int lo = (a[(b + 1) >> 6] >> ((b + 1) & 63)) & 1;
    return hi * 2 + lo;
}
static inline void tb_set(uint64_t* a, uint64_t i, int v) {
    uint64_t b = 2 * i;
    a[b >> 6] = (a[b >> 6] & ~(1ull << (b & 63))) | ((uint64_t)(v >> 1) << (b & 63));
    b++;
    a[b >> 6] = (a[b >> 6] & ~(1ull << (b & 63))) | ((uint64_t)(v & 1) << (b & 63));
}
static inline int bit_get(const uint64_t* a, uint64_t i) { return (a[i >> 6] >> (i & 63)) & 1; }
static inline void bit_set(uint64_t* a, uint64_t i) { a[i >> 6] |= 1ull << (i & 63); }

static int push(uint64_t* counts, int cap, int* n, uint64_t v) {
    if (*n >= cap) return -1;
    counts[(*n)++] = v;
    return 0;
}

/* InMemoryTwoBitBFS.cpp:24-69 */
static int bfs_two_bit(const orc_puzzle* p, uint64_t N, uint64_t init, uint64_t* counts, int cap,
                       uint64_t* fin, uint64_t fincap) {
    uint64_t W = words64(2 * N);
    uint64_t* a = calloc(W, 8);
    if (!a) return -3;
    int UNVISITED = 0, OLD = 1, CUR = 2, NEXT = 3, nd = 0, rc = 0;
    tb_set(a, init, CUR);
    if (push(counts, cap, &nd, 1)) { rc = -2; goto done; }
    uint64_t ch[ORC_MAXBR]; uint32_t ops[ORC_MAXBR];
    for (;;) {
        uint64_t count = 0;
        for (uint64_t i = 0; i < N; i++) {
            if (tb_get(a, i) != CUR) continue;
            tb_set(a, i, OLD);
            emitter e = { ch, ops, ORC_MAXBR, 0, 0 };
            expand_one(p, i, 0, &e);
            for (uint64_t k = 0; k < e.n; k++)
                if (tb_get(a, ch[k]) == UNVISITED) { count++; tb_set(a, ch[k], NEXT); }
        }
        if (count == 0) break;
        if (push(counts, cap, &nd, count)) { rc = -2; goto done; }
        int t = CUR; CUR = NEXT; NEXT = t;
    }
    (void)UNVISITED;
    if (fin) { if (fincap < W) { rc = -4; goto done; } memcpy(fin, a, W * 8); }
done:
    free(a);
    return rc ? rc : nd;
}

/* InMemoryThreeBitBFS.cpp:4-48 (three_bit=1) and InMemoryClassicBFS.cpp:4-45. */
static int bfs_bitsets(const orc_puzzle* p, uint64_t N, int odd, int classic, uint64_t init,
                       uint64_t* counts, int cap, uint64_t* fin, uint64_t fincap) {
    uint64_t W = words64(N);
    uint64_t* A = calloc(W, 8); /* three-bit: old;  classic: closed  */
    uint64_t* B = calloc(W, 8); /* three-bit: cur;  classic: open    */
    uint64_t* C = calloc(W, 8); /* three-bit: new;  classic: newOpen */
    int nd = 0, rc = 0;
    if (!A || !B || !C) { rc = -3; goto done; }
    bit_set(B, init);
    if (classic) bit_set(A, init);
    if (push(counts, cap, &nd, 1)) { rc = -2; goto done; }
    uint64_t ch[ORC_MAXBR]; uint32_t ops[ORC_MAXBR];
    for (;;) {
        for (uint64_t w = 0; w < W; w++) {
            uint64_t v = B[w];
            if (classic) B[w] = 0; /* ScanBitsAndClear */
            for (; v; v &= v - 1) {
                uint64_t i = w * 64 + (uint64_t)__builtin_ctzll(v);
                emitter e = { ch, ops, ORC_MAXBR, 0, 0 };
                expand_one(p, i, 0, &e);
                for (uint64_t k = 0; k < e.n; k++) bit_set(C, ch[k]);
            }
        }
        uint64_t count = 0;
        if (!classic) {
            if (odd) for (uint64_t w = 0; w < W; w++) C[w] &= ~B[w];
            for (uint64_t w = 0; w < W; w++) { C[w] &= ~A[w]; count += (uint64_t)__builtin_popcountll(C[w]); }
            if (count == 0) break;
            if (push(counts, cap, &nd, count)) { rc = -2; goto done; }
            uint64_t* t = A; A = B; B = C; C = t;  /* old<-cur, cur<-new, new<-old */
            memset(C, 0, W * 8);
        } else {
            for (uint64_t w = 0; w < W; w++) { C[w] &= ~A[w]; count += (uint64_t)__builtin_popcountll(C[w]); }
            for (uint64_t w = 0; w < W; w++) A[w] |= C[w];
            if (count == 0) break;
            if (push(counts, cap, &nd, count)) { rc = -2; goto done; }
            uint64_t* t = B; B = C; C = t;          /* swap(open, newOpen) */
        }
    }
    if (fin) {
        if (fincap < 3 * W) { rc = -4; goto done; }
        memcpy(fin, A, W * 8); memcpy(fin + W, B, W * 8); memcpy(fin + 2 * W, C, W * 8);
    }
done:
    free(A); free(B); free(C);
    return rc ? rc : nd;
}

/* InMemoryFrontierSearch.cpp:8-112: 4 used-operator bits per state; states
 * expanded at the previous level are excluded when the graph has odd cycles. */
static int bfs_frontier(const orc_puzzle* p, uint64_t N, int odd, uint64_t init, uint64_t* counts,
                        int cap, uint64_t* fin, uint64_t fincap) {
    uint64_t W4 = (N + 15) / 16, W1 = words64(N);
    uint64_t* cur = calloc(W4, 8);
    uint64_t* nxt = calloc(W4, 8);
    uint64_t* cex = odd ? calloc(W1, 8) : NULL;
    uint64_t* nex = odd ? calloc(W1, 8) : NULL;
    int nd = 0, rc = 0;
    if (!cur || !nxt || (odd && (!cex || !nex))) { rc = -3; goto done; }
    uint64_t ch[ORC_MAXBR]; uint32_t ops[ORC_MAXBR];
    for (int level = 0;; level++) {
        uint64_t count = 0;
#define FS_EXPAND(idx, bits)                                                              \
        do {                                                                              \
            emitter e = { ch, ops, ORC_MAXBR, 0, 0 };                                     \
            expand_one(p, (idx), (bits), &e);                                             \
            for (uint64_t k = 0; k < e.n; k++)                                            \
                nxt[ch[k] / 16] |= 1ull << (4 * (ch[k] % 16) + ops[k]);                   \
        } while (0)
        if (level == 0) {
            FS_EXPAND(init, 0);
            if (odd) bit_set(nex, init);
            count++;
        } else {
            for (uint64_t w = 0; w < W4; w++) {
                uint64_t v = cur[w];
                if (!v) continue;
                cur[w] = 0;
                while (v) { /* ScanFourBits, BitArray.h:36-44 */
                    int pos = __builtin_ctzll(v) / 4;
                    uint32_t bits = (uint32_t)((v >> (4 * pos)) & 15);
                    v &= ~(15ull << (4 * pos));
                    uint64_t idx = w * 16 + (uint64_t)pos;
                    if (odd) {
                        if (bit_get(cex, idx)) continue;
                        bit_set(nex, idx);
                    }
                    FS_EXPAND(idx, bits);
                    count++;
                }
            }
        }
#undef FS_EXPAND
        if (count == 0) break;
        uint64_t* t = cur; cur = nxt; nxt = t;
        if (odd) { t = cex; cex = nex; nex = t; memset(nex, 0, W1 * 8); }
        if (push(counts, cap, &nd, count)) { rc = -2; goto done; }
    }
    if (fin) {
        if (fincap < 2 * W4) { rc = -4; goto done; }
        memcpy(fin, cur, W4 * 8); memcpy(fin + W4, nxt, W4 * 8);
    }
done:
    free(cur); free(nxt); free(cex); free(nex);
    return rc ? rc : nd;
}

int orc_bfs(const orc_puzzle* p, int algo, uint64_t initial, uint64_t* counts, int cap,
            uint64_t* fin, uint64_t fincap) {
    uint64_t N; int ops, odd;
    if (orc_info(p, &N, &ops, 0, &odd)) return -1;
    if (initial >= N) return -1;
    switch (algo) {
    case ORC_TWO_BIT: return bfs_two_bit(p, N, initial, counts, cap, fin, fincap);
    case ORC_THREE_BIT: return bfs_bitsets(p, N, odd, 0, initial, counts, cap, fin, fincap);
    case ORC_CLASSIC: return bfs_bitsets(p, N, odd, 1, initial, counts, cap, fin, fincap);
    case ORC_FRONTIER:
        if (ops > 4) return -1; /* FourBitArray holds 4 operator bits per state */
        return bfs_frontier(p, N, odd, initial, counts, cap, fin, fincap);
    }
    return -1;
}

/* Distance of every state from `initial` (255 = not reached), by the level
 * sweep of InMemoryClassicBFS.cpp:4-45 over the same expander: the set of
 * states at each depth, which a spilled frontier is checked against.
 * Returns the number of depths, or <0 on error (-2: more than 254 depths). */
int orc_depths(const orc_puzzle* p, uint64_t initial, uint8_t* depth) {
    uint64_t N; int ops, odd;
    if (orc_info(p, &N, &ops, 0, &odd) || initial >= N) return -1;
    memset(depth, 255, N);
    depth[initial] = 0;
    uint64_t ch[ORC_MAXBR]; uint32_t chops[ORC_MAXBR];
    for (int d = 0;; d++) {
        if (d >= 254) return -2;
        uint64_t found = 0;
        for (uint64_t i = 0; i < N; i++) {
            if (depth[i] != d) continue;
            emitter e = { ch, chops, ORC_MAXBR, 0, 0 };
            expand_one(p, i, 0, &e);
            for (uint64_t k = 0; k < e.n; k++)
                if (depth[ch[k]] == 255) { depth[ch[k]] = (uint8_t)(d + 1); found++; }
        }
        if (!found) return d + 1;
    }
}

/* ------------------------------------------------------------------------- */
/* StreamVInt: Common/StreamVInt.cpp                                           */
/* ------------------------------------------------------------------------- */

static inline void put32(uint8_t* p, uint32_t v) { p[0] = (uint8_t)v; p[1] = (uint8_t)(v >> 8); p[2] = (uint8_t)(v >> 16); p[3] = (uint8_t)(v >> 24); }
static inline uint32_t get32(const uint8_t* p) { return (uint32_t)p[0] | ((uint32_t)p[1] << 8) | ((uint32_t)p[2] << 16) | ((uint32_t)p[3] << 24); }

/* StreamVInt.cpp:22-66,146-157: one descriptor byte (2 bits per value =
 * bytes-1), then each value's 1..4 little-endian bytes. */
int orc_svi_encode_tuple(const uint32_t* v, uint8_t* out) {
    uint8_t desc = 0; int pos = 1;
    for (int i = 0; i < 4; i++) {
        uint32_t x = v[i];
        int bytes = x >> 24 ? 4 : x >> 16 ? 3 : x >> 8 ? 2 : 1;
        desc |= (uint8_t)((bytes - 1) << (2 * i));
        for (int b = 0; b < bytes; b++) out[pos++] = (uint8_t)(x >> (8 * b));
    }
    out[0] = desc;
    return pos;
}

/* StreamVInt.cpp:69-113,159-167 */
int orc_svi_decode_tuple(const uint8_t* in, uint32_t* v) {
    uint8_t desc = in[0]; int pos = 1;
    for (int i = 0; i < 4; i++) {
        int bytes = 1 + ((desc >> (2 * i)) & 3);
        uint32_t x = 0;
        for (int b = 0; b < bytes; b++) x |= (uint32_t)in[pos++] << (8 * b);
        v[i] = x;
    }
    return pos;
}

/* StreamVInt.cpp:209-230: header u32 count, in-place delta, zero padding to a
 * multiple of 8, then tuples. */
int orc_svi_encode(int count, uint32_t* idx, uint8_t* out) {
    if (count == 0) return 0;
    int adj = (count + 7) / 8 * 8;
    for (int i = count - 1; i > 0; i--) idx[i] -= idx[i - 1];
    for (int i = count; i < adj; i++) idx[i] = 0;
    put32(out, (uint32_t)count);
    int pos = 4;
    for (int i = 0; i < adj; i += 4) pos += orc_svi_encode_tuple(idx + i, out + pos);
    return pos;
}

/* StreamVInt.cpp:232-251 with DecodeIndexesAndDiff (:132-145). */
int orc_svi_decode(int* size, const uint8_t* in, uint32_t* idx) {
    if (*size == 0) return 0;
    int count = (int)get32(in);
    int adj = (count + 7) / 8 * 8, pos = 4;
    uint32_t cur = 0;
    for (int i = 0; i < adj; i += 4) {
        pos += orc_svi_decode_tuple(in + pos, idx + i);
        for (int k = 0; k < 4; k++) cur = (idx[i + k] += cur);
    }
    *size = pos;
    return count;
}

/* StreamVInt.cpp:180-185 (bounds tuple): 8 nibbles packed into a u32 as
 * (all | all >> 28) where all is the 8 bytes read as a little-endian u64. */
int orc_svi_encode_bounds(int count, const uint32_t* unused, const uint8_t* bounds, uint8_t* out) {
    (void)unused;
    for (int i = 0; i < count; i += 8) {
        uint64_t all = 0;
        for (int k = 0; k < 8; k++) all |= (uint64_t)bounds[i + k] << (8 * k);
        put32(out + i / 2, (uint32_t)(all | (all >> 28)));
    }
    return count / 2;
}

/* StreamVInt.cpp:253-299: Encode/Decode with per-index operator bits
 * ("bounds"): the index stream as above, then the padded bounds packed two
 * nibbles per byte. */
int orc_svi_encode_ops(int count, uint32_t* idx, uint8_t* bounds, uint8_t* out) {
    if (count == 0) return 0;
    int adj = (count + 7) / 8 * 8;
    for (int i = count; i < adj; i++) bounds[i] = 0;
    int pos = orc_svi_encode(count, idx, out);
    pos += orc_svi_encode_bounds(adj, NULL, bounds, out + pos);
    return pos;
}

int orc_svi_decode_ops(int* size, const uint8_t* in, uint32_t* idx, uint8_t* bounds) {
    if (*size == 0) return 0;
    int count = orc_svi_decode(size, in, idx);
    int adj = (count + 7) / 8 * 8, pos = *size;
    for (int i = 0; i < adj; i += 8) {
        uint64_t st = get32(in + pos + i / 2);
        uint64_t all = (st & 0x0F0F0F0Full) | ((st & 0xF0F0F0F0ull) << 28);
        for (int k = 0; k < 8; k++) bounds[i + k] = (uint8_t)(all >> (8 * k));
    }
    *size = pos + adj / 2;
    return count;
}

/* OpBitsCompression<BITS> (Common/OpBitsCompression.cpp:10-76): every group
 * of 8 op-bit bytes (little-endian u64 `all`) becomes BITS bytes:
 *   BITS 2: u16 (all | all >> 14 | all >> 28 | all >> 42)
 *   BITS 4: u32 (all | all >> 28)            (the StreamVInt bounds packing)
 *   BITS 8: the 8 bytes unchanged.
 * count must be a multiple of 8; returns the bytes written / read. */
int64_t orc_opbits_encode(int bits, uint64_t count, const uint8_t* ops, uint8_t* out) {
    if ((count & 7) || (bits != 2 && bits != 4 && bits != 8)) return -1;
    uint64_t pos = 0;
    for (uint64_t i = 0; i < count; i += 8) {
        uint64_t all = 0;
        for (int k = 0; k < 8; k++) all |= (uint64_t)ops[i + k] << (8 * k);
        uint64_t packed = bits == 2 ? (all | (all >> 14) | (all >> 28) | (all >> 42)) : bits == 4 ? (all | (all >> 28)) : all;
        for (int k = 0; k < bits; k++) out[pos + k] = (uint8_t)(packed >> (8 * k));
        pos += (uint64_t)bits;
    }
    return (int64_t)pos;
}

int64_t orc_opbits_decode(int bits, uint64_t count, const uint8_t* in, uint8_t* ops) {
    if ((count & 7) || (bits != 2 && bits != 4 && bits != 8)) return -1;
    uint64_t pos = 0;
    for (uint64_t i = 0; i < count; i += 8) {
        uint64_t st = 0, all;
        for (int k = 0; k < bits; k++) st |= (uint64_t)in[pos + k] << (8 * k);
        if (bits == 2)
            all = (st & 0x0303ull) | ((st & 0x0C0Cull) << 14) | ((st & 0x3030ull) << 28) | ((st & 0xC0C0ull) << 42);
        else if (bits == 4)
            all = (st & 0x0F0F0F0Full) | ((st & 0xF0F0F0F0ull) << 28);
        else
            all = st;
        for (int k = 0; k < 8; k++) ops[i + k] = (uint8_t)(all >> (8 * k));
        pos += (uint64_t)bits;
    }
    return (int64_t)pos;
}

/* ------------------------------------------------------------------------- */
/* FrontierCompression: Common/FrontierCompression.cpp                         */
/* ------------------------------------------------------------------------- */

#define CODEC_MAP 0x80000000u

int orc_fc_is_bitmap(const uint8_t* in) { return (get32(in) & CODEC_MAP) != 0; }

/* FrontierCompression.cpp:28-34 */
static uint64_t bitmap_size(int count, const uint32_t* idx) {
    uint64_t first = idx[0], last = idx[count - 1];
    if (last < first) return ~(uint64_t)0;
    return (last - first + 63) / 64 * 8 + 8;
}

/* FrontierCompression.cpp:36-51: [u32 words|MAP][u32 first][bitmap of v-first-1]. */
int orc_fc_encode_bitmap(int count, const uint32_t* idx, uint8_t* out) {
    uint64_t first = idx[0], last = idx[count - 1];
    uint64_t words = (last - first + 63) / 64;
    put32(out, (uint32_t)(words | CODEC_MAP));
    put32(out + 4, (uint32_t)first);
    memset(out + 8, 0, words * 8);
    for (int i = 1; i < count; i++) {
        uint64_t v = (uint64_t)idx[i] - first - 1;
        if (v >= words * 64) continue; /* unsorted input: undefined in the reference */
        out[8 + v / 8] |= (uint8_t)(1u << (v % 8));
    }
    return (int)(8 + words * 8);
}

/* FrontierCompression.cpp:53-72 */
int orc_fc_encode_bitmap_with_check(int count, const uint32_t* idx, uint8_t* out) {
    uint64_t first = idx[0], last = idx[count - 1];
    if (last <= first) return -1;
    uint64_t max = last - first - 1;
    uint64_t words = (last - first + 63) / 64;
    put32(out, (uint32_t)(words | CODEC_MAP));
    put32(out + 4, (uint32_t)first);
    memset(out + 8, 0, words * 8);
    for (int i = 1; i < count; i++) {
        uint64_t v = (uint64_t)idx[i] - first - 1;
        if (v > max) return -1;
        out[8 + v / 8] |= (uint8_t)(1u << (v % 8));
    }
    return (int)(8 + words * 8);
}

static int decode_bitmap(int* size, const uint8_t* in, uint32_t* idx) {
    uint32_t words = get32(in) & ~CODEC_MAP;
    uint32_t first = get32(in + 4);
    int n = 0;
    idx[n++] = first;
    for (uint64_t i = 0; i < words; i++) {
        uint64_t w = 0;
        for (int k = 0; k < 8; k++) w |= (uint64_t)in[8 + i * 8 + k] << (8 * k);
        for (; w; w &= w - 1) idx[n++] = first + (uint32_t)(i * 64 + (uint64_t)__builtin_ctzll(w)) + 1;
    }
    *size = (int)(8 + (uint64_t)words * 8);
    return n;
}

/* FrontierCompression.cpp:92-102 */
int orc_fc_encode(int count, uint32_t* idx, uint8_t* out) {
    if (count == 0) return 0;
    uint64_t minBits = (uint64_t)count * 10;
    uint64_t hmBits = bitmap_size(count, idx) * 8;
    if (count > 128 && hmBits < minBits - 8) return orc_fc_encode_bitmap(count, idx, out);
    return orc_svi_encode(count, idx, out);
}

/* FrontierCompression.cpp:104-115 */
int orc_fc_encode_with_check(int count, uint32_t* idx, uint8_t* out) {
    if (count == 0) return 0;
    uint64_t minBits = (uint64_t)count * 10;
    uint64_t hmBits = bitmap_size(count, idx) * 8;
    if (count > 128 && hmBits < minBits) {
        int r = orc_fc_encode_bitmap_with_check(count, idx, out);
        if (r >= 0) return r;
    }
    return orc_svi_encode(count, idx, out);
}

/* FrontierCompression.cpp:117-125 */
int orc_fc_decode(int* size, const uint8_t* in, uint32_t* idx) {
    if (*size == 0) return 0;
    if (orc_fc_is_bitmap(in)) return decode_bitmap(size, in, idx);
    return orc_svi_decode(size, in, idx);
}
