/*
 * psb_oracle.h -- CPU oracle for the complete-BFS hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference's
 * CPU algorithms (lightln2/PuzzleSearch: Puzzles/PermutationMap.cpp,
 * Puzzles/...Simple.cpp, Common/InMemory...BFS.cpp, Common/StreamVInt.cpp,
 * Common/FrontierCompression.cpp).  It is used by tests/, by
 * __graft_entry__.smoke() and by bench.py's CPU-baseline leg as the checker.
 * The product library (puzzlesearch_b200/libpsb200.so) never links or calls it.
 *
 * Parity pin: every function here is checked against the reference's own
 * golden vectors (JSON fixtures under tests/golden, extracted from the reference's test
 * files) and, where the reference compiles in this container, against the
 * reference itself built from its sources into oracle/_ref/.
 */
#ifndef PSB_ORACLE_H
#define PSB_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { ORC_SLIDING = 1, ORC_PANCAKE = 2, ORC_HANOI4 = 3, ORC_PANCAKE_OPT = 4, ORC_HANOI4_OPT = 5, ORC_SLIDING_OPT = 6 };
enum { ORC_TWO_BIT = 1, ORC_THREE_BIT = 2, ORC_FRONTIER = 3, ORC_CLASSIC = 4 };

#define ORC_INVALID_INDEX (~(uint64_t)0)

typedef struct {
    int kind; /* ORC_SLIDING / ORC_PANCAKE / ORC_HANOI4 / ORC_PANCAKE_OPT / ORC_HANOI4_OPT / ORC_SLIDING_OPT */
    int a;    /* sliding: width;  pancake: size;  hanoi: disks */
    int b;    /* sliding: height; pancake: 0;     hanoi: symmetry flag; pancake opt: inverse-index flag */
} orc_puzzle;

/* Permutation index (Puzzles/PermutationMap.cpp:7-58). */
void orc_perm_compact(int* arr, int size);
void orc_perm_uncompact(int* arr, int size);
uint64_t orc_perm_rank(int* arr, int size);
void orc_perm_unrank(uint64_t index, int* arr, int size);

/* Puzzle interface (Common/Puzzle.h:16-48). Return 0 on success, <0 on bad puzzle. */
int orc_info(const orc_puzzle* p, uint64_t* indexes, int* ops, int* branching, int* odd_cycles);
int orc_parse(const orc_puzzle* p, const char* state, uint64_t* index);
int orc_to_string(const orc_puzzle* p, uint64_t index, char* buf, int cap);
/* Expands n parents in order; children are appended compactly (no INVALID
 * padding), exactly as the *Simple classes append them.  Returns the number of
 * children written, or -1 when cap is too small. */
int64_t orc_expand(const orc_puzzle* p, const uint64_t* parents, const uint32_t* opbits,
                   uint64_t n, uint64_t* children, uint32_t* child_ops, uint64_t cap);

/* In-memory BFS drivers (Common/InMemory{TwoBit,ThreeBit,Classic}BFS.cpp,
 * Common/InMemoryFrontierSearch.cpp).  Writes per-depth counts; returns the
 * number of depths, or <0 on error (-2: counts capacity too small).
 * If final_words != NULL, the final arrays are copied there in the
 * reference's memory layout:
 *   TWO_BIT:   one array of ceil(2N/64) words (vector<bool> layout, bit 2i = code/2, bit 2i+1 = code%2)
 *   THREE_BIT: old, cur, new -- three arrays of ceil(N/64) words each
 *   CLASSIC:   closed, open, newOpen -- three arrays of ceil(N/64) words
 *   FRONTIER:  current, next -- two arrays of ceil(N/16) words (4 bits per state)
 * final_words_cap is in words. */
int orc_bfs(const orc_puzzle* p, int algo, uint64_t initial, uint64_t* counts, int counts_cap,
            uint64_t* final_words, uint64_t final_words_cap);
uint64_t orc_final_words(const orc_puzzle* p, int algo);
/* Distance of every state from initial (depth[N]; 255 = not reached).
 * Returns the number of depths, <0 on error. */
int orc_depths(const orc_puzzle* p, uint64_t initial, uint8_t* depth);

/* StreamVInt (Common/StreamVInt.cpp) -- byte-exact format. */
int orc_svi_encode_tuple(const uint32_t* v4, uint8_t* out);       /* returns bytes (5..17) */
int orc_svi_decode_tuple(const uint8_t* in, uint32_t* v4);        /* returns bytes consumed */
int orc_svi_encode(int count, uint32_t* indexes, uint8_t* out);   /* delta in place; indexes needs round8(count) slots */
int orc_svi_decode(int* size, const uint8_t* in, uint32_t* indexes); /* returns count; *size = bytes consumed */
int orc_svi_encode_bounds(int count, const uint32_t* idx_deltas_unused, const uint8_t* bounds, uint8_t* out);
/* Index stream followed by the operator bits ("bounds", 4 bits per index). */
int orc_svi_encode_ops(int count, uint32_t* indexes, uint8_t* bounds, uint8_t* out);
int64_t orc_opbits_encode(int bits, uint64_t count, const uint8_t* ops, uint8_t* out);
int64_t orc_opbits_decode(int bits, uint64_t count, const uint8_t* in, uint8_t* ops);
int orc_svi_decode_ops(int* size, const uint8_t* in, uint32_t* indexes, uint8_t* bounds);

/* FrontierCompression (Common/FrontierCompression.cpp) -- byte-exact. */
int orc_fc_encode(int count, uint32_t* indexes, uint8_t* out);          /* bitmap or StreamVInt */
int orc_fc_encode_with_check(int count, uint32_t* indexes, uint8_t* out);
int orc_fc_encode_bitmap(int count, const uint32_t* indexes, uint8_t* out);
int orc_fc_encode_bitmap_with_check(int count, const uint32_t* indexes, uint8_t* out);
int orc_fc_decode(int* size, const uint8_t* in, uint32_t* indexes);
int orc_fc_is_bitmap(const uint8_t* in);

#ifdef __cplusplus
}
#endif

#endif
