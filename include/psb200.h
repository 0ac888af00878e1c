/*
 * psb200.h -- C ABI of puzzlesearch_b200, a B200-native (sm_100a) engine for
 * complete breadth-first search over ranked puzzle state spaces.
 *
 * It is a drop-in for the complete-BFS path of lightln2/PuzzleSearch: the
 * abstract Puzzle class (Common/Puzzle.h:16-48), its *Simple puzzles
 * (Puzzles/SlidingTilePuzzleSimple.h, PancakeSimple.h, FourPegHanoiSimple.h)
 * and the entry points InMemoryClassicBFS / InMemoryTwoBitBFS /
 * InMemoryThreeBitBFS / InMemoryFrontierSearch (Common/InMemoryBFS.h:5-11).
 * Indexes, operator codes, per-depth counts and final bit arrays are
 * identical to the reference's.  include/psb200.hpp wraps this ABI in the
 * reference's C++ interface.
 *
 * Conventions: plain C types only; every function returns int status
 * (PSB_OK = 0, negative = error; psb_last_error() gives the message of the
 * calling thread's last error).  No exceptions cross the ABI.  Calls on
 * distinct puzzle handles may run concurrently from different threads.
 */
#ifndef PSB200_H
#define PSB200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PSB_ABI_VERSION 1

/* Status codes. */
enum {
    PSB_OK = 0,
    PSB_ERR_ARG = -1,         /* bad argument (replaces the reference's ensure()/exit(-1), Common/Util.h:13-15) */
    PSB_ERR_CUDA = -2,        /* CUDA runtime error (the reference throws std::runtime_error, Puzzles/GPU.cu:5-10) */
    PSB_ERR_NOMEM = -3,       /* device or host allocation failed */
    PSB_ERR_CAPACITY = -4,    /* an output buffer is too small */
    PSB_ERR_UNSUPPORTED = -5, /* combination not supported (e.g. frontier search with > 4 operators) */
    PSB_ERR_DEVICE = -6,      /* a kernel reported an internal error (index out of range) */
    PSB_ERR_NO_DEVICE = -7,   /* no CUDA device visible */
    PSB_ERR_ABORTED = -8,     /* a callback (psb_spill_fn) returned non-zero */
    PSB_ERR_IO = -9           /* a file of a segment store could not be created, written, read or removed
                                 (the reference's file layer exits instead, Common/File.cpp) */
};

/* Puzzle kinds (the reference's *Simple classes). */
enum {
    PSB_SLIDING = 1, /* SlidingTilePuzzleSimple(width=a, height=b), 2 <= a*b <= 16 */
    PSB_PANCAKE = 2, /* PancakeSimple(size=a), 2 <= a <= 16 */
    PSB_HANOI4 = 3,  /* FourPegHanoiSimple(disks=a, useSymmetry=b), 1 <= a <= 31 */
    PSB_PANCAKE_OPT = 4, /* PancakeOptimized(size=a, inverseIndex=b), 2 <= a <= 16: for a >= 12 the index is
                            (rank / 12!) << 29 | rank % 12! over prod(13..a) * 2^29 indexes
                            (Puzzles/PancakeOptimized.cpp:26-105); offsets >= 12! are never reached */
    PSB_HANOI4_OPT = 5,  /* FourPegHanoiOptimized(disks=a, useSymmetry=b): FourPegHanoiSimple's index; with
                            symmetry it restores the peg order only when a move empties or fills a peg
                            (Puzzles/FourPegHanoiOptimized.cpp:180-204), the same children for canonical
                            states */
    PSB_SLIDING_OPT = 6  /* SlidingTilePuzzleOptimized<width=a, height=b>, a*b in {4, 6, 8, 9, 10, 12, 14, 15,
                            16}: blank + 16 * (the tiles' left-smaller digits 2..11, mixed radix), digits
                            12..14 as nibbles above bit 32 (Puzzles/SlidingTilePuzzleOptimized.cpp:99-212);
                            16 * (a*b-1)!/2 indexes up to 13 cells, 13, 221 or 3805 segments of 2^32 above.
                            Blank positions >= a*b and digit patterns above 13 cells name no board */
};

/* In-memory search algorithms (Common/InMemoryBFS.h:5-11). */
enum {
    PSB_TWO_BIT = 1,   /* InMemoryTwoBitBFS    (Common/InMemoryTwoBitBFS.cpp:24-69)   */
    PSB_THREE_BIT = 2, /* InMemoryThreeBitBFS  (Common/InMemoryThreeBitBFS.cpp:4-48)  */
    PSB_FRONTIER = 3,  /* InMemoryFrontierSearch (Common/InMemoryFrontierSearch.cpp:57-112) */
    PSB_CLASSIC = 4    /* InMemoryClassicBFS   (Common/InMemoryClassicBFS.cpp:4-45)   */
};

#define PSB_INVALID_INDEX (~(uint64_t)0) /* Puzzle::INVALID_INDEX, Common/Puzzle.h:19 */

typedef struct psb_puzzle psb_puzzle;

/* Library version string (static storage, never NULL). */
const char* psb_version(void);
/* Copies the calling thread's last error message (NUL-terminated). */
int psb_last_error(char* buf, int cap);
/* Number of visible CUDA devices (0 when none). */
int psb_device_count(int* count);
/* Name, compute capability and SM count of `device` (-1 = current), e.g. for
 * keying tuning results. */
int psb_device_name(int device, char* buf, int cap);

/* --- Puzzle (Common/Puzzle.h:16-48) --------------------------------------- */

/* Replaces the constructors SlidingTilePuzzleSimple(w,h), PancakeSimple(n),
 * FourPegHanoiSimple(n, sym).  No device memory is held by a puzzle. */
int psb_puzzle_create(int kind, int a, int b, psb_puzzle** out);
int psb_puzzle_destroy(psb_puzzle* p);
/* Puzzle::IndexesCount, OperatorsCount, BranchingFactor, HasOddLengthCycles. */
int psb_puzzle_info(const psb_puzzle* p, uint64_t* indexes, int* operators, int* branching, int* odd_cycles);
/* Puzzle::Name. */
int psb_puzzle_name(const psb_puzzle* p, char* buf, int cap);
/* Puzzle::Parse / Puzzle::ToString (host). */
int psb_parse(const psb_puzzle* p, const char* state, uint64_t* index);
int psb_to_string(const psb_puzzle* p, uint64_t index, char* buf, int cap);

/* --- Expand (Common/Puzzle.h:32-37; GPU twin of Puzzles/PuzzleGpu.cpp:53-82) */

#define PSB_EXPAND_HOST_POINTERS 1u /* all pointers are host memory (copied in and out) */
#define PSB_EXPAND_COMPACT 2u       /* drop INVALID slots (host pointers only) */
#define PSB_EXPAND_USE_OPBITS 4u    /* honour used-operator bits (skip operators whose bit is set) */

/* Expands n parents.  Without PSB_EXPAND_COMPACT the output has
 * BranchingFactor() slots per parent, the valid children first in the
 * *Simple classes' order, unused slots = PSB_INVALID_INDEX with operator
 * (1 << OperatorsCount()) - 1, as the reference's GPU puzzles emit them
 * (PuzzlesTests/SlidingPuzzleTest.cpp:43-60).  With PSB_EXPAND_COMPACT the
 * valid children are packed in order and *n_out is their count.  cap is the
 * capacity of children / child_ops in elements.  Parents must be < IndexesCount().
 * stream is a cudaStream_t (NULL = the legacy default stream); the call
 * returns after the results are available. */
int psb_expand(const psb_puzzle* p, const uint64_t* parents, const uint32_t* opbits, uint64_t n,
               uint64_t* children, uint32_t* child_ops, uint64_t cap, uint64_t* n_out,
               uint32_t flags, void* stream);

/* --- In-memory BFS (Common/InMemoryBFS.h:5-11) ----------------------------- */

/* Frontier spill: receives one segment of one depth's frontier as the
 * reference's compressed segment stream (see psb_frontier_encode), in pinned
 * host memory that stays valid until the callback returns.  `states` =
 * offsets in the stream; the segment holds states
 * segment * 2^segment_bits ... (SegmentedOptions::GetSegIdx,
 * Common/DiskBasedBFS.h:22-24).  Non-zero ends the search with
 * PSB_ERR_ABORTED. */
typedef int (*psb_spill_fn)(void* user, uint32_t depth, uint32_t segment, const uint8_t* stream, uint64_t bytes,
                            uint64_t states);

/* Long-range marks of a two-bit level (children outside the thread block's
 * window).  PSB_FAR_NONE: read the target's code, then OR NEXT into it if it
 * is UNVISITED (InMemoryTwoBitBFS.cpp:44-49 per child).  PSB_FAR_NEAR: marks
 * whose target lies in the parent's aligned block of 12! states (pancake
 * flips up to 12; every long-range mark of the other puzzles) set a bit in a
 * 1-bit-per-state far bitmap, folded into the codes after the level; the
 * flips of more than 12 read first.  PSB_FAR_ALL: every long-range mark goes
 * to the far bitmap.  PSB_FAR_AUTO picks by measurement on B200: NEAR for
 * pancake and sliding tiles, NONE for Hanoi (its marks are local; the fold
 * would not pay).  NEAR and ALL hold the
 * bitmap (N/8 bytes) in device memory; without room for it the search runs
 * as NONE. */
enum { PSB_FAR_AUTO = 0, PSB_FAR_NONE = 1, PSB_FAR_NEAR = 2, PSB_FAR_ALL = 3 };

typedef struct {
    uint32_t struct_size;  /* sizeof(psb_bfs_opts) */
    uint32_t max_depth;    /* stop after this depth (0 = until the frontier is empty; PuzzleOptions::maxSteps, Common/DiskBasedBFS.h:10) */
    int32_t window_bits;   /* log2 states per thread-block window (0 = automatic) */
    int32_t device;        /* CUDA device ordinal (-1 = current) */
    void* stream;          /* cudaStream_t (NULL = a stream owned by the call) */
    uint64_t* final_words; /* optional host buffer: final arrays in the reference's layout (see psb_final_words) */
    uint64_t final_cap;    /* capacity of final_words in 64-bit words */
    float* level_ms;       /* optional, counts_cap entries: entry d = device ms of the level that expanded depth d */
    uint64_t* level_children; /* optional, counts_cap entries: entry d = children generated from depth d
                              (two-bit writes one more entry, for its final empty sweep, when it fits) */
    int32_t direction;     /* PSB_DIR_AUTO (0), PSB_DIR_TOP_DOWN or PSB_DIR_BOTTOM_UP; see below */
    float bottom_up_ratio; /* PSB_DIR_AUTO: a dense level runs bottom-up when unvisited < ratio * frontier (0 = 1.0) */
    psb_spill_fn spill;    /* optional: every depth's frontier, encoded on the GPU segment by segment (below) */
    void* spill_user;      /* first argument of spill */
    int32_t segment_bits;  /* states per spilled segment = 2^segment_bits, 6..32 (0 = 32, the default of
                              PuzzleOptions::segmentBits, Common/DiskBasedBFS.h:11) */
    int32_t far_marks;     /* PSB_TWO_BIT top-down levels: where long-range marks go (PSB_FAR_*) */
    int32_t threads;       /* threads per block of the top-down two-bit and three-bit level kernels: 128, 256 or
                              512 (0 = 128 for two-bit pancake and Hanoi searches of 2^32 states or more, else
                              256); the other kernels use 256 */
    uint64_t* restored_counts; /* optional, counts_cap entries; 4-peg Hanoi with symmetry and PSB_TWO_BIT only:
                              the counts HanoiSearch reports (HanoiTowers/HanoiSearch.cpp:247-262), i.e. each
                              depth's canonical states weighted by their class size (PegsMult,
                              HanoiTowers/HanoiTowers.h:48-55) = the per-depth counts of the search without
                              symmetry; entry 0 is 1 */
} psb_bfs_opts;

/* With opts->spill set, the states at each depth d = 0, 1, ... (every depth
 * the counts report) are encoded on the GPU, segment by segment, into the
 * reference's CompressedSegmentWriter stream (Common/CompressedFrontier.cpp:
 * 103-140) and copied to pinned host memory; spill(user, d, segment, ...)
 * then receives each one, on the calling thread.  Calls come in ascending
 * (depth, segment) order, all before psb_bfs returns; empty segments are
 * skipped, as the reference writes nothing for them.  Depth d is encoded on
 * the GPU before the level that expands it; its copies to the host and its
 * callbacks run while that level is on the GPU.
 * This replaces SegmentWriter's files with pinned host buffers: the caller
 * keeps, writes or drops each stream.  The spill's memory (an extracted
 * segment bitmap for two-bit and frontier searches, the encoder's offset
 * list, about 7 bytes per frontier state of a segment, a device arena for
 * one depth's streams and two pinned host buffers of one segment's stream)
 * is allocated on first use, kept for the
 * device's next searches and freed by psb_release_cached_memory; it is not
 * part of psb_bfs_footprint. */

/* Level direction.  A top-down level expands every frontier state and marks
 * its children, as the reference does.  A bottom-up level (three-bit,
 * two-bit and classic searches of pancakes, sliding tiles and Hanoi without
 * symmetry) makes every still unvisited state probe its neighbours for a
 * frontier state; on the last, dense levels of a search that is far less
 * work.  Counts and final arrays are the same either way.  Three-bit searches
 * that may go bottom-up keep one more bit per state (the visited set) when
 * device memory allows; otherwise every level runs top-down. */
#define PSB_DIR_AUTO 0      /* top-down; bottom-up on dense levels once unvisited < ratio * frontier */
#define PSB_DIR_TOP_DOWN 1  /* every level top-down (no visited array) */
#define PSB_DIR_BOTTOM_UP 2 /* every level bottom-up where the search supports it (tests) */

typedef struct {
    uint32_t struct_size;     /* sizeof(psb_bfs_stats) */
    uint32_t levels;          /* level kernels launched */
    uint32_t window_bits;     /* window used */
    uint32_t threads;         /* threads per block of the level kernel */
    double total_ms;          /* device time of the whole search (CUDA events) */
    double expand_ms;         /* sum over levels of the fused sweep+expand+mark kernel */
    double finalize_ms;       /* sum over levels of the finalize kernel (three-bit and classic only) */
    uint64_t expanded;        /* parents expanded */
    uint64_t children;        /* valid children generated */
    uint64_t local_children;  /* children marked in the block's shared-memory window */
    uint64_t expand_launches; /* level-kernel launches (one per level) */
    uint64_t device_bytes;    /* device memory held by the search */
    uint64_t bottom_up_levels; /* levels that ran bottom-up (their "children" are probes) */
    double spill_ms;          /* host time in the spill: encoding plus handing over (the latter overlaps the
                                 level that follows) */
    uint64_t spill_bytes;     /* stream bytes passed to the spill callback */
    uint64_t spill_segments;  /* callback calls */
    uint64_t spill_launches;  /* kernels the spill launched (extraction and encoding) */
    double spill_encode_ms;   /* host time encoding depths (the search waits for it) */
    double spill_copy_ms;     /* device time of the copies to pinned host memory */
    uint64_t other_launches;  /* kernels besides the level kernels and the spill's: finalize, retire and
                                 far-bitmap fold passes */
} psb_bfs_stats;

/* Size in 64-bit words of the final arrays that psb_bfs copies out:
 *   PSB_TWO_BIT:   ceil(2N/64)  (vector<bool> layout of InMemoryTwoBitBFS.cpp:6-20: bit 2i = code/2, bit 2i+1 = code%2)
 *   PSB_THREE_BIT: 3*ceil(N/64) (old, cur, new)
 *   PSB_CLASSIC:   3*ceil(N/64) (closed, open, newOpen)
 *   PSB_FRONTIER:  2*ceil(N/16) (current, next; 4 operator bits per state) */
int psb_final_words(const psb_puzzle* p, int algo, uint64_t* words);

/* Runs the whole search on the GPU from initial_index.  depth_counts[d] =
 * number of states at distance d, as returned by the reference's InMemory*
 * functions; *n_depths = number of depths.  The bit arrays stay in device
 * memory for the whole search; only the per-depth counts (and, on request,
 * the final arrays) come back.  opts and stats may be NULL. */
int psb_bfs(const psb_puzzle* p, int algo, uint64_t initial_index, const psb_bfs_opts* opts,
            uint64_t* depth_counts, uint32_t counts_cap, uint32_t* n_depths, psb_bfs_stats* stats);

/* Device memory the search of psb_bfs would allocate (bytes), for the
 * default direction (PSB_DIR_AUTO). */
int psb_bfs_footprint(const psb_puzzle* p, int algo, uint64_t* bytes);

/* Reusable device state: allocate once, run many searches (benchmarks and
 * serving keep arrays resident between runs). */
typedef struct psb_bfs_session psb_bfs_session;
int psb_bfs_session_create(const psb_puzzle* p, int algo, const psb_bfs_opts* opts, psb_bfs_session** out);
int psb_bfs_session_run(psb_bfs_session* s, uint64_t initial_index, const psb_bfs_opts* opts,
                        uint64_t* depth_counts, uint32_t counts_cap, uint32_t* n_depths, psb_bfs_stats* stats);
int psb_bfs_session_destroy(psb_bfs_session* s);

/* Search arrays (psb_bfs and sessions) come from a per-device memory pool
 * that keeps freed memory reserved for the next search instead of returning
 * it to the driver after every call.  This returns the reserved memory of
 * `device` (-1 = current) to the driver, and frees the frontier spill's
 * cached buffers; it waits for the device first. */
int psb_release_cached_memory(int device);

/* --- Device bit arrays (Common/BitArray.h:69-169) -------------------------
 * Bit i of an array of n_bits bits is bit i%64 of 64-bit word i/64 (device
 * memory, ceil(n_bits/64) words), the reference's BitArray layout.  The
 * searches fuse these operations into their kernels; these calls run them on
 * their own.  Each returns after the stream has reached it when it returns a
 * count (scan, and_not_count); set_stride and or are only enqueued. */

/* BitArray::Set(first + k*stride) for every such index below n_bits (:81-83). */
int psb_bits_set_stride(uint64_t* d_words, uint64_t n_bits, uint64_t first, uint64_t stride, void* stream);

/* BitArray::ScanBits (:138-145), ScanBitsAndClear (clear != 0, :147-155) and
 * ScanBitsAndClearWithExcl (d_exclude != NULL, :157-166) with the callback
 * "count the index and add it to a sum": *count = bits visited, *index_sum =
 * sum of their indexes mod 2^64.  Whole words are scanned, as the reference does. */
int psb_bits_scan(uint64_t* d_words, const uint64_t* d_exclude, uint64_t n_bits, int clear, uint64_t* count,
                  uint64_t* index_sum, void* stream);

/* BitArray::AndNotAndCount (:117-125): words &= ~exclude; *count = bits left. */
int psb_bits_and_not_count(uint64_t* d_words, const uint64_t* d_exclude, uint64_t n_bits, uint64_t* count,
                           void* stream);

/* BitArray::Or (:103-107): words |= other. */
int psb_bits_or(uint64_t* d_words, const uint64_t* d_other, uint64_t n_bits, void* stream);

/* --- Frontier compression (Common/FrontierCompression.cpp, StreamVInt.cpp,
 *     CompressedFrontier.cpp) -------------------------------------------------
 * A segment's frontier -- the set bits of a bitmap range of at most 2^32
 * states, as ascending u32 offsets -- in the reference's segment stream:
 * blocks of up to 262,144 offsets (StreamVInt::MAX_INDEXES_COUNT), each
 * FrontierCompression::Encode'd (bitmap block when count > 128 and it is
 * smaller than 10 bits per offset, else StreamVInt), concatenated as
 * CompressedSegmentWriter does (Common/CompressedFrontier.cpp:103-140).
 * The stream bytes are identical to the reference's. */
typedef struct {
    uint64_t offset;    /* byte offset of the block in the stream */
    uint32_t count;     /* offsets in the block */
    uint32_t bytes;     /* encoded size */
    uint32_t first;     /* first offset (bitmap blocks; first delta for StreamVInt) */
    uint32_t is_bitmap;
} psb_codec_block;

/* Encodes the set bits of d_bits[first_bit .. first_bit + n_bits) (device
 * memory; first_bit a multiple of 64; n_bits <= 2^32) into d_out (device).
 * *out_bytes receives the stream size; if d_out is NULL or out_cap is too
 * small the call returns PSB_ERR_CAPACITY with *out_bytes set (ask, then
 * encode).  blocks (host, optional) receives the block table used by
 * psb_frontier_decode. */
int psb_frontier_encode(const uint64_t* d_bits, uint64_t first_bit, uint64_t n_bits, uint8_t* d_out,
                        uint64_t out_cap, uint64_t* out_bytes, psb_codec_block* blocks, uint32_t blocks_cap,
                        uint32_t* n_blocks, void* stream);
/* Builds the block table of a stream held in host memory (the reference's
 * own streams included): walks the block headers and StreamVInt descriptors. */
int psb_frontier_index(const uint8_t* stream, uint64_t stream_bytes, psb_codec_block* blocks, uint32_t cap,
                       uint32_t* n_blocks);
/* ORs the offsets of a device-resident stream into d_bits[first_bit ..
 * first_bit + n_bits) (bit first_bit + offset); blocks is the host table. */
int psb_frontier_decode(const uint8_t* d_stream, const psb_codec_block* blocks, uint32_t n_blocks,
                        uint64_t* d_bits, uint64_t first_bit, uint64_t n_bits, void* stream);

/* OpBitsCompression<bits>::Encode / Decode (Common/OpBitsCompression.cpp:
 * 10-76) on the GPU: `count` op-bit bytes (a multiple of 8, each below
 * 2^bits) <-> count * bits / 8 packed bytes; bits = 2, 4 or 8.  bits = 4 is
 * also StreamVInt's operator "bounds" packing (Common/StreamVInt.cpp:139-147).
 * Device pointers: the op-bit bytes 8-byte aligned, the packed bytes aligned
 * to `bits` bytes.  Asynchronous on `stream`. */
int psb_opbits_encode(int bits, const uint8_t* d_op_bits, uint64_t count, uint8_t* d_out, void* stream);
int psb_opbits_decode(int bits, const uint8_t* d_in, uint64_t count, uint8_t* d_op_bits, void* stream);

/* --- Segment store -----------------------------------------------------------------
 * The reference's Store (Common/Store.h:13-178): numbered segments, each a
 * list of chunks read back in the order they were written.  With
 * directories, the segments go round-robin over the directories (one per
 * disk, StoreOptions::directories) and, in each, to files_per_path files of
 * consecutive segments (StoreOptions::filesPerPath: 0 = one file per
 * segment, <dir>/<name>_<segment>; 1 = <dir>/<name>; k = <dir>/<name>_p0 ..
 * _p<k-1>).  A file exists while one of its segments holds data: it is
 * removed once they are all deleted, and by psb_store_destroy.  Without
 * directories the chunks stay in host memory.  Not thread-safe for
 * concurrent reads of one segment. */
typedef struct psb_store psb_store;
int psb_store_create(int max_segments, const char* name, const char* const* directories, int n_directories,
                     int files_per_path, psb_store** out);
int psb_store_destroy(psb_store* store);  /* removes its files */
int psb_store_write(psb_store* store, int segment, const void* buf, uint64_t size);  /* appends one chunk */
/* Next chunk of the segment into buf: *got = its size, 0 after the last one;
 * PSB_ERR_CAPACITY if the chunk is larger than cap. */
int psb_store_read(psb_store* store, int segment, void* buf, uint64_t cap, uint64_t* got);
int psb_store_rewind(psb_store* store, int segment);                   /* read from the first chunk again */
int psb_store_length(const psb_store* store, int segment, uint64_t* bytes);  /* segment < 0: all of them */
int psb_store_delete(psb_store* store, int segment);                   /* segment < 0: all of them */

/* --- Segmented (out-of-core) search -------------------------------------------
 * The reference's disk-based search, DiskBasedOptThreeBitBFS
 * (Common/DiskBasedOptThreeBitBFS.cpp:12-252): the state space is split into
 * segments of 2^segment_bits states (SegmentedOptions::GetSegIdx,
 * Common/DiskBasedBFS.h:22-24) and only one segment's three bit arrays
 * (3 x 2^segment_bits bits) plus an expansion buffer sit in device memory.
 * Every segment's last three frontier layers are kept as the reference's
 * compressed segment streams, and the children a segment's states have in
 * other segments as 4-byte offsets per target segment, in segment stores:
 * files in opts->directories (the reference's StoreOptions), else host
 * memory.  Per-depth counts equal the in-memory searches'.  A search larger
 * than device memory runs this way, and one larger than host memory with
 * directories; PCIe carries the layers and the cross-segment children. */
typedef struct {
    uint32_t struct_size;   /* sizeof(psb_segmented_opts) */
    uint32_t max_depth;     /* stop after this depth (0 = until the frontier is empty) */
    int32_t segment_bits;   /* 10..32 (0 = 32, PuzzleOptions::segmentBits' default) */
    int32_t device;         /* CUDA device (-1 = current) */
    uint64_t chunk_states;  /* states expanded per launch (bounds the child buffer; 0 = 2^22) */
    const char* const* directories; /* StoreOptions::directories: the layers and the cross-segment children go
                                       to files there (segment stores, above); none = host memory */
    int32_t n_directories;
    int32_t files_per_path; /* StoreOptions::filesPerPath (Common/Store.h:20-27); -1 = its default, 5 */
} psb_segmented_opts;
typedef struct {
    uint32_t struct_size;     /* sizeof(psb_segmented_stats) */
    uint32_t pad;
    uint64_t segments;        /* segments of the state space */
    uint64_t device_bytes;    /* device memory the search held */
    uint64_t peak_host_bytes; /* largest host memory held by layers and cross-segment children (with
                                 directories: the staging of the cross-segment children only) */
    uint64_t h2d_bytes, d2h_bytes;
    uint64_t cross_children;  /* children that landed in another segment than their parent's */
    double total_ms;          /* wall time of the call */
    uint64_t peak_disk_bytes; /* largest size of the store files (with directories) */
} psb_segmented_stats;
int psb_bfs_segmented(const psb_puzzle* p, uint64_t initial_index, const psb_segmented_opts* opts,
                      uint64_t* depth_counts, uint32_t counts_cap, uint32_t* n_depths, psb_segmented_stats* stats);

/* --- Batched and served solves -----------------------------------------------
 * No single counterpart in the reference (one InMemoryTwoBitBFS per call).
 * An engine keeps many independent two-bit searches on the GPU at once, each
 * with its own array in the reference's layout (InMemoryTwoBitBFS.cpp:6-20),
 * packed back to back in one device pool.  psb_engine_step advances every
 * active search by one level: one persistent kernel over an
 * (instance, window) work queue, captured once as a CUDA graph.  Searches
 * may be added between steps (continuous batching); finished ones are
 * collected with psb_engine_poll.  Per-depth counts equal psb_bfs's.
 * Puzzles: sliding tile with 6, 8, 9, 10 or 12 cells, pancake 7..12,
 * 4-peg Hanoi up to 16 disks. */
typedef struct psb_engine psb_engine;
typedef struct {
    uint32_t struct_size;   /* sizeof(psb_engine_opts) */
    uint32_t max_instances; /* instance slots */
    uint32_t max_depths;    /* per-depth counts kept per instance */
    int32_t device;         /* CUDA device (-1 = current) */
    uint64_t pool_bytes;    /* device pool for the instances' two-bit arrays (admission limit) */
    int32_t blocks_per_sm;  /* persistent blocks per SM (0 = 2) */
    int32_t use_graph;      /* 1 = replay each step as a CUDA graph */
    int32_t direction;      /* PSB_DIR_AUTO (0): each instance's dense late levels run bottom-up;
                               PSB_DIR_TOP_DOWN: every level top-down */
    int32_t window_bits_offset; /* each instance's window is 2^(log2 states - 6 + offset) states, clamped to
                                   2^10 .. 2^16 (0 = the rule; -6..6) */
} psb_engine_opts;
int psb_engine_create(const psb_engine_opts* opts, psb_engine** out);
int psb_engine_destroy(psb_engine* e);
/* Device bytes one instance takes in the pool: its two-bit array (2 bits per
 * state, padded) plus two bytes per window of active-window flags. */
int psb_engine_footprint(int kind, int a, int b, uint64_t* bytes);
/* Admits one search; PSB_ERR_CAPACITY when no slot or pool space is free. */
int psb_engine_add(psb_engine* e, int kind, int a, int b, uint64_t initial_index, uint64_t tag, uint32_t* slot);
/* Advances all active searches by `levels` levels (returns after the GPU is done). */
int psb_engine_step(psb_engine* e, uint32_t levels);
/* Collects up to cap finished searches: their tags, depth counts and per-depth
 * counts (row i of counts holds max_depths entries); frees their slots. */
int psb_engine_poll(psb_engine* e, uint64_t* tags, uint32_t* n_depths, uint64_t* counts, uint32_t cap, uint32_t* n);
/* Active searches, largest free pool extent, levels stepped so far. */
int psb_engine_info(psb_engine* e, uint32_t* active, uint64_t* largest_free_bytes, uint64_t* levels_run);

/* --- Solve server (continuous batching) -------------------------------------
 * No counterpart in the reference.  Two lanes share the GPU:
 *   * the batch lane: a server thread owns a psb_engine; it admits submitted
 *     requests smallest first while a slot and pool space are free
 *     (admission by HBM footprint) and advances all resident searches
 *     together, level by level (continuous batching);
 *   * the large lane: requests with more than large_states states run one at
 *     a time as single two-bit searches (psb_bfs sessions, one per puzzle
 *     size, reused) on a second thread and stream, overlapping the batch
 *     lane's steps on the device.  A large search's levels would otherwise
 *     set the pace of every small search resident with it.
 * Each request completes with its per-depth counts, its eccentricity
 * (n_depths - 1) and its latency from submission.  Submit and poll are
 * non-blocking and may be called from any thread. */
typedef struct psb_server psb_server;
typedef struct {
    uint32_t struct_size;     /* sizeof(psb_server_opts) */
    uint32_t levels_per_step; /* BFS levels per engine step while no request waits for admission (0 = 1); one
                                 level per step while requests wait */
    psb_engine_opts engine;
    uint64_t large_states;    /* requests with more states go to the large lane (0 = 2^26; UINT64_MAX = none) */
} psb_server_opts;
int psb_server_start(const psb_server_opts* opts, psb_server** out);
int psb_server_submit(psb_server* s, int kind, int a, int b, uint64_t initial_index, uint64_t* ticket);
/* Completed requests: ticket, status (PSB_OK or the admission error), depth
 * count, per-depth counts (max_depths per row), latency in seconds. */
int psb_server_poll(psb_server* s, uint64_t* tickets, int* status, uint32_t* n_depths, uint64_t* counts,
                    double* latency_s, uint32_t cap, uint32_t* n);
/* Queued and running requests, completed requests, engine steps; returns the
 * server's fatal error if it stopped on one. */
int psb_server_info(psb_server* s, uint32_t* queued, uint32_t* running, uint64_t* completed, uint64_t* steps);
int psb_server_stop(psb_server* s);

/* --- Search without device allocation --------------------------------------
 * No counterpart in the reference.  For callers that may not call cudaMalloc
 * (all device memory is owned by another allocator or a pre-reserved arena):
 * the same search as psb_bfs, but the caller passes the bit arrays in
 * d_arrays (device memory of at least psb_bfs_footprint() bytes, given in
 * 64-bit words as d_array_words) and the function allocates nothing: no
 * cudaMalloc/cudaFree, no pinned host memory, no stream or event.  Its few
 * bytes of scratch (level counters and active-window flags) sit in a static
 * device array of 4 MiB + 256 bytes that every GPU loading the library holds
 * until exit; searches needing more than 2^21 windows (more than ~1.4e11
 * states) return PSB_ERR_CAPACITY.  All calls share that array: calls whose
 * GPU work overlaps race, so run them one after the other.  d_arrays must be
 * 256-byte aligned (PSB_ERR_ARG otherwise, before the device is touched).
 * The first call on a device loads the library's kernels and the static
 * array (lazy module loading takes device memory from the driver then), so a
 * caller that reserves all device memory for its arena makes one small call
 * first.  Every call synchronizes `stream` once per level, so it must not be
 * called while that stream is being captured.  For PSB_TWO_BIT the final
 * code array is d_arrays[0 .. ceil(2N/64)) on return, in the reference's
 * layout. */
int psb_bfs_noalloc(const psb_puzzle* p, int algo, uint64_t initial_index, uint64_t* d_arrays,
                    uint64_t d_array_words, uint32_t max_depth, void* stream, uint64_t* depth_counts,
                    uint32_t counts_cap, uint32_t* n_depths);

#ifdef __cplusplus
}
#endif

#endif /* PSB200_H */
