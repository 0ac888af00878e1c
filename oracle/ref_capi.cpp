// ref_capi.cpp -- C ABI over the reference's own CPU classes (test
// infrastructure only).  Compiled by oracle/build_ref.sh together with the
// reference's sources (Common/InMemory*.cpp, Puzzles/*Simple.cpp,
// Common/StreamVInt.cpp, Common/FrontierCompression.cpp) into
// oracle/_ref/libpsbref.so.  Used by tests to pin the oracle restatement and
// by bench.py --impl reference for the CPU baseline.
#include "Common/InMemoryBFS.h"
#include "Common/FrontierCompression.h"
#include "Common/OpBitsCompression.h"
#include "Common/StreamVInt.h"
#include "Puzzles/FourPegHanoiOptimized.h"
#include "Puzzles/FourPegHanoiSimple.h"
#include "Puzzles/PancakeOptimized.h"
#include "Puzzles/PancakeSimple.h"
#include "Puzzles/PermutationMap.h"
#include "Puzzles/SlidingTilePuzzleOptimized.h"
#include "Puzzles/SlidingTilePuzzleSimple.h"

#include <cstring>
#include <iostream>
#include <memory>
#include <string>
#include <vector>

namespace {

// The shapes the reference instantiates (SlidingTilePuzzleOptimized.cpp:293-307).
// Only their Parse / ToString / IndexesCount run here: their Expand needs the
// reference's CUDA kernel (see ref_gpu_stubs.cpp).
std::unique_ptr<Puzzle> MakeSlidingOptimized(int w, int h) {
    switch (w * 16 + h) {
    case 0x22: return std::make_unique<SlidingTilePuzzleOptimized<2, 2>>();
    case 0x32: return std::make_unique<SlidingTilePuzzleOptimized<3, 2>>();
    case 0x42: return std::make_unique<SlidingTilePuzzleOptimized<4, 2>>();
    case 0x52: return std::make_unique<SlidingTilePuzzleOptimized<5, 2>>();
    case 0x62: return std::make_unique<SlidingTilePuzzleOptimized<6, 2>>();
    case 0x72: return std::make_unique<SlidingTilePuzzleOptimized<7, 2>>();
    case 0x82: return std::make_unique<SlidingTilePuzzleOptimized<8, 2>>();
    case 0x33: return std::make_unique<SlidingTilePuzzleOptimized<3, 3>>();
    case 0x43: return std::make_unique<SlidingTilePuzzleOptimized<4, 3>>();
    case 0x53: return std::make_unique<SlidingTilePuzzleOptimized<5, 3>>();
    case 0x44: return std::make_unique<SlidingTilePuzzleOptimized<4, 4>>();
    }
    return nullptr;
}

std::unique_ptr<Puzzle> MakePuzzle(int kind, int a, int b) {
    switch (kind) {
    case 1: return std::make_unique<SlidingTilePuzzleSimple>(a, b);
    case 2: return std::make_unique<PancakeSimple>(a);
    case 3: return std::make_unique<FourPegHanoiSimple>(a, b != 0);
    case 4: return std::make_unique<PancakeOptimized>(a, b != 0);
    case 5: return std::make_unique<FourPegHanoiOptimized>(a, b != 0);
    case 6: return MakeSlidingOptimized(a, b);
    }
    return nullptr;
}

// Forwards to a Simple puzzle and records every parent handed to Expand
// (the reference's frontier sets, level after level).
class RecordingPuzzle : public Puzzle {
public:
    explicit RecordingPuzzle(Puzzle& inner) : inner(inner) {}
    std::string Name() const override { return inner.Name(); }
    int OperatorsCount() const override { return inner.OperatorsCount(); }
    int BranchingFactor() const override { return inner.BranchingFactor(); }
    uint64_t IndexesCount() const override { return inner.IndexesCount(); }
    bool HasOddLengthCycles() const override { return inner.HasOddLengthCycles(); }
    std::string ToString(uint64_t index) override { return inner.ToString(index); }
    uint64_t Parse(std::string state) override { return inner.Parse(state); }
    void Expand(std::vector<uint64_t>& indexes, std::vector<int>& ops, std::vector<uint64_t>& ci,
                std::vector<int>& co, ExpandHint hint) override {
        parents.insert(parents.end(), indexes.begin(), indexes.end());
        inner.Expand(indexes, ops, ci, co, hint);
    }
    std::vector<uint64_t> parents;

private:
    Puzzle& inner;
};

struct QuietCerr {
    std::streambuf* saved;
    QuietCerr() : saved(std::cerr.rdbuf(nullptr)) {}
    ~QuietCerr() { std::cerr.rdbuf(saved); std::cerr.clear(); }
};

std::vector<uint64_t> RunBfs(Puzzle& puzzle, int algo, const std::string& init) {
    switch (algo) {
    case 1: return InMemoryTwoBitBFS(puzzle, init);
    case 2: return InMemoryThreeBitBFS(puzzle, init);
    case 3: return InMemoryFrontierSearch(puzzle, init);
    case 4: return InMemoryClassicBFS(puzzle, init);
    }
    return {};
}

}  // namespace

extern "C" {

int ref_bfs(int kind, int a, int b, int algo, const char* init, uint64_t* counts, int cap, int quiet) {
    auto puzzle = MakePuzzle(kind, a, b);
    if (!puzzle) return -1;
    std::vector<uint64_t> r;
    if (quiet) { QuietCerr q; r = RunBfs(*puzzle, algo, init); }
    else r = RunBfs(*puzzle, algo, init);
    if ((int)r.size() > cap) return -2;
    std::copy(r.begin(), r.end(), counts);
    return (int)r.size();
}

// Runs a BFS through RecordingPuzzle; returns the number of recorded parents
// (all of them, in expansion order) or -2 if cap is too small.
int64_t ref_bfs_parents(int kind, int a, int b, int algo, const char* init, uint64_t* parents, uint64_t cap) {
    auto puzzle = MakePuzzle(kind, a, b);
    if (!puzzle) return -1;
    RecordingPuzzle rec(*puzzle);
    { QuietCerr q; RunBfs(rec, algo, init); }
    if (rec.parents.size() > cap) return -2;
    std::copy(rec.parents.begin(), rec.parents.end(), parents);
    return (int64_t)rec.parents.size();
}

int64_t ref_expand(int kind, int a, int b, const uint64_t* parents, const uint32_t* opbits, uint64_t n,
                   uint64_t* children, uint32_t* ops, uint64_t cap) {
    auto puzzle = MakePuzzle(kind, a, b);
    if (!puzzle) return -1;
    std::vector<uint64_t> idx(parents, parents + n), ci;
    std::vector<int> ob(n), co;
    for (uint64_t i = 0; i < n; i++) ob[i] = opbits ? (int)opbits[i] : 0;
    try {
        puzzle->Expand(idx, ob, ci, co, {});
    } catch (const std::exception&) {
        return -3;  // an Expand that needs the GPU
    }
    if (ci.size() > cap) return -2;
    for (size_t i = 0; i < ci.size(); i++) { children[i] = ci[i]; ops[i] = (uint32_t)co[i]; }
    return (int64_t)ci.size();
}

uint64_t ref_indexes_count(int kind, int a, int b) {
    auto puzzle = MakePuzzle(kind, a, b);
    return puzzle ? puzzle->IndexesCount() : 0;
}

int ref_parse(int kind, int a, int b, const char* state, uint64_t* index) {
    auto puzzle = MakePuzzle(kind, a, b);
    if (!puzzle) return -1;
    *index = puzzle->Parse(state);
    return 0;
}

int ref_to_string(int kind, int a, int b, uint64_t index, char* buf, int cap) {
    auto puzzle = MakePuzzle(kind, a, b);
    if (!puzzle) return -1;
    std::string s = puzzle->ToString(index);
    if ((int)s.size() + 1 > cap) return -2;
    std::memcpy(buf, s.c_str(), s.size() + 1);
    return (int)s.size();
}

uint64_t ref_perm_rank(const int* arr, int size) {
    int tmp[16];
    std::memcpy(tmp, arr, sizeof(int) * size);
    return PermutationRank(tmp, size);
}

void ref_perm_unrank(uint64_t index, int* arr, int size) { PermutationUnrank(index, arr, size); }

int ref_svi_encode_tuple(const uint32_t* v, uint8_t* out) {
    uint8_t tmp[32] = {0};
    int n = StreamVInt::EncodeTuple(v, tmp);
    std::memcpy(out, tmp, n);
    return n;
}

// indexes must hold round8(count) slots; out must hold >= 1 MiB (the
// reference asserts MAX_BUFFER_SIZE capacity).
int ref_svi_encode(int count, uint32_t* indexes, uint8_t* out, int out_cap) {
    return StreamVInt::Encode(count, indexes, out, out_cap);
}

int ref_svi_decode(int* size, uint8_t* in, uint32_t* indexes, int cap) {
    return StreamVInt::Decode(*size, in, indexes, cap);
}

int ref_svi_encode_bounds(int count, uint32_t* indexes, uint8_t* bounds, uint8_t* out, int out_cap) {
    return StreamVInt::Encode(count, indexes, bounds, out, out_cap);
}

int ref_fc_encode(int count, uint32_t* indexes, uint8_t* out, int out_cap) {
    return FrontierCompression::Encode(count, indexes, out, out_cap);
}

int ref_fc_encode_with_check(int count, uint32_t* indexes, uint8_t* out, int out_cap) {
    return FrontierCompression::EncodeWithCheck(count, indexes, out, out_cap);
}

int ref_fc_decode(int* size, uint8_t* in, uint32_t* indexes, int cap) {
    return FrontierCompression::Decode(*size, in, indexes, cap);
}

int64_t ref_opbits_encode(int bits, uint64_t count, const uint8_t* ops, uint8_t* out) {
    switch (bits) {
    case 2: return int64_t(OpBitsCompression<2>::Encode(count, ops, out));
    case 4: return int64_t(OpBitsCompression<4>::Encode(count, ops, out));
    case 8: return int64_t(OpBitsCompression<8>::Encode(count, ops, out));
    }
    return -1;
}

}  // extern "C"
