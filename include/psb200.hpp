// psb200.hpp -- header-only C++ adapter: the reference's interface on top of
// the C ABI of psb200.h.
//
// It mirrors, name for name, what lightln2/PuzzleSearch callers use on the
// complete-BFS path:
//   Puzzle                      Common/Puzzle.h:16-48
//   ExpandHint                  Common/Puzzle.h:11-14
//   ExpandBuffer                Common/Puzzle.h:50-120
//   SlidingTilePuzzleSimple     Puzzles/SlidingTilePuzzleSimple.h:8-40
//   PancakeSimple               Puzzles/PancakeSimple.h:8-37
//   FourPegHanoiSimple          Puzzles/FourPegHanoiSimple.h:8-40
//   InMemoryClassicBFS, InMemoryTwoBitBFS, InMemoryThreeBitBFS,
//   InMemoryFrontierSearch      Common/InMemoryBFS.h:5-11
// so the reference's tests and drivers compile against it by swapping
// includes.  The names live in namespace psb200; define
// PSB200_GLOBAL_NAMES before including to also declare them in the global
// namespace, as the reference does.
//
// Differences, all on the error path: failures throw psb200::Error (a
// std::runtime_error carrying the C status code) where the reference calls
// ensure() -> exit(-1) or throws std::runtime_error from GPU.cu.
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "psb200.h"

namespace psb200 {

class Error : public std::runtime_error {
public:
    Error(int code, const std::string& msg) : std::runtime_error(msg), code_(code) {}
    int code() const { return code_; }

private:
    int code_;
};

inline void check(int rc) {
    if (rc < 0) {
        char buf[512] = {0};
        psb_last_error(buf, sizeof buf);
        throw Error(rc, std::string("psb200: ") + buf);
    }
}

struct ExpandHint {
    int SegmentBits = 0;
    bool CrossSegment = false;
};

class Puzzle {
public:
    static constexpr size_t MAX_INDEXES_BUFFER = 2 * 1024 * 1024;
    static constexpr uint64_t INVALID_INDEX = uint64_t(-1);

    Puzzle(const Puzzle&) = delete;
    Puzzle& operator=(const Puzzle&) = delete;
    virtual ~Puzzle() { psb_puzzle_destroy(h_); }

    std::string Name() const {
        char buf[256];
        check(psb_puzzle_name(h_, buf, sizeof buf));
        return buf;
    }
    int OperatorsCount() const { return ops_; }
    int BranchingFactor() const { return branching_; }
    uint64_t IndexesCount() const { return n_; }
    bool HasOddLengthCycles() const { return odd_ != 0; }

    std::string ToString(uint64_t index) {
        char buf[512];
        check(psb_to_string(h_, index, buf, sizeof buf));
        return buf;
    }

    uint64_t Parse(std::string state) {
        uint64_t idx = 0;
        check(psb_parse(h_, state.c_str(), &idx));
        return idx;
    }

    // Puzzle::Expand: children appended in the reference's order; like
    // SetupOutputBuffers (Common/Puzzle.cpp:15-26) the outputs are cleared
    // first.  The hint only matters to the reference's segmented disk
    // drivers, which this library does not provide.
    void Expand(std::vector<uint64_t>& indexes, std::vector<int>& usedOperatorBits,
                std::vector<uint64_t>& expandedIndexes, std::vector<int>& expandedOperators, ExpandHint hint = {}) {
        (void)hint;
        const size_t n = indexes.size();
        if (!usedOperatorBits.empty() && usedOperatorBits.size() != n)
            throw Error(PSB_ERR_ARG, "psb200: usedOperatorBits and indexes differ in size");
        expandedIndexes.assign(n * size_t(branching_), 0);
        std::vector<uint32_t> ops(n * size_t(branching_));
        std::vector<uint32_t> used(usedOperatorBits.begin(), usedOperatorBits.end());
        uint64_t n_out = 0;
        uint32_t flags = PSB_EXPAND_HOST_POINTERS | PSB_EXPAND_COMPACT;
        if (!used.empty()) flags |= PSB_EXPAND_USE_OPBITS;
        check(psb_expand(h_, indexes.data(), used.empty() ? nullptr : used.data(), n, expandedIndexes.data(),
                         ops.data(), expandedIndexes.size(), &n_out, flags, nullptr));
        expandedIndexes.resize(n_out);
        expandedOperators.assign(ops.begin(), ops.begin() + n_out);
    }

    const psb_puzzle* handle() const { return h_; }

protected:
    Puzzle(int kind, int a, int b) {
        check(psb_puzzle_create(kind, a, b, &h_));
        check(psb_puzzle_info(h_, &n_, &ops_, &branching_, &odd_));
    }

private:
    psb_puzzle* h_ = nullptr;
    uint64_t n_ = 0;
    int ops_ = 0, branching_ = 0, odd_ = 0;
};

class SlidingTilePuzzleSimple : public Puzzle {
public:
    SlidingTilePuzzleSimple(int width, int height) : Puzzle(PSB_SLIDING, width, height) {}
};

class PancakeSimple : public Puzzle {
public:
    explicit PancakeSimple(int size) : Puzzle(PSB_PANCAKE, size, 0) {}
};

class FourPegHanoiSimple : public Puzzle {
public:
    explicit FourPegHanoiSimple(int size, bool useSymmetry = false)
        : Puzzle(PSB_HANOI4, size, useSymmetry ? 1 : 0), size_(size), sym_(useSymmetry) {}
    int Size() const { return size_; }
    bool UseSymmetry() const { return sym_; }

private:
    int size_;
    bool sym_;
};

// ExpandBuffer (Common/Puzzle.h:50-120): collects parents, expands them in
// batches of MAX_INDEXES_BUFFER on the GPU and calls func(child, op) for
// every valid child.
class ExpandBuffer {
public:
    explicit ExpandBuffer(Puzzle& puzzle) : puzzle_(puzzle) {
        indexes_.reserve(Puzzle::MAX_INDEXES_BUFFER);
        ops_.reserve(Puzzle::MAX_INDEXES_BUFFER);
    }
    void SetExpandHint(int segmentBits, bool crossSegment) {
        hint_.SegmentBits = segmentBits;
        hint_.CrossSegment = crossSegment;
    }
    template <typename F>
    void Add(uint64_t index, int usedOperatorBits, F func) {
        indexes_.push_back(index);
        ops_.push_back(usedOperatorBits);
        if (indexes_.size() == Puzzle::MAX_INDEXES_BUFFER) Expand(func);
    }
    template <typename F>
    void Finish(F func) {
        if (!indexes_.empty()) Expand(func);
        SetExpandHint(0, false);
    }

private:
    template <typename F>
    void Expand(F func) {
        puzzle_.Expand(indexes_, ops_, children_, child_ops_, hint_);
        for (size_t i = 0; i < children_.size(); i++)
            if (children_[i] != Puzzle::INVALID_INDEX) func(children_[i], child_ops_[i]);
        indexes_.clear();
        ops_.clear();
    }
    Puzzle& puzzle_;
    ExpandHint hint_;
    std::vector<uint64_t> indexes_, children_;
    std::vector<int> ops_, child_ops_;
};

// In-memory searches (Common/InMemoryBFS.h:5-11): the whole search runs on
// the GPU with the bit arrays resident in device memory; the result is the
// number of states at each depth, element 0 = 1 (the initial state).
inline std::vector<uint64_t> RunInMemory(Puzzle& puzzle, int algo, const std::string& initialState,
                                         const psb_bfs_opts* opts = nullptr, psb_bfs_stats* stats = nullptr) {
    const uint64_t init = puzzle.Parse(initialState);
    std::vector<uint64_t> counts(1 << 16);
    uint32_t n = 0;
    check(psb_bfs(puzzle.handle(), algo, init, opts, counts.data(), uint32_t(counts.size()), &n, stats));
    counts.resize(n);
    return counts;
}

inline std::vector<uint64_t> InMemoryClassicBFS(Puzzle& puzzle, std::string initialState) {
    return RunInMemory(puzzle, PSB_CLASSIC, initialState);
}
inline std::vector<uint64_t> InMemoryTwoBitBFS(Puzzle& puzzle, std::string initialState) {
    return RunInMemory(puzzle, PSB_TWO_BIT, initialState);
}
inline std::vector<uint64_t> InMemoryThreeBitBFS(Puzzle& puzzle, std::string initialState) {
    return RunInMemory(puzzle, PSB_THREE_BIT, initialState);
}
inline std::vector<uint64_t> InMemoryFrontierSearch(Puzzle& puzzle, std::string initialState) {
    return RunInMemory(puzzle, PSB_FRONTIER, initialState);
}

}  // namespace psb200

#ifdef PSB200_GLOBAL_NAMES
using psb200::ExpandBuffer;
using psb200::ExpandHint;
using psb200::FourPegHanoiSimple;
using psb200::InMemoryClassicBFS;
using psb200::InMemoryFrontierSearch;
using psb200::InMemoryThreeBitBFS;
using psb200::InMemoryTwoBitBFS;
using psb200::PancakeSimple;
using psb200::Puzzle;
using psb200::SlidingTilePuzzleSimple;
#endif
