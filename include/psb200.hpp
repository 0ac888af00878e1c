// psb200.hpp -- header-only C++ adapter: the reference's interface on top of
// the C ABI of psb200.h.
//
// It mirrors, name for name, what lightln2/PuzzleSearch callers use on the
// complete-BFS path:
//   Puzzle (abstract)           Common/Puzzle.h:16-48
//   ExpandHint                  Common/Puzzle.h:11-14
//   ExpandBuffer                Common/Puzzle.h:50-120, Common/Puzzle.cpp:3-13
//   Buffer<T> (the fixed-capacity buffer CrossSegmentPostProcess takes)
//                               Common/Buffer.h:10-60
//   SlidingTilePuzzleSimple     Puzzles/SlidingTilePuzzleSimple.h:8-40
//   SlidingTilePuzzleGpu        Puzzles/SlidingTilePuzzleGpu.h:7-30
//   PancakeSimple               Puzzles/PancakeSimple.h:8-37
//   PancakeOptimized            Puzzles/PancakeOptimized.h:8-52
//   FourPegHanoiSimple          Puzzles/FourPegHanoiSimple.h:8-40
//   FourPegHanoiGPU             Puzzles/FourPegHanoiGPU.h:8-22
//   FourPegHanoiOptimized       Puzzles/FourPegHanoiOptimized.h:8-40
//   InMemoryClassicBFS, InMemoryTwoBitBFS, InMemoryThreeBitBFS,
//   InMemoryFrontierSearch      Common/InMemoryBFS.h:5-11
//   StoreOptions, PuzzleOptions, DiskBased*BFS / *FrontierSearch
//                               Common/Store.h:18-28, Common/DiskBasedBFS.h:9-46
//   HanoiTowers<size>, SearchOptions, HanoiSearch<size>
//                               HanoiTowers/HanoiTowers.h:9-70, HanoiSearch.h:9-18
// so the reference's tests and drivers compile against it by swapping
// includes.  The names live in namespace psb200; define
// PSB200_GLOBAL_NAMES before including to also declare them in the global
// namespace, as the reference does.
//
// The *Gpu classes use the same index spaces as the *Simple ones (n! tile
// permutations, 4^n peg assignments), as in the reference, and so does every
// search here: all of them run on the GPU.
//
// Puzzle is abstract, as in the reference, so callers may derive their own
// puzzles: ExpandBuffer batches work for any Puzzle (it calls the virtual
// Expand), but the InMemory*BFS searches run only on this library's puzzle
// classes, whose expanders are device kernels.  Given any other Puzzle they
// throw psb200::Error with code PSB_ERR_UNSUPPORTED.
//
// Other differences, all on the error path: failures throw psb200::Error (a
// std::runtime_error carrying the C status code) where the reference calls
// ensure() -> exit(-1) or throws std::runtime_error from GPU.cu.
#pragma once

#include <atomic>
#include <chrono>
#include <cstdint>
#include <iostream>
#include <stdexcept>
#include <string>
#include <utility>
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

// Buffer<T> (Common/Buffer.h:10-60): a buffer of fixed capacity whose size
// changes without initialising its elements.
template <typename T>
class Buffer {
public:
    explicit Buffer(size_t capacity) : size_(0), data_(capacity) {}
    size_t Capacity() const { return data_.size(); }
    void SetCapacity(size_t capacity) { data_.resize(capacity); }
    size_t Size() const { return size_; }
    void SetSize(size_t size) {
        if (size > Capacity()) throw Error(PSB_ERR_CAPACITY, "psb200: Buffer size above capacity");
        size_ = size;
    }
    T& operator[](size_t index) { return data_[index]; }
    const T& operator[](size_t index) const { return data_[index]; }
    void Add(T value) { data_[size_++] = value; }
    void Clear() { size_ = 0; }
    bool IsFull() const { return size_ == Capacity(); }
    bool IsEmpty() const { return size_ == 0; }
    T* Buf() { return data_.data(); }
    const T* Buf() const { return data_.data(); }

private:
    size_t size_;
    std::vector<T> data_;
};

// Puzzle (Common/Puzzle.h:16-48): the abstract state space.
class Puzzle {
public:
    static constexpr size_t MAX_INDEXES_BUFFER = 2 * 1024 * 1024;
    static constexpr uint64_t INVALID_INDEX = uint64_t(-1);

    virtual ~Puzzle() = default;

    virtual std::string Name() const = 0;
    virtual int OperatorsCount() const = 0;
    virtual int BranchingFactor() const = 0;
    virtual uint64_t IndexesCount() const = 0;
    virtual bool HasOddLengthCycles() const = 0;

    virtual std::string ToString(uint64_t index) = 0;

    virtual uint64_t Parse(std::string state) = 0;

    virtual void Expand(std::vector<uint64_t>& indexes, std::vector<int>& usedOperatorBits,
                        std::vector<uint64_t>& expandedIndexes, std::vector<int>& expandedOperators,
                        ExpandHint hint) = 0;

    // Only the reference's segmented disk drivers call this; a no-op by default.
    virtual void CrossSegmentPostProcess(int op, int segment, int segmentBits, Buffer<uint32_t>& expandedIndexes) {
        (void)op, (void)segment, (void)segmentBits, (void)expandedIndexes;
    }

    // This library's handle when the puzzle is one of its device classes;
    // NULL for puzzles defined elsewhere (the searches reject those).
    virtual const psb_puzzle* handle() const { return nullptr; }

protected:
    // Common/Puzzle.cpp:15-26: room for a full batch's children, then empty.
    virtual void SetupOutputBuffers(std::vector<uint64_t>& expandedIndexes, std::vector<int>& expandedOperators) {
        const size_t capacity = MAX_INDEXES_BUFFER * size_t(BranchingFactor());
        if (expandedIndexes.capacity() < capacity) expandedIndexes.reserve(capacity);
        if (expandedOperators.capacity() < capacity) expandedOperators.reserve(capacity);
        expandedIndexes.clear();
        expandedOperators.clear();
    }
};

// The library's puzzles: every method goes through the C ABI, Expand runs the
// device expander, and the searches run on the GPU.
class DevicePuzzle : public Puzzle {
public:
    DevicePuzzle(const DevicePuzzle&) = delete;
    DevicePuzzle& operator=(const DevicePuzzle&) = delete;
    ~DevicePuzzle() override { psb_puzzle_destroy(h_); }

    std::string Name() const override {
        char buf[256];
        check(psb_puzzle_name(h_, buf, sizeof buf));
        return buf;
    }
    int OperatorsCount() const override { return ops_; }
    int BranchingFactor() const override { return branching_; }
    uint64_t IndexesCount() const override { return n_; }
    bool HasOddLengthCycles() const override { return odd_ != 0; }

    std::string ToString(uint64_t index) override {
        char buf[512];
        check(psb_to_string(h_, index, buf, sizeof buf));
        return buf;
    }

    uint64_t Parse(std::string state) override {
        uint64_t idx = 0;
        check(psb_parse(h_, state.c_str(), &idx));
        return idx;
    }

    // Puzzle::Expand: children appended in the reference's order; like
    // SetupOutputBuffers (Common/Puzzle.cpp:15-26) the outputs are cleared
    // first.  The hint only matters to the reference's segmented disk
    // drivers, which this library does not provide.
    void Expand(std::vector<uint64_t>& indexes, std::vector<int>& usedOperatorBits,
                std::vector<uint64_t>& expandedIndexes, std::vector<int>& expandedOperators,
                ExpandHint hint = {}) override {
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

    const psb_puzzle* handle() const override { return h_; }

protected:
    DevicePuzzle(int kind, int a, int b) {
        check(psb_puzzle_create(kind, a, b, &h_));
        check(psb_puzzle_info(h_, &n_, &ops_, &branching_, &odd_));
    }

private:
    psb_puzzle* h_ = nullptr;
    uint64_t n_ = 0;
    int ops_ = 0, branching_ = 0, odd_ = 0;
};

class SlidingTilePuzzleSimple : public DevicePuzzle {
public:
    SlidingTilePuzzleSimple(int width, int height) : DevicePuzzle(PSB_SLIDING, width, height) {}
};

// The reference's GPU sliding-tile class: the same n! index space as the
// Simple class.
class SlidingTilePuzzleGpu : public DevicePuzzle {
public:
    SlidingTilePuzzleGpu(int width, int height)
        : DevicePuzzle(PSB_SLIDING, width, height), width_(width), height_(height) {}
    std::string Name() const override {
        return "Sliding-Tile GPU: " + std::to_string(width_) + " x " + std::to_string(height_);
    }

private:
    int width_, height_;
};

// SlidingTilePuzzleOptimized<width, height> (Puzzles/SlidingTilePuzzleOptimized.h:
// 13-53): the sliding-tile puzzle in the reference's packed index (the tiles'
// left-smaller digits, the blank in the low nibble; 16 * (cells-1)!/2 indexes
// up to 13 cells, segments of 2^32 above).
template <int width, int height>
class SlidingTilePuzzleOptimized : public DevicePuzzle {
public:
    static constexpr int size = width * height;
    SlidingTilePuzzleOptimized() : DevicePuzzle(PSB_SLIDING_OPT, width, height) {}
};

class PancakeSimple : public DevicePuzzle {
public:
    explicit PancakeSimple(int size) : DevicePuzzle(PSB_PANCAKE, size, 0) {}
};

// PancakeOptimized (Puzzles/PancakeOptimized.h:8-52): the pancake puzzle in
// the reference's GPU pancake index (a 29-bit split above 11 pancakes).
// inverseIndex only affects CrossSegmentPostProcess in the reference's
// segmented drivers; it is kept and reported by Name().
class PancakeOptimized : public DevicePuzzle {
public:
    explicit PancakeOptimized(int size, bool inverseIndex = false)
        : DevicePuzzle(PSB_PANCAKE_OPT, size, inverseIndex ? 1 : 0), size_(size), inv_(inverseIndex) {}
    int Size() const { return size_; }
    bool InvIndex() const { return inv_; }

private:
    int size_;
    bool inv_;
};

class FourPegHanoiSimple : public DevicePuzzle {
public:
    explicit FourPegHanoiSimple(int size, bool useSymmetry = false)
        : DevicePuzzle(PSB_HANOI4, size, useSymmetry ? 1 : 0), size_(size), sym_(useSymmetry) {}
    int Size() const { return size_; }
    bool UseSymmetry() const { return sym_; }

private:
    int size_;
    bool sym_;
};

// FourPegHanoiOptimized (Puzzles/FourPegHanoiOptimized.h:8-40): the Simple
// class's index space; with symmetry the peg order is restored only when a
// move empties or fills a peg (the same children for every reachable state).
class FourPegHanoiOptimized : public DevicePuzzle {
public:
    explicit FourPegHanoiOptimized(int size, bool useSymmetry = false)
        : DevicePuzzle(PSB_HANOI4_OPT, size, useSymmetry ? 1 : 0), size_(size), sym_(useSymmetry) {}
    int Size() const { return size_; }
    bool UseSymmetry() const { return sym_; }

private:
    int size_;
    bool sym_;
};

// The reference's GPU Hanoi class: the Simple class's 4^n index space, at
// most 24 disks (Puzzles/FourPegHanoiGPU.h:10-14).
class FourPegHanoiGPU : public DevicePuzzle {
public:
    FourPegHanoiGPU(int size, bool useSymmetry)
        : DevicePuzzle(PSB_HANOI4, checked_size(size), useSymmetry ? 1 : 0), size_(size), sym_(useSymmetry) {}
    std::string Name() const override {
        return "Four-Peg Hanoi Towers (GPU), size=" + std::to_string(size_) + "; symmetry=" + std::to_string(int(sym_));
    }

private:
    static int checked_size(int size) {
        if (size > 24) throw Error(PSB_ERR_ARG, "psb200: FourPegHanoiGPU holds at most 24 disks");
        return size;
    }
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

    // Expand batches, parents and time over all buffers (Common/Puzzle.cpp:7-13).
    static void PrintStats() {
        std::cerr << "Expand: " << stats().times.load() << " times, " << stats().nodes.load() << " nodes in "
                  << stats().nanos.load() / 1000000 << " ms" << std::endl;
    }

private:
    struct Stats {
        std::atomic<uint64_t> nodes{0}, nanos{0}, times{0};
    };
    static Stats& stats() {
        static Stats s;
        return s;
    }
    template <typename F>
    void Expand(F func) {
        const auto t0 = std::chrono::steady_clock::now();
        puzzle_.Expand(indexes_, ops_, children_, child_ops_, hint_);
        stats().times++;
        stats().nodes += indexes_.size();
        stats().nanos += uint64_t(
            std::chrono::duration_cast<std::chrono::nanoseconds>(std::chrono::steady_clock::now() - t0).count());
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

// StoreOptions (Common/Store.h:18-28) and PuzzleOptions (Common/DiskBasedBFS.h:
// 9-14).  The segmented searches keep their segment data in host memory:
// directories and filesPerPath are accepted and unused, and so is threads
// (the GPU runs each segment's work); segmentBits and maxSteps apply.
struct StoreOptions {
    std::vector<std::string> directories = {"."};
    int filesPerPath = 5;
};
struct PuzzleOptions {
    size_t maxSteps = 10000;
    int segmentBits = 32;
    int threads = 1;
    StoreOptions storeOptions;
};

// The reference's disk-based searches (Common/DiskBasedBFS.h:40-46) all
// return the per-depth counts of the whole space; here each is the segmented
// out-of-core search of psb_bfs_segmented (one segment's arrays on the
// device at a time, DiskBasedOptThreeBitBFS's three-layer scheme), whose
// segment files go to opts.storeOptions.directories (filesPerPath files of
// consecutive segments per directory) as the reference's do; an empty
// directory list keeps them in host memory.
inline std::vector<uint64_t> RunSegmented(Puzzle& puzzle, const std::string& initialState, const PuzzleOptions& opts) {
    if (!puzzle.handle())
        throw Error(PSB_ERR_UNSUPPORTED, "psb200: the segmented searches run on the GPU for this library's puzzle "
                                         "classes only; '" + puzzle.Name() + "' has no device expander");
    const uint64_t init = puzzle.Parse(initialState);
    psb_segmented_opts o{};
    o.struct_size = sizeof(psb_segmented_opts);
    o.segment_bits = opts.segmentBits;
    o.device = -1;
    o.max_depth = opts.maxSteps < 10000 ? uint32_t(opts.maxSteps) : 0;
    std::vector<const char*> dirs;
    for (const std::string& d : opts.storeOptions.directories) dirs.push_back(d.c_str());
    o.directories = dirs.empty() ? nullptr : dirs.data();
    o.n_directories = int32_t(dirs.size());
    o.files_per_path = opts.storeOptions.filesPerPath;
    std::vector<uint64_t> counts(1 << 16);
    uint32_t n = 0;
    check(psb_bfs_segmented(puzzle.handle(), init, &o, counts.data(), uint32_t(counts.size()), &n, nullptr));
    counts.resize(n);
    return counts;
}
inline std::vector<uint64_t> DiskBasedClassicBFS(Puzzle& puzzle, std::string initialState, PuzzleOptions opts = {}) {
    return RunSegmented(puzzle, initialState, opts);
}
inline std::vector<uint64_t> DiskBasedTwoBitBFS(Puzzle& puzzle, std::string initialState, PuzzleOptions opts = {}) {
    return RunSegmented(puzzle, initialState, opts);
}
inline std::vector<uint64_t> DiskBasedThreeBitBFS(Puzzle& puzzle, std::string initialState, PuzzleOptions opts = {}) {
    return RunSegmented(puzzle, initialState, opts);
}
inline std::vector<uint64_t> DiskBasedFrontierSearch(Puzzle& puzzle, std::string initialState,
                                                     PuzzleOptions opts = {}) {
    return RunSegmented(puzzle, initialState, opts);
}
inline std::vector<uint64_t> DiskBasedOptFrontierSearch(Puzzle& puzzle, std::string initialState,
                                                        PuzzleOptions opts = {}) {
    return RunSegmented(puzzle, initialState, opts);
}
inline std::vector<uint64_t> DiskBasedOptThreeBitBFS(Puzzle& puzzle, std::string initialState,
                                                     PuzzleOptions opts = {}) {
    return RunSegmented(puzzle, initialState, opts);
}
inline std::vector<uint64_t> DiskBasedOptThreeBitBFS2(Puzzle& puzzle, std::string initialState,
                                                      PuzzleOptions opts = {}) {
    return RunSegmented(puzzle, initialState, opts);
}

// HanoiTowers<size> (HanoiTowers/HanoiTowers.h:9-70): the index space of the
// reference's symmetric 4-peg Hanoi search: 2 bits per disk, the same layout
// and ToString/Parse format as FourPegHanoiSimple.
template <int size>
class HanoiTowers {
public:
    static constexpr int Size = size;
    static uint64_t IndexesCount() { return uint64_t(1) << (size * 2); }
    static int MaxSegments() { return int((IndexesCount() + 0xFFFFFFFFull) >> 32); }
    static std::string ToString(uint64_t index) { return FourPegHanoiSimple(size, true).ToString(index); }
    static uint64_t Parse(std::string state) { return FourPegHanoiSimple(size, true).Parse(state); }
    static std::pair<int, uint32_t> SplitIndex(uint64_t index) { return {int(index >> 32), uint32_t(index)}; }
    // Size of the symmetry class of a canonical state (pegs 1..3 ordered by
    // their bottom disk): 6 with disks on pegs 1 and 2, 3 with disks on peg 1 only.
    static int PegsMult(uint64_t index) {
        const uint64_t even = 0x5555555555555555ull, hi = index >> 1, lo = index;
        const uint64_t pegs1 = ~hi & lo & even, pegs2 = hi & ~lo & even;
        return 6 - int(pegs2 == 0) * 3 - int(pegs1 == 0);
    }
};

// SearchOptions (HanoiTowers/HanoiSearch.h:9-13).  The search runs in device
// memory: threads and directories (the reference's disk stores) are accepted
// and unused; maxSteps bounds the depth.
struct SearchOptions {
    int maxSteps = 1000000;
    int threads = 4;
    std::vector<std::string> directories = {"."};
};

// HanoiSearch<size> (HanoiTowers/HanoiSearch.cpp:204-290): BFS over the
// symmetric 4-peg Hanoi space from initialState; entry d is the number of
// states at depth d of the full (unreduced) space: each canonical state
// counts PegsMult times, depth 0 counts 1.  A two-bit search on the GPU.
template <int size>
std::vector<uint64_t> HanoiSearch(std::string initialState, SearchOptions options = {}) {
    FourPegHanoiSimple puzzle(size, true);
    const uint64_t init = puzzle.Parse(initialState);
    std::vector<uint64_t> counts(1 << 16), restored(1 << 16);
    psb_bfs_opts o{};
    o.struct_size = sizeof(psb_bfs_opts);
    o.device = -1;
    o.max_depth = options.maxSteps > 0 && options.maxSteps < 1000000 ? uint32_t(options.maxSteps) : 0;
    o.restored_counts = restored.data();
    uint32_t n = 0;
    check(psb_bfs(puzzle.handle(), PSB_TWO_BIT, init, &o, counts.data(), uint32_t(counts.size()), &n, nullptr));
    restored.resize(n);
    return restored;
}

// In-memory searches (Common/InMemoryBFS.h:5-11): the whole search runs on
// the GPU with the bit arrays resident in device memory; the result is the
// number of states at each depth, element 0 = 1 (the initial state).
inline std::vector<uint64_t> RunInMemory(Puzzle& puzzle, int algo, const std::string& initialState,
                                         const psb_bfs_opts* opts = nullptr, psb_bfs_stats* stats = nullptr) {
    if (!puzzle.handle())
        throw Error(PSB_ERR_UNSUPPORTED, "psb200: the in-memory searches run on the GPU for this library's puzzle "
                                         "classes only; '" + puzzle.Name() + "' has no device expander");
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
using psb200::Buffer;
using psb200::DiskBasedClassicBFS;
using psb200::DiskBasedFrontierSearch;
using psb200::DiskBasedOptFrontierSearch;
using psb200::DiskBasedOptThreeBitBFS;
using psb200::DiskBasedOptThreeBitBFS2;
using psb200::DiskBasedThreeBitBFS;
using psb200::DiskBasedTwoBitBFS;
using psb200::ExpandBuffer;
using psb200::ExpandHint;
using psb200::FourPegHanoiGPU;
using psb200::FourPegHanoiOptimized;
using psb200::FourPegHanoiSimple;
using psb200::HanoiSearch;
using psb200::HanoiTowers;
using psb200::InMemoryClassicBFS;
using psb200::InMemoryFrontierSearch;
using psb200::InMemoryThreeBitBFS;
using psb200::InMemoryTwoBitBFS;
using psb200::PancakeOptimized;
using psb200::PancakeSimple;
using psb200::Puzzle;
using psb200::PuzzleOptions;
using psb200::SearchOptions;
using psb200::SlidingTilePuzzleGpu;
using psb200::SlidingTilePuzzleOptimized;
using psb200::SlidingTilePuzzleSimple;
using psb200::StoreOptions;
#endif
