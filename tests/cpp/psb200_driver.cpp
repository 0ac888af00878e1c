// psb200_driver.cpp -- exercises include/psb200.hpp the way the reference's
// tests use its classes (PuzzlesTests/PuzzleSearchTests.cpp, PancakeTest.cpp,
// FourPegHanoiTest.cpp).  Reads commands on stdin, one per line:
//   bfs <kind> <a> <b> <classic|two_bit|three_bit|frontier> <state...>
//   expand <kind> <a> <b> <state...>
//   custom <n>
//   hanoisearch <disks 8..19> <maxSteps>
//   disk <kind> <a> <b> <Classic|TwoBit|ThreeBit|FrontierSearch|OptFrontierSearch|OptThreeBit> <segmentBits> <threads> <state...>
// with kind one of sliding, sliding_gpu, sliding_opt, pancake, pancake_opt, hanoi4, hanoi4_gpu, hanoi4_opt (the
// *_gpu kinds construct the reference's GPU class names,
// SlidingTilePuzzleGpu and FourPegHanoiGPU), and prints one result line per
// command (space-separated counts, or "child-state|op" items separated by
// ';').  `hanoisearch` runs HanoiSearch<disks> from all disks on peg 0, as
// the reference's HanoiSearchTests do.  `custom` drives a Puzzle subclass
// defined here, as a caller would:
// it prints the number of children ExpandBuffer delivers over all n states,
// then what InMemoryTwoBitBFS does with it.  tests/test_gpu_cpp_adapter.py
// feeds it the reference's golden vectors.
#define PSB200_GLOBAL_NAMES
#include "../../include/psb200.hpp"

#include <iostream>
#include <memory>
#include <sstream>
#include <string>

// SlidingTilePuzzleOptimized<w, h> for the shapes the reference builds it for.
static std::unique_ptr<Puzzle> make_sliding_opt(int w, int h) {
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
    throw std::runtime_error("no SlidingTilePuzzleOptimized<" + std::to_string(w) + ", " + std::to_string(h) + ">");
}

static std::unique_ptr<Puzzle> make(const std::string& kind, int a, int b) {
    if (kind == "sliding") return std::make_unique<SlidingTilePuzzleSimple>(a, b);
    if (kind == "sliding_opt") return make_sliding_opt(a, b);
    if (kind == "sliding_gpu") return std::make_unique<SlidingTilePuzzleGpu>(a, b);
    if (kind == "pancake") return std::make_unique<PancakeSimple>(a);
    if (kind == "pancake_opt") return std::make_unique<PancakeOptimized>(a, b != 0);
    if (kind == "hanoi4_gpu") return std::make_unique<FourPegHanoiGPU>(a, b != 0);
    if (kind == "hanoi4_opt") return std::make_unique<FourPegHanoiOptimized>(a, b != 0);
    return std::make_unique<FourPegHanoiSimple>(a, b != 0);
}

// A caller's own puzzle: n states on a ring, two moves each (i-1 and i+1).
class RingPuzzle : public Puzzle {
public:
    explicit RingPuzzle(uint64_t n) : n_(n) {}
    std::string Name() const override { return "ring of " + std::to_string(n_); }
    int OperatorsCount() const override { return 2; }
    int BranchingFactor() const override { return 2; }
    uint64_t IndexesCount() const override { return n_; }
    bool HasOddLengthCycles() const override { return n_ % 2 == 1; }
    std::string ToString(uint64_t index) override { return std::to_string(index); }
    uint64_t Parse(std::string state) override { return std::stoull(state); }
    void Expand(std::vector<uint64_t>& indexes, std::vector<int>& usedOperatorBits,
                std::vector<uint64_t>& expandedIndexes, std::vector<int>& expandedOperators, ExpandHint) override {
        SetupOutputBuffers(expandedIndexes, expandedOperators);
        for (size_t i = 0; i < indexes.size(); i++) {
            if (!(usedOperatorBits[i] & 1)) { expandedIndexes.push_back((indexes[i] + n_ - 1) % n_); expandedOperators.push_back(1); }
            if (!(usedOperatorBits[i] & 2)) { expandedIndexes.push_back((indexes[i] + 1) % n_); expandedOperators.push_back(0); }
        }
    }

private:
    uint64_t n_;
};

int main() {
    std::string line;
    while (std::getline(std::cin, line)) {
        std::istringstream in(line);
        std::string cmd, kind;
        int a = 0, b = 0;
        in >> cmd;
        if (cmd == "custom") {
            uint64_t n = 0;
            in >> n;
            RingPuzzle ring(n);
            uint64_t children = 0;
            ExpandBuffer nodes(ring);
            auto count = [&](uint64_t, int) { children++; };
            for (uint64_t i = 0; i < n; i++) nodes.Add(i, 0, count);
            nodes.Finish(count);
            std::cout << children;
            try {
                InMemoryTwoBitBFS(ring, "0");
                std::cout << " searched\n";
            } catch (const psb200::Error& e) {
                std::cout << " ERROR " << e.code() << " " << e.what() << "\n";
            }
            std::cout.flush();
            continue;
        }
        if (cmd == "hanoisearch") {
            int disks = 0, steps = 0;
            in >> disks >> steps;
            try {
                std::vector<uint64_t> r;
                switch (disks) {
#define HANOI_CASE(n)                                              \
    case n: {                                                      \
        SearchOptions opts;                                        \
        if (steps > 0) opts.maxSteps = steps;                      \
        r = HanoiSearch<HanoiTowers<n>::Size>(HanoiTowers<n>::ToString(0), opts); \
        break;                                                     \
    }
                    HANOI_CASE(8) HANOI_CASE(9) HANOI_CASE(10) HANOI_CASE(11) HANOI_CASE(12) HANOI_CASE(13)
                    HANOI_CASE(14) HANOI_CASE(15) HANOI_CASE(16) HANOI_CASE(17) HANOI_CASE(18) HANOI_CASE(19)
#undef HANOI_CASE
                default: std::cout << "ERROR -1 unsupported size\n"; std::cout.flush(); continue;
                }
                for (size_t i = 0; i < r.size(); i++) std::cout << (i ? " " : "") << r[i];
                std::cout << "\n";
            } catch (const psb200::Error& e) {
                std::cout << "ERROR " << e.code() << " " << e.what() << "\n";
            }
            std::cout.flush();
            continue;
        }
        in >> kind >> a >> b;
        try {
            auto puzzle = make(kind, a, b);
            if (cmd == "disk") {  // a disk-based test body: PuzzleOptions with segmentBits and threads
                std::string algo, state;
                PuzzleOptions opts;
                in >> algo >> opts.segmentBits >> opts.threads;
                std::getline(in, state);
                if (state.empty() || state == " ") state = puzzle->ToString(0);
                std::vector<uint64_t> r;
                if (algo == "Classic") r = DiskBasedClassicBFS(*puzzle, state, opts);
                else if (algo == "TwoBit") r = DiskBasedTwoBitBFS(*puzzle, state, opts);
                else if (algo == "ThreeBit") r = DiskBasedThreeBitBFS(*puzzle, state, opts);
                else if (algo == "FrontierSearch") r = DiskBasedFrontierSearch(*puzzle, state, opts);
                else if (algo == "OptFrontierSearch") r = DiskBasedOptFrontierSearch(*puzzle, state, opts);
                else r = DiskBasedOptThreeBitBFS(*puzzle, state, opts);
                for (size_t i = 0; i < r.size(); i++) std::cout << (i ? " " : "") << r[i];
                std::cout << "\n";
            } else if (cmd == "bfs") {
                std::string algo, state;
                in >> algo;
                std::getline(in, state);
                if (state.empty() || state == " ") state = puzzle->ToString(0);
                std::vector<uint64_t> r;
                if (algo == "classic") r = InMemoryClassicBFS(*puzzle, state);
                else if (algo == "two_bit") r = InMemoryTwoBitBFS(*puzzle, state);
                else if (algo == "three_bit") r = InMemoryThreeBitBFS(*puzzle, state);
                else r = InMemoryFrontierSearch(*puzzle, state);
                for (size_t i = 0; i < r.size(); i++) std::cout << (i ? " " : "") << r[i];
                std::cout << "\n";
            } else {
                std::string state;
                std::getline(in, state);
                std::vector<uint64_t> indexes{state.empty() || state == " " ? 0 : puzzle->Parse(state)};
                std::vector<int> used{0};
                std::vector<uint64_t> children;
                std::vector<int> ops;
                puzzle->Expand(indexes, used, children, ops, {});
                for (size_t i = 0; i < children.size(); i++)
                    std::cout << (i ? ";" : "") << puzzle->ToString(children[i]) << "|" << ops[i];
                std::cout << "\n";
            }
        } catch (const psb200::Error& e) {
            std::cout << "ERROR " << e.code() << " " << e.what() << "\n";
        }
        std::cout.flush();
    }
    return 0;
}
