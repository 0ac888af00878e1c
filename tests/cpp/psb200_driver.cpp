// psb200_driver.cpp -- exercises include/psb200.hpp the way the reference's
// tests use its classes (PuzzlesTests/PuzzleSearchTests.cpp, PancakeTest.cpp,
// FourPegHanoiTest.cpp).  Reads commands on stdin, one per line:
//   bfs <sliding|pancake|hanoi4> <a> <b> <classic|two_bit|three_bit|frontier> <state...>
//   expand <sliding|pancake|hanoi4> <a> <b> <state...>
// and prints one result line per command (space-separated counts, or
// "child-state|op" items separated by ';').  tests/test_gpu_cpp_adapter.py
// feeds it the reference's golden vectors.
#define PSB200_GLOBAL_NAMES
#include "../../include/psb200.hpp"

#include <iostream>
#include <memory>
#include <sstream>
#include <string>

static std::unique_ptr<Puzzle> make(const std::string& kind, int a, int b) {
    if (kind == "sliding") return std::make_unique<SlidingTilePuzzleSimple>(a, b);
    if (kind == "pancake") return std::make_unique<PancakeSimple>(a);
    return std::make_unique<FourPegHanoiSimple>(a, b != 0);
}

int main() {
    std::string line;
    while (std::getline(std::cin, line)) {
        std::istringstream in(line);
        std::string cmd, kind;
        int a = 0, b = 0;
        in >> cmd >> kind >> a >> b;
        try {
            auto puzzle = make(kind, a, b);
            if (cmd == "bfs") {
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
