// ref_mt_bfs.cpp -- multi-threaded three-bit BFS over the reference's own
// puzzle classes (test infrastructure only; built by oracle/build_ref.sh into
// oracle/_ref/psbref_mt).  It produces per-depth count fixtures for state
// spaces that the reference's single-threaded InMemoryThreeBitBFS needs many
// hours for (18-disk Hanoi, 14-pancake).
//
//   psbref_mt <kind 1|2|3> <a> <b> <threads> [initial state]
//
// Children come from the reference's own code: each thread owns an
// ExpandBuffer (Common/Puzzle.h:50-120) over the reference's *Simple puzzle
// (Puzzles/PancakeSimple.cpp:62-87, Puzzles/FourPegHanoiSimple.cpp:156-235,
// Puzzles/SlidingTilePuzzleSimple.cpp:61-113), whose Expand keeps no state
// between calls, so threads may share the puzzle object.  The level loop
// restates InMemoryThreeBitBFS (Common/InMemoryThreeBitBFS.cpp:4-48) over
// threads: scan `cur`, expand, set `new`; `new &= ~cur` when the puzzle has
// odd-length cycles; count = popc(new &= ~old); rotate old <- cur <- new.
// The only difference is that `new` is set with an atomic OR per 64-bit word
// and that the sweeps are split over threads; the sets and counts are the
// same as the reference's.  Its output is checked against the unmodified
// reference on every puzzle the tests run it on.
#include "Common/Puzzle.h"
#include "Puzzles/FourPegHanoiSimple.h"
#include "Puzzles/PancakeSimple.h"
#include "Puzzles/SlidingTilePuzzleSimple.h"

#include <atomic>
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <memory>
#include <string>
#include <thread>
#include <vector>

namespace {

std::unique_ptr<Puzzle> MakePuzzle(int kind, int a, int b) {
    switch (kind) {
    case 1: return std::make_unique<SlidingTilePuzzleSimple>(a, b);
    case 2: return std::make_unique<PancakeSimple>(a);
    case 3: return std::make_unique<FourPegHanoiSimple>(a, b != 0);
    }
    return nullptr;
}

struct Bits {
    uint64_t words = 0;
    uint64_t* w = nullptr;
    explicit Bits(uint64_t n) : words((n + 63) / 64) {
        w = static_cast<uint64_t*>(std::calloc(words, sizeof(uint64_t)));
        if (!w) { std::fprintf(stderr, "psbref_mt: out of memory\n"); std::exit(4); }
    }
    ~Bits() { std::free(w); }
};

// Runs fn(begin_word, end_word) over [0, words) in chunks taken from a
// shared counter, on `threads` threads.
template <typename F>
void ParallelWords(uint64_t words, int threads, F fn) {
    const uint64_t chunk = 1 << 16;
    std::atomic<uint64_t> next{0};
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; t++) {
        pool.emplace_back([&, t] {
            for (;;) {
                uint64_t b = next.fetch_add(chunk);
                if (b >= words) break;
                fn(t, b, std::min(words, b + chunk));
            }
        });
    }
    for (auto& th : pool) th.join();
}

}  // namespace

int main(int argc, char** argv) {
    if (argc < 5) {
        std::fprintf(stderr, "usage: psbref_mt kind a b threads [state]\n");
        return 2;
    }
    int kind = std::atoi(argv[1]), a = std::atoi(argv[2]), b = std::atoi(argv[3]);
    int threads = std::max(1, std::atoi(argv[4]));
    auto puzzle = MakePuzzle(kind, a, b);
    if (!puzzle) return 2;
    std::string init = argc > 5 ? std::string(argv[5]) : puzzle->ToString(0);

    auto t0 = std::chrono::steady_clock::now();
    const uint64_t size = puzzle->IndexesCount();
    Bits oldb(size), cur(size), nxt(size);
    const uint64_t words = cur.words;
    uint64_t start = puzzle->Parse(init);
    cur.w[start / 64] |= 1ull << (start % 64);
    std::vector<uint64_t> result{1};
    const bool odd = puzzle->HasOddLengthCycles();

    std::vector<std::unique_ptr<ExpandBuffer>> buffers;
    for (int t = 0; t < threads; t++) buffers.push_back(std::make_unique<ExpandBuffer>(*puzzle));

    for (;;) {
        auto tl = std::chrono::steady_clock::now();
        // Expand every state of `cur`; children are ORed into `nxt`.
        {
            std::vector<std::thread> pool;
            std::atomic<uint64_t> next{0};
            const uint64_t chunk = 1 << 14;
            for (int t = 0; t < threads; t++) {
                pool.emplace_back([&, t] {
                    ExpandBuffer& nodes = *buffers[t];
                    auto mark = [&](uint64_t child, int) {
                        std::atomic_ref<uint64_t>(nxt.w[child / 64]).fetch_or(1ull << (child % 64),
                                                                              std::memory_order_relaxed);
                    };
                    for (;;) {
                        uint64_t bw = next.fetch_add(chunk);
                        if (bw >= words) break;
                        uint64_t ew = std::min(words, bw + chunk);
                        for (uint64_t i = bw; i < ew; i++) {
                            uint64_t v = cur.w[i];
                            while (v) {
                                int bit = __builtin_ctzll(v);
                                v &= v - 1;
                                nodes.Add(i * 64 + bit, 0, mark);
                            }
                        }
                    }
                    nodes.Finish(mark);
                });
            }
            for (auto& th : pool) th.join();
        }
        // new &= ~cur (odd cycles); count = popc(new &= ~old).
        std::vector<uint64_t> part(threads, 0);
        ParallelWords(words, threads, [&](int t, uint64_t bw, uint64_t ew) {
            uint64_t c = 0;
            for (uint64_t i = bw; i < ew; i++) {
                uint64_t v = nxt.w[i];
                if (odd) v &= ~cur.w[i];
                v &= ~oldb.w[i];
                nxt.w[i] = v;
                c += __builtin_popcountll(v);
            }
            part[t] += c;
        });
        uint64_t count = 0;
        for (auto c : part) count += c;
        double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - tl).count();
        std::fprintf(stderr, "depth %zu: %llu (%.1f s)\n", result.size(), (unsigned long long)count, secs);
        if (count == 0) break;
        result.push_back(count);
        // old <- cur, cur <- new, new <- cleared old.
        std::swap(oldb.w, cur.w);
        std::swap(cur.w, nxt.w);
        ParallelWords(words, threads, [&](int, uint64_t bw, uint64_t ew) {
            std::memset(nxt.w + bw, 0, (ew - bw) * sizeof(uint64_t));
        });
    }
    double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    uint64_t total = 0;
    std::printf("{\"seconds\": %.3f, \"threads\": %d, \"depths\": %zu, \"counts\": [", secs, threads, result.size());
    for (size_t i = 0; i < result.size(); i++) {
        total += result[i];
        std::printf(i ? ", %llu" : "%llu", (unsigned long long)result[i]);
    }
    std::printf("], \"states\": %llu}\n", (unsigned long long)total);
    return 0;
}
