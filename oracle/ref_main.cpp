// ref_main.cpp -- CLI around the reference's own in-memory BFS (test and
// CPU-baseline infrastructure only; built by oracle/build_ref.sh).
//
//   psbref <kind 1|2|3> <a> <b> <algo 1..4> [initial state]
//
// kind: 1 sliding-tile (a=width, b=height), 2 pancake (a=size), 3 four-peg
// Hanoi (a=disks, b=symmetry); algo: 1 two-bit, 2 three-bit, 3 frontier
// search, 4 classic.  Prints one JSON line: per-depth counts, states reached
// and wall seconds of the reference call.
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

extern "C" int ref_bfs(int kind, int a, int b, int algo, const char* init, uint64_t* counts, int cap, int quiet);
extern "C" int ref_to_string(int kind, int a, int b, uint64_t index, char* buf, int cap);

int main(int argc, char** argv) {
    if (argc < 5) {
        std::fprintf(stderr, "usage: psbref kind a b algo [state]\n");
        return 2;
    }
    int kind = std::atoi(argv[1]), a = std::atoi(argv[2]), b = std::atoi(argv[3]), algo = std::atoi(argv[4]);
    std::string init;
    if (argc > 5) init = argv[5];
    else {
        char buf[512];
        if (ref_to_string(kind, a, b, 0, buf, sizeof buf) < 0) return 2;
        init = buf;
    }
    std::vector<uint64_t> counts(100000);
    auto t0 = std::chrono::steady_clock::now();
    int n = ref_bfs(kind, a, b, algo, init.c_str(), counts.data(), (int)counts.size(), 1);
    double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (n < 0) return 3;
    uint64_t total = 0;
    std::printf("{\"seconds\": %.6f, \"depths\": %d, \"counts\": [", secs, n);
    for (int i = 0; i < n; i++) { total += counts[i]; std::printf(i ? ", %llu" : "%llu", (unsigned long long)counts[i]); }
    std::printf("], \"states\": %llu}\n", (unsigned long long)total);
    return 0;
}
