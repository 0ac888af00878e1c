// psb_noalloc.cu -- psb_bfs_noalloc: the in-memory search for callers that
// cannot allocate device memory.  It has no counterpart in the reference.
//
// Some callers may not call cudaMalloc at all.  Examples: code that must not
// touch the device allocator while another component (a framework's caching
// allocator, a memory pool sized at start-up) owns all device memory, or
// hosts that hand every buffer in from one pre-reserved arena.  They pass the
// bit arrays in.  The few bytes of scratch a search also needs live here, in
// one file-scope __device__ array:
//   [0, 64)                        level counters (frontier states, children, local children, error flag, count)
//   [256, 256 + kMaxWindows)       active-window flags A
//   [256 + kMaxWindows, ... )      active-window flags B
// kMaxWindows = 2^21 windows, so the array is 4 MiB + 256 bytes and every GPU
// that loads the library holds it until the process exits.  Searches whose
// window count exceeds kMaxWindows are rejected with PSB_ERR_CAPACITY.
//
// The array is shared by every call: each call clears what must start at
// zero.  Calls whose GPU work overlaps (two host threads, or two streams)
// race on it; run them one after the other.  Every call looks up the array's
// device address (cudaGetSymbolAddress) with the caller's device current, so
// a context rebuilt after cudaDeviceReset gets its own address.
//
// The CUDA runtime loads a module lazily: the first call on a device loads
// this file's module (with the array) and the level kernels' modules, and
// that load takes device memory from the driver.  A caller that reserves all
// device memory for its own arena makes one call (any small search) first.
// Each call synchronizes `stream` at every level (it reads the level's
// counters back), so it must not be called while that stream is captured.
//
// d_arrays must be 256-byte aligned: the finalize sweeps read it 16 bytes at
// a time and the arrays inside it are padded to 256 bytes.  Any other pointer
// is rejected with PSB_ERR_ARG before the device is touched.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/psb200.h"
#include "psb_internal.h"

namespace {

constexpr uint64_t kMaxWindows = uint64_t(1) << 21;
constexpr size_t kScratchBytes = 256 + 2 * kMaxWindows;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

int na_fail(int code, const std::string& msg) { return psb_set_error(code, msg.c_str()); }

#define NA_CUDA(call)                                                                    \
    do {                                                                                 \
        cudaError_t e_ = (call);                                                         \
        if (e_ != cudaSuccess)                                                           \
            return na_fail(PSB_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

// Device address of the scratch array on the current device.  Looked up on
// every call: it is cheap, and a cached address would go stale when the
// context is rebuilt.
int scratch_address(unsigned char** out) {
    void* ptr = nullptr;
    NA_CUDA(cudaGetSymbolAddress(&ptr, g_noalloc_scratch));
    *out = static_cast<unsigned char*>(ptr);
    return PSB_OK;
}

uint64_t words_for(uint64_t bits) { return (bits + 63) / 64; }
uint64_t padded(uint64_t words) { return (words + 31) / 32 * 32; }

int window_bits_for(const psb_puzzle* p, int algo) {  // same policy as psb_bfs
    int lg = 0;
    while (lg < 63 && (uint64_t(1) << (lg + 1)) <= p->n_states) lg++;
    const int cap = (p->kind == PSB_HANOI4 || p->kind == PSB_HANOI4_OPT) ? 17 : 16;
    int wb = std::max(10, std::min(cap, lg - 10));
    if (algo == PSB_FRONTIER) wb = std::min(wb, 16);
    return wb;
}

}  // namespace

extern "C" int psb_bfs_noalloc(const psb_puzzle* p, int algo, uint64_t initial, uint64_t* d_arrays,
                               uint64_t d_array_words, uint32_t max_depth, void* stream_ptr, uint64_t* counts,
                               uint32_t cap, uint32_t* n_depths) {
    if (!p || !d_arrays || !counts || !n_depths || cap == 0) return na_fail(PSB_ERR_ARG, "bad argument");
    if (reinterpret_cast<uintptr_t>(d_arrays) % 256 != 0)
        return na_fail(PSB_ERR_ARG, "d_arrays must be 256-byte aligned");
    const uint64_t N = p->n_states;
    if (initial >= N) return na_fail(PSB_ERR_ARG, "initial index >= IndexesCount()");
    int mode = -1, n_arr = 0;
    uint64_t words[4] = {0, 0, 0, 0};
    switch (algo) {
    case PSB_THREE_BIT: mode = psb::kThreeBit; n_arr = 3; words[0] = words[1] = words[2] = padded(words_for(N)); break;
    case PSB_CLASSIC: mode = psb::kClassic; n_arr = 3; words[0] = words[1] = words[2] = padded(words_for(N)); break;
    case PSB_TWO_BIT: mode = psb::kTwoBit; n_arr = 1; words[0] = padded(words_for(2 * N)); break;
    case PSB_FRONTIER:
        if (p->ops > 4) return na_fail(PSB_ERR_UNSUPPORTED, "frontier search keeps 4 operator bits per state");
        mode = psb::kFrontier;
        n_arr = p->odd ? 4 : 2;
        words[0] = words[1] = padded((N + 15) / 16);
        if (p->odd) words[2] = words[3] = padded(words_for(N));
        break;
    default: return na_fail(PSB_ERR_ARG, "unknown algorithm");
    }
    const uint64_t need = words[0] + words[1] + words[2] + words[3];
    if (d_array_words < need)
        return na_fail(PSB_ERR_CAPACITY, "d_arrays needs " + std::to_string(need) + " 64-bit words");
    const int wb = window_bits_for(p, algo);
    const uint64_t n_windows = (N + (uint64_t(1) << wb) - 1) >> wb;
    if (n_windows > kMaxWindows)
        return na_fail(PSB_ERR_CAPACITY, "search needs " + std::to_string(n_windows) + " windows; the static scratch holds " +
                                             std::to_string(kMaxWindows));
    unsigned char* scratch = nullptr;
    if (int rc = scratch_address(&scratch)) return rc;
    unsigned long long* d_stats = reinterpret_cast<unsigned long long*>(scratch);
    uint8_t* wflags[2] = {scratch + 256, scratch + 256 + kMaxWindows};
    cudaStream_t s = static_cast<cudaStream_t>(stream_ptr);

    uint64_t* arr[4] = {nullptr, nullptr, nullptr, nullptr};
    uint64_t off = 0;
    for (int i = 0; i < n_arr; i++) { arr[i] = d_arrays + off; off += words[i]; }
    for (int i = 0; i < n_arr; i++) NA_CUDA(cudaMemsetAsync(arr[i], 0, words[i] * 8, s));

    const uint64_t W1 = words_for(N), W2 = words_for(2 * N), W4 = (N + 15) / 16;
    auto set_bit = [&](uint64_t* base, uint64_t bit) -> int {
        const uint64_t word = uint64_t(1) << (bit & 63);
        NA_CUDA(cudaMemcpyAsync(base + (bit >> 6), &word, 8, cudaMemcpyHostToDevice, s));
        NA_CUDA(cudaStreamSynchronize(s));
        return PSB_OK;
    };
    uint64_t *old_ = arr[0], *cur = arr[1], *nw = arr[2];
    uint64_t *closed = arr[0], *open = arr[1], *nopen = arr[2];
    uint64_t* codes = arr[0];
    uint64_t *fcur = arr[0], *fnext = arr[1], *cex = arr[2], *nex = arr[3];
    int rc = PSB_OK;
    if (algo == PSB_THREE_BIT) rc = set_bit(cur, initial);
    if (algo == PSB_CLASSIC) { rc = set_bit(open, initial); if (!rc) rc = set_bit(closed, initial); }
    if (algo == PSB_TWO_BIT) rc = set_bit(codes, 2 * initial);
    if (rc) return rc;

    int flags_valid = -1;
    if (algo != PSB_FRONTIER) {
        const uint8_t one = 1;
        NA_CUDA(cudaMemsetAsync(wflags[0], 0, n_windows, s));
        NA_CUDA(cudaMemcpyAsync(wflags[0] + (initial >> wb), &one, 1, cudaMemcpyHostToDevice, s));
        NA_CUDA(cudaStreamSynchronize(s));
        flags_valid = 0;
    }
    psb::LevelArgs a{};
    a.n_states = N;
    a.window_bits = wb;
    a.odd = p->odd;
    a.pz = p->pz;
    a.stats = d_stats;
    const unsigned grid = unsigned(n_windows);
    const size_t W = size_t(1) << wb;
    const size_t smem = psb::level_smem_bytes(mode, W, psb::level_threads(mode));
    uint32_t cur_code = 2;
    uint64_t estimate = 1;
    const uint64_t sparse_limit = N / 64;
    std::vector<uint64_t> res;
    bool first = true;
    for (;;) {
        if (max_depth && res.size() >= size_t(max_depth) + 1) break;
        NA_CUDA(cudaMemsetAsync(d_stats, 0, 8 * sizeof(unsigned long long), s));
        const bool produce = estimate < sparse_limit;
        const int flags_next = flags_valid < 0 ? 0 : 1 - flags_valid;
        if (produce) NA_CUDA(cudaMemsetAsync(wflags[flags_next], 0, n_windows, s));
        a.wflag_cur = flags_valid >= 0 ? wflags[flags_valid] : nullptr;
        a.wflag_next = produce ? wflags[flags_next] : nullptr;
        if (algo == PSB_FRONTIER && first) {
            a.marks = fnext; a.excl_next = nex; a.mark_words = W4;
            NA_CUDA(p->k.seed(a, initial, s));
        } else {
            switch (algo) {
            case PSB_THREE_BIT: a.front = cur; a.marks = nw; a.front_words = W1; a.mark_words = W1; break;
            case PSB_CLASSIC: a.front = open; a.marks = nopen; a.front_words = W1; a.mark_words = W1; break;
            case PSB_TWO_BIT: a.front = codes; a.marks = codes; a.front_words = W2; a.mark_words = W2; a.cur_code = cur_code; break;
            case PSB_FRONTIER:
                a.front = fcur; a.marks = fnext; a.excl_cur = cex; a.excl_next = nex;
                a.front_words = W4; a.mark_words = W4;
                break;
            }
            NA_CUDA(p->k.level[mode](a, grid, smem, s));
        }
        if (algo == PSB_THREE_BIT || algo == PSB_CLASSIC) {
            const uint64_t n2 = (W1 + 1) / 2;
            if (algo == PSB_THREE_BIT)
                psb::finalize_three_bit<<<148 * 8, psb::kThreads, 0, s>>>(
                    reinterpret_cast<const ulonglong2*>(cur), reinterpret_cast<ulonglong2*>(nw),
                    reinterpret_cast<ulonglong2*>(old_), n2, p->odd, 1, d_stats + 4);
            else
                psb::finalize_classic<<<148 * 8, psb::kThreads, 0, s>>>(
                    reinterpret_cast<ulonglong2*>(nopen), reinterpret_cast<ulonglong2*>(closed), n2, d_stats + 4);
            NA_CUDA(cudaGetLastError());
        }
        unsigned long long h[8];
        NA_CUDA(cudaMemcpyAsync(h, d_stats, sizeof h, cudaMemcpyDeviceToHost, s));
        NA_CUDA(cudaStreamSynchronize(s));
        if (h[3]) return na_fail(PSB_ERR_DEVICE, "level kernel produced a child index >= IndexesCount()");
        uint64_t count = 0;
        switch (algo) {
        case PSB_THREE_BIT:
            count = h[4];
            if (first) res.push_back(1);
            if (count == 0) goto done;
            res.push_back(count);
            { uint64_t* t = old_; old_ = cur; cur = nw; nw = t; }
            break;
        case PSB_CLASSIC:
            count = h[4];
            if (first) res.push_back(1);
            if (count == 0) goto done;
            res.push_back(count);
            std::swap(open, nopen);
            break;
        case PSB_TWO_BIT:
            count = h[0];
            if (count == 0) goto done;
            res.push_back(count);
            cur_code = 5 - cur_code;
            break;
        case PSB_FRONTIER:
            count = first ? 1 : h[0];
            if (count == 0) goto done;
            res.push_back(count);
            std::swap(fcur, fnext);
            if (p->odd) {
                std::swap(cex, nex);
                NA_CUDA(cudaMemsetAsync(nex, 0, W1 * 8, s));
            }
            break;
        }
        first = false;
        flags_valid = produce ? flags_next : -1;
        estimate = count;
        if (res.size() > cap) return na_fail(PSB_ERR_CAPACITY, "more depths than counts_cap");
    }
done:
    if (res.size() > cap) return na_fail(PSB_ERR_CAPACITY, "more depths than counts_cap");
    std::copy(res.begin(), res.end(), counts);
    *n_depths = uint32_t(res.size());
    return PSB_OK;
}
