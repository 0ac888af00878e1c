// psb_engine.cu -- many independent two-bit searches at once.
//
// Batched and served solves (no single counterpart in the reference, which
// runs one InMemoryTwoBitBFS per call, Common/InMemoryTwoBitBFS.cpp:24-69):
// every instance keeps its own two-bit array, identical in codes and layout
// to InMemoryTwoBitBFS's, in one device pool, back to back.  One engine step
// advances every active instance by one BFS level:
//
//   build_queue  (1 block): exclusive scan of the active instances' window
//                counts -> the level's (instance, window) work queue
//   batch_level  (persistent, #SM x k blocks): blocks pull work items and run
//                the same per-window level pass as psb_bfs (level_window)
//   retire       (persistent): CUR -> OLD and the depth count for the
//                instances whose level ran bottom-up (see psb_bfs)
//   epilogue     (1 block): each instance's count of CUR states becomes its
//                next per-depth count; an instance whose count is 0 is done
//                and its slot id is appended to a completion list.  It also
//                picks each instance's next direction with psb_bfs's rule:
//                bottom-up once the frontier is dense (>= N/64) and larger
//                than the unvisited states
//
// The three launches are captured once as a CUDA graph and replayed; all
// per-level state lives in device tables, so instances added between
// replays (continuous batching) simply appear in the next queue.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "../../include/psb200.h"
#include "psb_internal.h"

namespace psb {

// Puzzle shapes the engine compiles in (one level_window instantiation each).
enum EngineType : uint32_t {
    kE_S6 = 0, kE_S8, kE_S9, kE_S10, kE_S12,
    kE_P7, kE_P8, kE_P9, kE_P10, kE_P11, kE_P12,
    kE_H,
    kE_Types
};

constexpr int kEThreads = 256;
constexpr int kEMinBlocks = 2;
constexpr uint32_t kEWindowBitsMax = 16;

struct EngineSlot {
    LevelArgs args;     // per-instance level arguments (front = marks = probe = its codes)
    uint8_t* flags[2];  // active-window flags, windows bytes each (see psb_bfs)
    uint32_t type;      // EngineType
    uint32_t state;     // 0 free, 1 active, 2 done (waiting for the host to collect)
    uint32_t depth;     // counts recorded so far
    uint32_t windows;   // windows of this instance
    uint32_t bu;        // this level runs bottom-up
    uint32_t can_bu;    // the puzzle allows bottom-up levels (not Hanoi with symmetry)
    uint64_t seen;      // states at depths below the current frontier's
};

struct EngineDev {
    EngineSlot* slots;
    unsigned long long* stats;   // 8 per slot
    unsigned long long* counts;  // max_depths per slot
    uint32_t* item_start;        // n_slots + 1
    uint32_t* queue_head;
    uint32_t* retire_head;       // work-queue counter of the retire pass
    uint32_t* n_items;
    uint32_t* done_list;         // slot ids, ring of n_slots
    uint32_t* done_count;        // monotonically increasing
    uint32_t* n_active;
    unsigned long long* err;
    uint32_t n_slots;
    uint32_t max_depths;
};

__global__ void __launch_bounds__(1024) engine_build_queue(EngineDev d) {
    __shared__ uint32_t warp_tot[32];
    __shared__ uint32_t carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    uint32_t active = 0;
    for (uint32_t base = 0; base < d.n_slots; base += 1024) {
        const uint32_t s = base + threadIdx.x;
        uint32_t w = 0;
        if (s < d.n_slots && d.slots[s].state == 1) { w = d.slots[s].windows; active++; }
        uint32_t incl = w;
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
            if (lane >= o) incl += y;
        }
        if (lane == 31) warp_tot[warp] = incl;
        __syncthreads();
        if (warp == 0) {
            uint32_t t = warp_tot[lane];
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, t, o);
                if (lane >= o) t += y;
            }
            warp_tot[lane] = t;
        }
        __syncthreads();
        const uint32_t excl = carry + (warp ? warp_tot[warp - 1] : 0) + incl - w;
        if (s < d.n_slots) d.item_start[s] = excl;
        const uint32_t block_total = warp_tot[31];
        __syncthreads();
        if (threadIdx.x == 0) carry += block_total;
        __syncthreads();
    }
    (void)active;
    if (threadIdx.x == 0) {
        d.item_start[d.n_slots] = carry;
        *d.n_items = carry;
        *d.queue_head = 0;
        *d.retire_head = 0;
    }
}

template <int T>
__device__ __forceinline__ void engine_window(const LevelArgs& a, uint64_t window, unsigned long long* smem,
                                              WindowShared& sh) {
    if constexpr (T == kE_S6) level_window<SlidingK<6>, kTwoBit, kEThreads>(a, window, smem, sh);
    if constexpr (T == kE_S8) level_window<SlidingK<8>, kTwoBit, kEThreads>(a, window, smem, sh);
    if constexpr (T == kE_S9) level_window<SlidingK<9>, kTwoBit, kEThreads>(a, window, smem, sh);
    if constexpr (T == kE_S10) level_window<SlidingK<10>, kTwoBit, kEThreads>(a, window, smem, sh);
    if constexpr (T == kE_S12) level_window<SlidingK<12>, kTwoBit, kEThreads>(a, window, smem, sh);
    if constexpr (T == kE_P7) level_window<PancakeK<7>, kTwoBit, kEThreads>(a, window, smem, sh);
    if constexpr (T == kE_P8) level_window<PancakeK<8>, kTwoBit, kEThreads>(a, window, smem, sh);
    if constexpr (T == kE_P9) level_window<PancakeK<9>, kTwoBit, kEThreads>(a, window, smem, sh);
    if constexpr (T == kE_P10) level_window<PancakeK<10>, kTwoBit, kEThreads>(a, window, smem, sh);
    if constexpr (T == kE_P11) level_window<PancakeK<11>, kTwoBit, kEThreads>(a, window, smem, sh);
    if constexpr (T == kE_P12) level_window<PancakeK<12>, kTwoBit, kEThreads>(a, window, smem, sh);
    if constexpr (T == kE_H) level_window<HanoiK, kTwoBit, kEThreads>(a, window, smem, sh);
}

template <int T>
__device__ __forceinline__ void engine_window_bu(const LevelArgs& a, uint64_t window, unsigned long long* smem,
                                                 WindowShared& sh) {
    if constexpr (T == kE_S6) level_window<SlidingK<6>, kTwoBit, kEThreads, true>(a, window, smem, sh);
    if constexpr (T == kE_S8) level_window<SlidingK<8>, kTwoBit, kEThreads, true>(a, window, smem, sh);
    if constexpr (T == kE_S9) level_window<SlidingK<9>, kTwoBit, kEThreads, true>(a, window, smem, sh);
    if constexpr (T == kE_S10) level_window<SlidingK<10>, kTwoBit, kEThreads, true>(a, window, smem, sh);
    if constexpr (T == kE_S12) level_window<SlidingK<12>, kTwoBit, kEThreads, true>(a, window, smem, sh);
    if constexpr (T == kE_P7) level_window<PancakeK<7>, kTwoBit, kEThreads, true>(a, window, smem, sh);
    if constexpr (T == kE_P8) level_window<PancakeK<8>, kTwoBit, kEThreads, true>(a, window, smem, sh);
    if constexpr (T == kE_P9) level_window<PancakeK<9>, kTwoBit, kEThreads, true>(a, window, smem, sh);
    if constexpr (T == kE_P10) level_window<PancakeK<10>, kTwoBit, kEThreads, true>(a, window, smem, sh);
    if constexpr (T == kE_P11) level_window<PancakeK<11>, kTwoBit, kEThreads, true>(a, window, smem, sh);
    if constexpr (T == kE_P12) level_window<PancakeK<12>, kTwoBit, kEThreads, true>(a, window, smem, sh);
    if constexpr (T == kE_H) level_window<HanoiK, kTwoBit, kEThreads, true>(a, window, smem, sh);
}

template <int T>
__device__ __forceinline__ void engine_pass(bool bu, const LevelArgs& a, uint64_t window, unsigned long long* smem,
                                            WindowShared& sh) {
    if (bu) engine_window_bu<T>(a, window, smem, sh);
    else engine_window<T>(a, window, smem, sh);
}

__global__ void __launch_bounds__(kEThreads, kEMinBlocks) engine_level(EngineDev d) {
    extern __shared__ __align__(16) unsigned long long smem64[];
    __shared__ WindowShared sh;
    __shared__ uint32_t s_item;
    const uint32_t n_items = *d.n_items;
    for (;;) {
        if (threadIdx.x == 0) s_item = atomicAdd(d.queue_head, 1u);
        __syncthreads();
        const uint32_t item = s_item;
        __syncthreads();  // every thread read s_item before thread 0 may overwrite it
        if (item >= n_items) break;
        // instance owning this item: last s with item_start[s] <= item
        uint32_t lo = 0, hi = d.n_slots;  // item_start[lo] <= item < item_start[hi]
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) / 2;
            if (d.item_start[mid] <= item) lo = mid; else hi = mid;
        }
        const LevelArgs la = d.slots[lo].args;  // uniform loads: one copy per thread, broadcast by L1
        const uint32_t type = d.slots[lo].type;
        const bool bu = d.slots[lo].bu != 0;
        const uint64_t window = item - d.item_start[lo];
        switch (type) {
        case kE_S6: engine_pass<kE_S6>(bu, la, window, smem64, sh); break;
        case kE_S8: engine_pass<kE_S8>(bu, la, window, smem64, sh); break;
        case kE_S9: engine_pass<kE_S9>(bu, la, window, smem64, sh); break;
        case kE_S10: engine_pass<kE_S10>(bu, la, window, smem64, sh); break;
        case kE_S12: engine_pass<kE_S12>(bu, la, window, smem64, sh); break;
        case kE_P7: engine_pass<kE_P7>(bu, la, window, smem64, sh); break;
        case kE_P8: engine_pass<kE_P8>(bu, la, window, smem64, sh); break;
        case kE_P9: engine_pass<kE_P9>(bu, la, window, smem64, sh); break;
        case kE_P10: engine_pass<kE_P10>(bu, la, window, smem64, sh); break;
        case kE_P11: engine_pass<kE_P11>(bu, la, window, smem64, sh); break;
        case kE_P12: engine_pass<kE_P12>(bu, la, window, smem64, sh); break;
        default: engine_pass<kE_H>(bu, la, window, smem64, sh); break;
        }
    }
}

// After a bottom-up level: the instance's CUR codes become OLD and are
// counted (the depth's count, stats[4]), window by window as in retire_two_bit.
__global__ void __launch_bounds__(256) engine_retire(EngineDev d) {
    __shared__ uint32_t s_item;
    const uint32_t n_items = *d.n_items;
    for (;;) {
        if (threadIdx.x == 0) s_item = atomicAdd(d.retire_head, 1u);
        __syncthreads();
        const uint32_t item = s_item;
        __syncthreads();
        if (item >= n_items) break;
        uint32_t lo = 0, hi = d.n_slots;  // item_start[lo] <= item < item_start[hi]
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) / 2;
            if (d.item_start[mid] <= item) lo = mid; else hi = mid;
        }
        const EngineSlot& slot = d.slots[lo];
        if (!slot.bu) continue;  // uniform: the whole block skips the item
        const LevelArgs& a = slot.args;
        const uint64_t window = item - d.item_start[lo];
        const uint64_t w0 = (window << a.window_bits) >> 5, nw = (uint64_t(1) << a.window_bits) >> 5;
        unsigned long long* codes = reinterpret_cast<unsigned long long*>(a.front);
        uint32_t c = 0;
        for (uint64_t i = w0 + threadIdx.x; i < w0 + nw && i < a.front_words; i += blockDim.x) {
            const uint64_t x = codes[i], hib = x & kEven, lob = (x >> 1) & kEven;
            const uint64_t cur = hib & (a.cur_code == 3 ? lob : ~lob);
            if (cur) codes[i] = x ^ (cur | (a.cur_code == 2 ? (cur << 1) : 0));
            c += __popcll(cur);
        }
        c = __reduce_add_sync(0xFFFFFFFFu, c);
        if ((threadIdx.x & 31) == 0 && c) atomicAdd(&a.stats[4], (unsigned long long)c);
    }
}

// Records each active instance's count of this level (InMemoryTwoBitBFS.cpp:42-65:
// a level with no new state ends the search) and rotates its CUR/NEXT codes.
__global__ void __launch_bounds__(1024) engine_epilogue(EngineDev d) {
    for (uint32_t s = threadIdx.x; s < d.n_slots; s += 1024) {
        EngineSlot& slot = d.slots[s];
        if (slot.state != 1) continue;
        unsigned long long* st = d.stats + 8ull * s;
        if (st[3]) atomicOr(d.err, 1ull);
        const unsigned long long count = slot.bu ? st[4] : st[0];  // this depth's states
        const unsigned long long next_est = st[5];                 // the next frontier (estimate)
        for (int k = 0; k < 8; k++) st[k] = 0;
        if (count == 0 || slot.depth >= d.max_depths) {
            if (count != 0) atomicOr(d.err, 2ull);  // more depths than the engine records
            slot.state = 2;
            const uint32_t pos = atomicAdd(d.done_count, 1u);
            d.done_list[pos % d.n_slots] = s;
            continue;
        }
        d.counts[uint64_t(s) * d.max_depths + slot.depth] = count;
        slot.depth++;
        slot.args.cur_code = 5u - slot.args.cur_code;
        slot.seen += count;
        const uint64_t n = slot.args.n_states;
        const uint64_t unvisited = n - (slot.seen + next_est < n ? slot.seen + next_est : n);
        slot.bu = (slot.can_bu && next_est >= n / 64 && unvisited < next_est) ? 1u : 0u;
        // Active-window flags, the psb_bfs policy: the flags this level
        // recorded (if it recorded any) steer the next level's sweep, and the
        // next level records flags when this level's frontier is sparse.
        uint8_t* produced = slot.args.wflag_next;
        slot.args.wflag_cur = produced;
        if (!slot.bu && count < slot.args.n_states / 64) {  // bottom-up levels record no flags
            uint8_t* other = produced == slot.flags[0] ? slot.flags[1] : slot.flags[0];
            uint4* z = reinterpret_cast<uint4*>(other);
            for (uint32_t i = 0; i < (slot.windows + 15) / 16; i++) z[i] = make_uint4(0, 0, 0, 0);
            slot.args.wflag_next = other;
        } else {
            slot.args.wflag_next = nullptr;
        }
    }
}

// Copies the finished instances [first, first + n) of the completion list into
// one staging buffer: per instance [slot, depth, counts[max_depths]].
__global__ void engine_collect(EngineDev d, uint32_t first, uint32_t n, unsigned long long* staging) {
    const uint32_t i = blockIdx.x;
    if (i >= n) return;
    const uint32_t s = d.done_list[(first + i) % d.n_slots];
    unsigned long long* row = staging + uint64_t(i) * (d.max_depths + 2);
    if (threadIdx.x == 0) {
        row[0] = s;
        row[1] = d.slots[s].depth;
    }
    for (uint32_t k = threadIdx.x; k < d.max_depths; k += blockDim.x)
        row[2 + k] = d.counts[uint64_t(s) * d.max_depths + k];
}

// Frees the slots the host has collected.
__global__ void engine_release(EngineDev d, const uint32_t* slots, uint32_t n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) d.slots[slots[i]].state = 0;
}

}  // namespace psb

struct psb_engine {
    int device = -1;
    cudaStream_t stream = nullptr;
    uint32_t n_slots = 0, max_depths = 0;
    uint64_t pool_words = 0;
    uint64_t* pool = nullptr;
    psb::EngineDev d{};
    std::vector<psb::EngineSlot> host_slots;
    std::vector<uint64_t> slot_off, slot_words, slot_tag;
    std::vector<uint32_t> free_slots;
    std::map<uint64_t, uint64_t> free_space;  // offset -> words (first fit)
    uint32_t done_seen = 0;
    uint32_t active = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    bool use_graph = true;
    bool bottom_up = true;  // instances may run bottom-up levels
    int wb_offset = 0;      // window bits relative to engine_window_bits' rule
    unsigned grid = 0;
    size_t smem = 0;
    uint64_t levels_run = 0;
    uint32_t* h_done_count = nullptr;  // pinned
    unsigned long long* h_err = nullptr;  // pinned: the error word, read with the done count after each step
    bool done_fresh = false;           // *h_done_count was read after the last step and nothing ran since
    unsigned long long* d_staging = nullptr;  // collect rows (device)
    std::vector<unsigned long long> h_staging;

    ~psb_engine() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        cudaFree(pool);
        cudaFree(d.slots);
        cudaFree(d.stats);
        cudaFree(d.counts);
        cudaFree(d.item_start);
        cudaFree(d.err);
        if (h_done_count) cudaFreeHost(h_done_count);
        if (h_err) cudaFreeHost(h_err);
        cudaFree(d_staging);
        if (stream) cudaStreamDestroy(stream);
    }
};

namespace {

#define EN_CUDA(call)                                                                           \
    do {                                                                                        \
        cudaError_t e_ = (call);                                                                \
        if (e_ != cudaSuccess)                                                                  \
            return psb_set_error(e_ == cudaErrorMemoryAllocation ? PSB_ERR_NOMEM : PSB_ERR_CUDA, \
                                 (std::string(#call) + ": " + cudaGetErrorString(e_)).c_str());  \
    } while (0)

int engine_type(int kind, int a, int b, uint32_t* type) {
    if (kind == PSB_SLIDING) {
        switch (a * b) {
        case 6: *type = psb::kE_S6; return PSB_OK;
        case 8: *type = psb::kE_S8; return PSB_OK;
        case 9: *type = psb::kE_S9; return PSB_OK;
        case 10: *type = psb::kE_S10; return PSB_OK;
        case 12: *type = psb::kE_S12; return PSB_OK;
        }
    } else if (kind == PSB_PANCAKE) {
        if (a >= 7 && a <= 12) { *type = psb::kE_P7 + uint32_t(a - 7); return PSB_OK; }
    } else if (kind == PSB_HANOI4) {
        if (a >= 1 && a <= 16) { *type = psb::kE_H; return PSB_OK; }
    }
    return psb_set_error(PSB_ERR_UNSUPPORTED,
                         "engine puzzles: sliding tile with 6, 8, 9, 10 or 12 cells, pancake 7..12, Hanoi up to 16 disks");
}

// An instance's window: 2^(log2 n - 6 + offset) states, within 2^10 .. 2^16
// (offset: psb_engine_opts.window_bits_offset, picked by the autotuner).
int engine_window_bits(uint64_t n, int offset = 0) {
    int lg = 0;
    while (lg < 63 && (uint64_t(1) << (lg + 1)) <= n) lg++;
    return std::max(10, std::min(int(psb::kEWindowBitsMax), lg - 6 + offset));
}

uint64_t two_bit_words(uint64_t n) { return ((2 * n + 63) / 64 + 31) / 32 * 32; }

uint32_t instance_windows(uint64_t n, int wb) { return uint32_t((n + (uint64_t(1) << wb) - 1) >> wb); }

// Two 256-byte-aligned arrays of one flag byte per window, sized for the
// smallest window (2^10 states), so an instance's footprint does not depend
// on the engine's window offset.
uint64_t flag_words_for(uint64_t n) { return 2 * ((uint64_t(instance_windows(n, 10)) + 255) / 256 * 32); }

// Pool words of one instance: its two-bit array plus its window flags.
uint64_t instance_words(uint64_t n) { return two_bit_words(n) + flag_words_for(n); }

int alloc_space(psb_engine* e, uint64_t words, uint64_t* off) {
    for (auto it = e->free_space.begin(); it != e->free_space.end(); ++it) {
        if (it->second >= words) {
            *off = it->first;
            const uint64_t rest = it->second - words;
            const uint64_t at = it->first + words;
            e->free_space.erase(it);
            if (rest) e->free_space[at] = rest;
            return PSB_OK;
        }
    }
    return psb_set_error(PSB_ERR_CAPACITY, "engine pool is full");
}

void free_space(psb_engine* e, uint64_t off, uint64_t words) {
    auto it = e->free_space.emplace(off, words).first;
    auto next = std::next(it);
    if (next != e->free_space.end() && it->first + it->second == next->first) {
        it->second += next->second;
        e->free_space.erase(next);
    }
    if (it != e->free_space.begin()) {
        auto prev = std::prev(it);
        if (prev->first + prev->second == it->first) {
            prev->second += it->second;
            e->free_space.erase(it);
        }
    }
}

int record_step(psb_engine* e) {
    cudaStream_t s = e->stream;
    psb::engine_build_queue<<<1, 1024, 0, s>>>(e->d);
    psb::engine_level<<<e->grid, psb::kEThreads, e->smem, s>>>(e->d);
    psb::engine_retire<<<e->grid, 256, 0, s>>>(e->d);
    psb::engine_epilogue<<<1, 1024, 0, s>>>(e->d);
    EN_CUDA(cudaGetLastError());
    return PSB_OK;
}

}  // namespace

extern "C" {

int psb_engine_create(const psb_engine_opts* opts, psb_engine** out) {
    if (!opts || !out || opts->struct_size != sizeof(psb_engine_opts)) return psb_set_error(PSB_ERR_ARG, "bad options");
    if (opts->max_instances == 0 || opts->max_depths == 0 || opts->pool_bytes < 256)
        return psb_set_error(PSB_ERR_ARG, "max_instances, max_depths and pool_bytes must be positive");
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) return psb_set_error(PSB_ERR_NO_DEVICE, "no CUDA device visible");
    auto e = std::make_unique<psb_engine>();
    if (opts->device >= 0) EN_CUDA(cudaSetDevice(opts->device));
    EN_CUDA(cudaGetDevice(&e->device));
    e->n_slots = opts->max_instances;
    e->max_depths = opts->max_depths;
    e->pool_words = opts->pool_bytes / 8;
    e->use_graph = opts->use_graph != 0;
    e->bottom_up = opts->direction != PSB_DIR_TOP_DOWN;
    if (opts->window_bits_offset < -6 || opts->window_bits_offset > 6)
        return psb_set_error(PSB_ERR_ARG, "window_bits_offset outside -6..6");
    e->wb_offset = opts->window_bits_offset;
    EN_CUDA(cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking));
    EN_CUDA(cudaMalloc(&e->pool, e->pool_words * 8));
    e->free_space[0] = e->pool_words;
    EN_CUDA(cudaMalloc(&e->d.slots, sizeof(psb::EngineSlot) * e->n_slots));
    EN_CUDA(cudaMalloc(&e->d.stats, 8 * 8ull * e->n_slots));
    EN_CUDA(cudaMalloc(&e->d.counts, 8ull * e->n_slots * e->max_depths));
    // small counters in one allocation
    const size_t ints = size_t(e->n_slots + 1) + 5 + 2 * size_t(e->n_slots) + 2;  // + release scratch
    uint32_t* ib = nullptr;
    EN_CUDA(cudaMalloc(&ib, ints * 4 + 16));
    e->d.item_start = ib;
    e->d.queue_head = ib + e->n_slots + 1;
    e->d.n_items = e->d.queue_head + 1;
    e->d.retire_head = e->d.n_items + 1;
    e->d.done_count = e->d.retire_head + 1;
    e->d.n_active = e->d.done_count + 1;
    e->d.done_list = e->d.n_active + 1;
    EN_CUDA(cudaMalloc(&e->d.err, 8));
    EN_CUDA(cudaMemsetAsync(e->d.err, 0, 8, e->stream));
    e->d.n_slots = e->n_slots;
    e->d.max_depths = e->max_depths;
    EN_CUDA(cudaMemsetAsync(e->d.slots, 0, sizeof(psb::EngineSlot) * e->n_slots, e->stream));
    EN_CUDA(cudaMemsetAsync(e->d.stats, 0, 8 * 8ull * e->n_slots, e->stream));
    EN_CUDA(cudaMemsetAsync(ib, 0, ints * 4 + 16, e->stream));
    EN_CUDA(cudaMallocHost(&e->h_done_count, 4));
    EN_CUDA(cudaMallocHost(&e->h_err, 8));
    EN_CUDA(cudaMalloc(&e->d_staging, 8ull * e->n_slots * (e->max_depths + 2)));
    e->h_staging.resize(size_t(e->n_slots) * (e->max_depths + 2));
    e->host_slots.assign(e->n_slots, psb::EngineSlot{});
    e->slot_off.assign(e->n_slots, 0);
    e->slot_words.assign(e->n_slots, 0);
    e->slot_tag.assign(e->n_slots, 0);
    for (uint32_t i = e->n_slots; i > 0; i--) e->free_slots.push_back(i - 1);
    int sms = 0;
    EN_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, e->device));
    const int per_sm = opts->blocks_per_sm > 0 ? opts->blocks_per_sm : psb::kEMinBlocks;
    e->grid = unsigned(sms * per_sm);
    e->smem = psb::level_smem_bytes(psb::kTwoBit, size_t(1) << psb::kEWindowBitsMax, psb::kEThreads);
    EN_CUDA(cudaFuncSetAttribute(psb::engine_level, cudaFuncAttributeMaxDynamicSharedMemorySize, int(e->smem)));
    EN_CUDA(cudaStreamSynchronize(e->stream));
    if (e->use_graph) {
        EN_CUDA(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal));
        const int rc = record_step(e.get());
        cudaGraph_t g = nullptr;
        const cudaError_t ce = cudaStreamEndCapture(e->stream, &g);
        if (rc) { if (g) cudaGraphDestroy(g); return rc; }
        EN_CUDA(ce);
        e->graph = g;
        EN_CUDA(cudaGraphInstantiate(&e->exec, e->graph, 0));
    }
    *out = e.release();
    return PSB_OK;
}

int psb_engine_destroy(psb_engine* e) {
    delete e;
    return PSB_OK;
}

int psb_engine_footprint(int kind, int a, int b, uint64_t* bytes) {
    psb_puzzle* p = nullptr;
    if (int rc = psb_puzzle_create(kind, a, b, &p)) return rc;
    *bytes = instance_words(p->n_states) * 8;
    psb_puzzle_destroy(p);
    return PSB_OK;
}

int psb_engine_add(psb_engine* e, int kind, int a, int b, uint64_t initial, uint64_t tag, uint32_t* slot_out) {
    if (!e) return psb_set_error(PSB_ERR_ARG, "engine is NULL");
    uint32_t type = 0;
    if (int rc = engine_type(kind, a, b, &type)) return rc;
    psb_puzzle* p = nullptr;
    if (int rc = psb_puzzle_create(kind, a, b, &p)) return rc;
    std::unique_ptr<psb_puzzle, int (*)(psb_puzzle*)> guard(p, psb_puzzle_destroy);
    if (initial >= p->n_states) return psb_set_error(PSB_ERR_ARG, "initial index >= IndexesCount()");
    if (e->free_slots.empty()) return psb_set_error(PSB_ERR_CAPACITY, "no free instance slot");
    const int wb = engine_window_bits(p->n_states, e->wb_offset);
    const uint32_t windows = instance_windows(p->n_states, wb);
    const uint64_t code_words = two_bit_words(p->n_states);
    const uint64_t flag_words = flag_words_for(p->n_states);
    const uint64_t words = instance_words(p->n_states);
    if (words > e->pool_words)  // can never fit, however much space is freed
        return psb_set_error(PSB_ERR_NOMEM, ("search needs " + std::to_string(words * 8) +
                                             " bytes; the engine pool holds " + std::to_string(e->pool_words * 8))
                                                .c_str());
    uint64_t off = 0;
    if (int rc = alloc_space(e, words, &off)) return rc;
    const uint32_t s = e->free_slots.back();
    e->free_slots.pop_back();
    e->slot_off[s] = off;
    e->slot_words[s] = words;
    e->slot_tag[s] = tag;
    psb::EngineSlot slot{};
    slot.type = type;
    slot.state = 1;
    slot.depth = 0;
    slot.windows = windows;
    slot.flags[0] = reinterpret_cast<uint8_t*>(e->pool + off + code_words);
    slot.flags[1] = slot.flags[0] + flag_words * 4;
    psb::LevelArgs& la = slot.args;
    la.front = la.marks = e->pool + off;
    la.probe = la.front;
    slot.bu = 0;
    slot.can_bu = (e->bottom_up && !(kind == PSB_HANOI4 && b)) ? 1u : 0u;
    slot.seen = 0;
    la.n_states = p->n_states;
    la.front_words = la.mark_words = (2 * p->n_states + 63) / 64;
    la.window_bits = wb;
    la.cur_code = 2;
    la.odd = p->odd;
    la.pz = p->pz;
    la.stats = e->d.stats + 8ull * s;
    // Level 0 sweeps only the start state's window and records flags for level 1.
    la.wflag_cur = slot.flags[0];
    la.wflag_next = slot.flags[1];
    cudaStream_t st = e->stream;
    EN_CUDA(cudaMemsetAsync(e->pool + off, 0, words * 8, st));
    static thread_local uint8_t one;
    one = 1;
    EN_CUDA(cudaMemcpyAsync(slot.flags[0] + (initial >> wb), &one, 1, cudaMemcpyHostToDevice, st));
    static thread_local uint64_t word;
    word = uint64_t(1) << ((2 * initial) & 63);  // code CUR = 2 at the initial state: bit 2i
    EN_CUDA(cudaMemcpyAsync(e->pool + off + (2 * initial) / 64, &word, 8, cudaMemcpyHostToDevice, st));
    EN_CUDA(cudaMemsetAsync(e->d.stats + 8ull * s, 0, 64, st));
    e->host_slots[s] = slot;
    EN_CUDA(cudaMemcpyAsync(e->d.slots + s, &e->host_slots[s], sizeof(psb::EngineSlot), cudaMemcpyHostToDevice, st));
    EN_CUDA(cudaStreamSynchronize(st));
    e->active++;
    *slot_out = s;
    return PSB_OK;
}

int psb_engine_step(psb_engine* e, uint32_t levels) {
    if (!e) return psb_set_error(PSB_ERR_ARG, "engine is NULL");
    for (uint32_t l = 0; l < levels; l++) {
        if (e->use_graph) EN_CUDA(cudaGraphLaunch(e->exec, e->stream));
        else if (int rc = record_step(e)) return rc;
        e->levels_run++;
    }
    // One host round trip per step: the error word and the completion count
    // together (psb_engine_poll reuses the count).
    EN_CUDA(cudaMemcpyAsync(e->h_err, e->d.err, 8, cudaMemcpyDeviceToHost, e->stream));
    EN_CUDA(cudaMemcpyAsync(e->h_done_count, e->d.done_count, 4, cudaMemcpyDeviceToHost, e->stream));
    EN_CUDA(cudaStreamSynchronize(e->stream));
    e->done_fresh = true;
    const unsigned long long err = *e->h_err;
    if (err & 1) return psb_set_error(PSB_ERR_DEVICE, "a level produced a child index >= IndexesCount()");
    if (err & 2) return psb_set_error(PSB_ERR_CAPACITY, "an instance has more depths than max_depths");
    return PSB_OK;
}

int psb_engine_poll(psb_engine* e, uint64_t* tags, uint32_t* n_depths, uint64_t* counts, uint32_t cap, uint32_t* n) {
    if (!e || !n || (cap && (!tags || !n_depths || !counts))) return psb_set_error(PSB_ERR_ARG, "bad argument");
    *n = 0;
    cudaStream_t st = e->stream;
    if (!e->done_fresh) {
        EN_CUDA(cudaMemcpyAsync(e->h_done_count, e->d.done_count, 4, cudaMemcpyDeviceToHost, st));
        EN_CUDA(cudaStreamSynchronize(st));
    }
    const uint32_t done = *e->h_done_count;
    const uint32_t k = std::min(cap, done - e->done_seen);
    if (k == 0) return PSB_OK;
    e->done_fresh = false;  // the release below changes the ring
    const size_t row = size_t(e->max_depths) + 2;
    psb::engine_collect<<<k, 128, 0, st>>>(e->d, e->done_seen, k, e->d_staging);
    EN_CUDA(cudaGetLastError());
    EN_CUDA(cudaMemcpyAsync(e->h_staging.data(), e->d_staging, 8 * row * k, cudaMemcpyDeviceToHost, st));
    EN_CUDA(cudaStreamSynchronize(st));
    std::vector<uint32_t> released(k);
    for (uint32_t i = 0; i < k; i++) {
        const unsigned long long* r = e->h_staging.data() + row * i;
        const uint32_t s = uint32_t(r[0]);
        tags[i] = e->slot_tag[s];
        n_depths[i] = uint32_t(r[1]);
        std::memcpy(counts + uint64_t(i) * e->max_depths, r + 2, 8ull * e->max_depths);
        free_space(e, e->slot_off[s], e->slot_words[s]);
        e->free_slots.push_back(s);
        released[i] = s;
    }
    uint32_t* d_rel = e->d.done_list + e->n_slots;  // scratch after the ring
    EN_CUDA(cudaMemcpyAsync(d_rel, released.data(), 4ull * k, cudaMemcpyHostToDevice, st));
    psb::engine_release<<<(k + 255) / 256, 256, 0, st>>>(e->d, d_rel, k);
    EN_CUDA(cudaGetLastError());
    EN_CUDA(cudaStreamSynchronize(st));
    e->done_seen += k;
    e->active -= k;
    *n = k;
    return PSB_OK;
}

int psb_engine_info(psb_engine* e, uint32_t* active, uint64_t* free_bytes, uint64_t* levels_run) {
    if (!e) return psb_set_error(PSB_ERR_ARG, "engine is NULL");
    if (active) *active = e->active;
    if (free_bytes) {
        uint64_t best = 0;
        for (auto& kv : e->free_space) best = std::max(best, kv.second);
        *free_bytes = best * 8;
    }
    if (levels_run) *levels_run = e->levels_run;
    return PSB_OK;
}

}  // extern "C"
