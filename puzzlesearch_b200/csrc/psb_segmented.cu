// psb_segmented.cu -- psb_bfs_segmented: a search over a state space split
// into segments of 2^segment_bits states, holding only one segment's bit
// arrays in device memory at a time.  Everything else lives in host memory:
// every segment's last three frontier layers as compressed segment streams,
// and the children each segment's new states have in other segments.
//
// It restates the reference's out-of-core three-layer search,
// DiskBasedOptThreeBitBFS (Common/DiskBasedOptThreeBitBFS.cpp:12-252), whose
// segment files become host buffers and whose per-segment loops become
// device kernels.  For depth d, segment g:
//   1. next  = the children that segment g received from the other segments'
//              states at depth d (their offsets, collected one step earlier);
//   2. next |= the children inside g of g's depth-d states (decoded from
//              g's layer d);
//   3. next &= ~(g's layer d-1), and &= ~(g's layer d) on puzzles with odd
//              cycles; its set bits are g's states at depth d+1: counted and
//              encoded as g's layer d+1 (the reference's segment stream);
//   4. the children outside g of those new states are collected, by target
//      segment, for step 1 of depth d+1.
// The counts equal the in-memory searches' (and the reference's disk-based
// searches'): every state is expanded once into its own segment (step 2, one
// depth after it is found) and once into the others (step 4, when found).
//
// Host traffic per depth: each segment's layers (about half a byte per state
// of the frontier) and 4 bytes per cross-segment child, both ways over PCIe.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/psb200.h"
#include "psb_internal.h"

namespace psb {

// new &= ~old (& ~cur on puzzles with odd cycles); count = popc(new).
__global__ void __launch_bounds__(kThreads) seg_finish(uint64_t* __restrict__ nw, const uint64_t* __restrict__ old,
                                                      const uint64_t* __restrict__ cur, uint64_t words, int odd,
                                                      unsigned long long* count) {
    uint32_t c = 0;
    for (uint64_t i = blockIdx.x * uint64_t(kThreads) + threadIdx.x; i < words; i += uint64_t(gridDim.x) * kThreads) {
        uint64_t v = nw[i] & ~old[i];
        if (odd) v &= ~cur[i];
        nw[i] = v;
        c += __popcll(v);
    }
    c = __reduce_add_sync(0xFFFFFFFFu, c);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(count, (unsigned long long)c);
}

// ORs segment-relative offsets into a segment bitmap.
__global__ void __launch_bounds__(kThreads) seg_set_offsets(uint64_t* __restrict__ bits,
                                                           const uint32_t* __restrict__ offs, uint64_t n) {
    for (uint64_t i = blockIdx.x * uint64_t(kThreads) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * kThreads) {
        const uint32_t o = offs[i];
        atomicOr(reinterpret_cast<unsigned int*>(bits) + (o >> 5), 1u << (o & 31u));
    }
}

// Partition of cross-segment children by target segment: a histogram, then
// a scatter of each child's offset into its segment's run (order within a
// run does not matter: the offsets are ORed into a bitmap).
__global__ void __launch_bounds__(kThreads) seg_histogram(const uint64_t* __restrict__ kids, uint64_t n, int sb,
                                                         unsigned int* __restrict__ hist) {
    for (uint64_t i = blockIdx.x * uint64_t(kThreads) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * kThreads)
        atomicAdd(&hist[kids[i] >> sb], 1u);
}
__global__ void __launch_bounds__(kThreads) seg_scatter(const uint64_t* __restrict__ kids, uint64_t n, int sb,
                                                       unsigned int* __restrict__ cursor,
                                                       uint32_t* __restrict__ out) {
    const uint64_t mask = (sb >= 64) ? ~uint64_t(0) : ((uint64_t(1) << sb) - 1);
    for (uint64_t i = blockIdx.x * uint64_t(kThreads) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * kThreads) {
        const uint64_t c = kids[i];
        const unsigned int pos = atomicAdd(&cursor[c >> sb], 1u);
        out[pos] = uint32_t(c & mask);
    }
}

}  // namespace psb

namespace {

#define SG_CUDA(call)                                                                                   \
    do {                                                                                                \
        cudaError_t e_ = (call);                                                                        \
        if (e_ != cudaSuccess)                                                                          \
            return psb_set_error(PSB_ERR_CUDA, (std::string(#call) + ": " + cudaGetErrorString(e_)).c_str()); \
    } while (0)

// One segment's frontier layer: the reference's compressed segment stream
// and its block table (for the device decoder).
struct Layer {
    std::vector<uint8_t> bytes;
    std::vector<psb_codec_block> blocks;
    uint64_t count = 0;
};

template <class T>
struct DevBuf {
    T* p = nullptr;
    uint64_t cap = 0;  // elements
    ~DevBuf() { cudaFree(p); }
    int grow(uint64_t n) {
        if (n <= cap) return PSB_OK;
        cudaFree(p);
        p = nullptr;
        cap = 0;
        const uint64_t want = n + n / 4;
        SG_CUDA(cudaMalloc(reinterpret_cast<void**>(&p), want * sizeof(T)));
        cap = want;
        return PSB_OK;
    }
};

struct Run {
    const psb_puzzle* P = nullptr;
    cudaStream_t s = nullptr;
    int sb = 0;
    uint64_t seg_states = 0, seg_words = 0, n_segments = 0;
    uint64_t chunk_words = 0;
    DevBuf<uint64_t> next, cur, old, kids;
    DevBuf<uint32_t> offs;
    DevBuf<uint8_t> stream_buf[2];  // the two layers decoded for one segment
    DevBuf<psb_codec_block> block_tab[2];
    DevBuf<unsigned int> hist;
    DevBuf<unsigned long long> scalars;  // [0] count, [1] children appended, [2] error flag, [3] decode error
    psb::SegmentEncoder* enc = nullptr;  // device scratch kept from segment to segment
    psb_segmented_stats st{};

    ~Run() { if (enc) psb::encoder_destroy(enc); }

    uint64_t states_in(uint64_t g) const { return std::min(seg_states, P->n_states - g * seg_states); }

    // Decodes a layer into a cleared segment bitmap (slot 0 or 1: the two
    // layers of one segment are in flight together).  Nothing waits: a bad
    // offset sets scalars[3], read at the end of the depth.
    int decode(const Layer& L, uint64_t* bits, uint64_t g, int slot) {
        SG_CUDA(cudaMemsetAsync(bits, 0, seg_words * 8, s));
        if (L.count == 0) return PSB_OK;
        if (int rc = stream_buf[slot].grow(L.bytes.size())) return rc;
        if (int rc = block_tab[slot].grow(L.blocks.size())) return rc;
        SG_CUDA(cudaMemcpyAsync(stream_buf[slot].p, L.bytes.data(), L.bytes.size(), cudaMemcpyHostToDevice, s));
        SG_CUDA(cudaMemcpyAsync(block_tab[slot].p, L.blocks.data(), L.blocks.size() * sizeof(psb_codec_block),
                                cudaMemcpyHostToDevice, s));
        st.h2d_bytes += L.bytes.size();
        return psb::frontier_decode_async(stream_buf[slot].p, block_tab[slot].p, uint32_t(L.blocks.size()), bits,
                                          states_in(g), scalars.p + 3, s);
    }

    // Encodes a segment bitmap holding `count` states into a layer.
    int encode(const uint64_t* bits, uint64_t g, uint64_t count, Layer* L) {
        L->bytes.clear();
        L->blocks.clear();
        L->count = count;
        if (count == 0) return PSB_OK;
        uint64_t bytes = 0, n = 0;
        if (int rc = psb::encoder_plan(enc, bits, states_in(g), s, false, &bytes, &n)) return rc;
        if (n != count) return psb_set_error(PSB_ERR_DEVICE, "segmented search: layer count mismatch");
        if (int rc = stream_buf[0].grow(bytes)) return rc;
        if (int rc = psb::encoder_write(enc, stream_buf[0].p, s)) return rc;
        L->bytes.resize(bytes);
        SG_CUDA(cudaMemcpyAsync(L->bytes.data(), stream_buf[0].p, bytes, cudaMemcpyDeviceToHost, s));
        SG_CUDA(cudaStreamSynchronize(s));
        // The block table, for the decoder: read back from the stream's own headers.
        uint32_t nb = 0;
        if (int rc = psb_frontier_index(L->bytes.data(), bytes, nullptr, 0, &nb)) return rc;
        L->blocks.resize(nb);
        if (int rc = psb_frontier_index(L->bytes.data(), bytes, L->blocks.data(), nb, &nb)) return rc;
        st.d2h_bytes += bytes;
        return PSB_OK;
    }

    // ORs the offsets a segment received into `bits`.
    int receive(const std::vector<uint32_t>& list, uint64_t* bits) {
        for (uint64_t at = 0; at < list.size(); at += offs.cap) {
            const uint64_t n = std::min<uint64_t>(offs.cap, list.size() - at);
            SG_CUDA(cudaMemcpyAsync(offs.p, list.data() + at, n * 4, cudaMemcpyHostToDevice, s));
            st.h2d_bytes += n * 4;
            psb::seg_set_offsets<<<unsigned(std::min<uint64_t>((n + psb::kThreads - 1) / psb::kThreads, 148 * 16)),
                                   psb::kThreads, 0, s>>>(bits, offs.p, n);
            SG_CUDA(cudaGetLastError());
            SG_CUDA(cudaStreamSynchronize(s));  // the staging buffer is reused
        }
        return PSB_OK;
    }

    // Expands the states of `bits` (segment g) chunk by chunk: cross == 0
    // marks the children inside g in `next`; cross == 1 appends the offsets
    // of the children outside g to their target segments' lists.
    int expand(const uint64_t* bits, uint64_t g, int cross, std::vector<std::vector<uint32_t>>* lists) {
        psb::SegExpandArgs a{};
        a.bits = bits;
        a.seg_base = g * seg_states;
        a.seg_states = states_in(g);
        a.next = next.p;
        a.out = kids.p;
        a.out_n = scalars.p + 1;
        a.out_cap = kids.cap;
        a.n_states = P->n_states;
        a.cross = cross;
        a.pz = P->pz;
        a.err = scalars.p + 2;
        for (uint64_t w = 0; w < seg_words; w += chunk_words) {
            a.word_lo = w;
            a.word_hi = std::min(seg_words, w + chunk_words);
            SG_CUDA(cudaMemsetAsync(scalars.p + 1, 0, 8, s));
            const unsigned grid = unsigned(std::min<uint64_t>((a.word_hi - w + psb::kThreads - 1) / psb::kThreads,
                                                              148 * 8));
            SG_CUDA(P->k.segment_expand(a, grid, s));
            if (!cross) continue;
            unsigned long long n = 0;
            SG_CUDA(cudaMemcpyAsync(&n, scalars.p + 1, 8, cudaMemcpyDeviceToHost, s));
            SG_CUDA(cudaStreamSynchronize(s));
            if (n > kids.cap) return psb_set_error(PSB_ERR_DEVICE, "segmented search: child buffer overflow");
            if (n == 0) continue;
            st.cross_children += n;
            SG_CUDA(cudaMemsetAsync(hist.p, 0, n_segments * 4, s));
            const unsigned pg = unsigned(std::min<uint64_t>((n + psb::kThreads - 1) / psb::kThreads, 148 * 16));
            psb::seg_histogram<<<pg, psb::kThreads, 0, s>>>(kids.p, n, sb, hist.p);
            std::vector<unsigned int> h(n_segments);
            SG_CUDA(cudaMemcpyAsync(h.data(), hist.p, n_segments * 4, cudaMemcpyDeviceToHost, s));
            SG_CUDA(cudaStreamSynchronize(s));
            std::vector<unsigned int> start(n_segments);
            unsigned int acc = 0;
            for (uint64_t t = 0; t < n_segments; t++) { start[t] = acc; acc += h[t]; }
            SG_CUDA(cudaMemcpyAsync(hist.p, start.data(), n_segments * 4, cudaMemcpyHostToDevice, s));
            if (int rc = offs.grow(n)) return rc;
            psb::seg_scatter<<<pg, psb::kThreads, 0, s>>>(kids.p, n, sb, hist.p, offs.p);
            SG_CUDA(cudaGetLastError());
            std::vector<uint32_t> host(n);
            SG_CUDA(cudaMemcpyAsync(host.data(), offs.p, n * 4, cudaMemcpyDeviceToHost, s));
            SG_CUDA(cudaStreamSynchronize(s));
            st.d2h_bytes += n * 4;
            for (uint64_t t = 0; t < n_segments; t++)
                if (h[t]) (*lists)[t].insert((*lists)[t].end(), host.begin() + start[t], host.begin() + start[t] + h[t]);
        }
        SG_CUDA(cudaStreamSynchronize(s));
        return PSB_OK;
    }
};

uint64_t host_bytes(const std::vector<Layer>& a, const std::vector<Layer>& b, const std::vector<Layer>& c,
                    const std::vector<std::vector<uint32_t>>& x, const std::vector<std::vector<uint32_t>>& y) {
    uint64_t n = 0;
    for (auto* v : {&a, &b, &c})
        for (const Layer& L : *v) n += L.bytes.size();
    for (auto* v : {&x, &y})
        for (const auto& l : *v) n += l.size() * 4;
    return n;
}

}  // namespace

extern "C" int psb_bfs_segmented(const psb_puzzle* p, uint64_t initial, const psb_segmented_opts* opts,
                                 uint64_t* counts, uint32_t cap, uint32_t* n_depths, psb_segmented_stats* stats) {
    if (!p || !counts || !n_depths || cap == 0) return psb_set_error(PSB_ERR_ARG, "bad argument");
    if (opts && opts->struct_size != sizeof(psb_segmented_opts))
        return psb_set_error(PSB_ERR_ARG, "psb_segmented_opts.struct_size mismatch");
    if (initial >= p->n_states) return psb_set_error(PSB_ERR_ARG, "initial index >= IndexesCount()");
    const int sb = opts && opts->segment_bits ? opts->segment_bits : 32;
    if (sb < 10 || sb > 32) return psb_set_error(PSB_ERR_ARG, "segment_bits outside 10..32");
    int dev_count = 0;
    if (cudaGetDeviceCount(&dev_count) != cudaSuccess || dev_count == 0)
        return psb_set_error(PSB_ERR_NO_DEVICE, "no CUDA device visible");
    if (opts && opts->device >= 0) SG_CUDA(cudaSetDevice(opts->device));
    const auto t0 = std::chrono::steady_clock::now();

    Run R;
    R.P = p;
    R.sb = sb;
    R.seg_states = std::min<uint64_t>(uint64_t(1) << sb, p->n_states);
    R.seg_words = (R.seg_states + 63) / 64;
    R.n_segments = (p->n_states + (uint64_t(1) << sb) - 1) >> sb;
    if (R.n_segments > (uint64_t(1) << 20)) return psb_set_error(PSB_ERR_ARG, "more than 2^20 segments");
    // Expansion chunk: its children fit the child buffer even if every state is set.
    R.chunk_words = std::min<uint64_t>(R.seg_words, opts && opts->chunk_states ? std::max<uint64_t>(1, opts->chunk_states / 64)
                                                                                 : uint64_t(1) << 16);
    SG_CUDA(cudaStreamCreateWithFlags(&R.s, cudaStreamNonBlocking));
    struct StreamGuard { cudaStream_t s; ~StreamGuard() { cudaStreamSynchronize(s); cudaStreamDestroy(s); } } guard{R.s};
    for (auto* b : {&R.next, &R.cur, &R.old})
        if (int rc = b->grow(R.seg_words)) return rc;
    if (int rc = R.kids.grow(R.chunk_words * 64 * uint64_t(p->branching))) return rc;
    R.kids.cap = R.chunk_words * 64 * uint64_t(p->branching);
    if (int rc = R.offs.grow(uint64_t(1) << 22)) return rc;
    if (int rc = R.hist.grow(R.n_segments)) return rc;
    if (int rc = R.scalars.grow(4)) return rc;
    if (int rc = R.stream_buf[0].grow(uint64_t(1) << 20)) return rc;
    if (!(R.enc = psb::encoder_create())) return psb_set_error(PSB_ERR_NOMEM, "segmented search: encoder");
    SG_CUDA(cudaMemsetAsync(R.scalars.p, 0, 4 * 8, R.s));

    const uint64_t S = R.n_segments;
    std::vector<Layer> old_l(S), cur_l(S), new_l(S);
    std::vector<std::vector<uint32_t>> recv(S), recv_next(S);

    // Depth 0: the initial state is segment g0's layer; its children in the
    // other segments are collected at once (SetInitialNode,
    // DiskBasedOptThreeBitBFS.cpp:34-53).
    const uint64_t g0 = initial >> sb;
    {
        SG_CUDA(cudaMemsetAsync(R.next.p, 0, R.seg_words * 8, R.s));
        const uint64_t off = initial - g0 * R.seg_states;
        const uint64_t word = uint64_t(1) << (off & 63);
        SG_CUDA(cudaMemcpyAsync(R.next.p + off / 64, &word, 8, cudaMemcpyHostToDevice, R.s));
        if (int rc = R.encode(R.next.p, g0, 1, &cur_l[g0])) return rc;
        if (int rc = R.expand(R.next.p, g0, 1, &recv)) return rc;
    }
    std::vector<uint64_t> res{1};
    const uint32_t max_depth = opts ? opts->max_depth : 0;
    const bool odd = p->odd != 0;
    for (;;) {
        if (max_depth && res.size() >= size_t(max_depth) + 1) break;
        uint64_t total = 0;
        for (uint64_t g = 0; g < S; g++) {
            if (cur_l[g].count == 0 && recv[g].empty()) {  // no state of depth d+1 can be in g
                new_l[g] = Layer();
                continue;
            }
            SG_CUDA(cudaMemsetAsync(R.next.p, 0, R.seg_words * 8, R.s));
            if (int rc = R.receive(recv[g], R.next.p)) return rc;
            std::vector<uint32_t>().swap(recv[g]);
            if (int rc = R.decode(cur_l[g], R.cur.p, g, 0)) return rc;
            if (cur_l[g].count)
                if (int rc = R.expand(R.cur.p, g, 0, nullptr)) return rc;
            if (int rc = R.decode(old_l[g], R.old.p, g, 1)) return rc;
            SG_CUDA(cudaMemsetAsync(R.scalars.p, 0, 8, R.s));
            psb::seg_finish<<<148 * 8, psb::kThreads, 0, R.s>>>(R.next.p, R.old.p, R.cur.p, R.seg_words, odd ? 1 : 0,
                                                               R.scalars.p);
            SG_CUDA(cudaGetLastError());
            unsigned long long c = 0;
            SG_CUDA(cudaMemcpyAsync(&c, R.scalars.p, 8, cudaMemcpyDeviceToHost, R.s));
            SG_CUDA(cudaStreamSynchronize(R.s));
            total += c;
            if (int rc = R.encode(R.next.p, g, c, &new_l[g])) return rc;
            if (c)
                if (int rc = R.expand(R.next.p, g, 1, &recv_next)) return rc;
            R.st.peak_host_bytes = std::max(R.st.peak_host_bytes, host_bytes(old_l, cur_l, new_l, recv, recv_next));
        }
        unsigned long long err[2] = {0, 0};
        SG_CUDA(cudaMemcpyAsync(err, R.scalars.p + 2, 16, cudaMemcpyDeviceToHost, R.s));
        SG_CUDA(cudaStreamSynchronize(R.s));
        if (err[0]) return psb_set_error(PSB_ERR_DEVICE, "segmented search produced a child index >= IndexesCount()");
        if (err[1]) return psb_set_error(PSB_ERR_DEVICE, "segmented search: a layer decoded outside its segment");
        if (total == 0) break;
        if (res.size() >= cap) return psb_set_error(PSB_ERR_CAPACITY, "more depths than counts_cap");
        res.push_back(total);
        // layers: old <- cur <- new; received children: the next step's
        old_l.swap(cur_l);
        cur_l.swap(new_l);
        recv.swap(recv_next);
        for (auto& l : recv_next) std::vector<uint32_t>().swap(l);
    }
    std::copy(res.begin(), res.end(), counts);
    *n_depths = uint32_t(res.size());
    if (stats && stats->struct_size >= sizeof(psb_segmented_stats)) {
        R.st.struct_size = stats->struct_size;
        R.st.segments = S;
        R.st.device_bytes = (R.next.cap + R.cur.cap + R.old.cap + R.kids.cap) * 8 + R.offs.cap * 4 +
                            R.stream_buf[0].cap + R.stream_buf[1].cap;
        R.st.total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        *stats = R.st;
    }
    return PSB_OK;
}
