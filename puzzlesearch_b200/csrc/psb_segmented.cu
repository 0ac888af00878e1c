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

// Staged cross-segment children of one target segment are written to the
// store in chunks of up to this many offsets (the reference's Multiplexor
// buffers, Common/Multiplexor.cpp:5-33), fewer when there are many segments.
constexpr uint64_t kStageMax = 16384;
constexpr uint64_t kStageBudget = uint64_t(1) << 26;  // bytes of staging over all segments

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
    psb::DecodeScratch* dec = nullptr;
    std::vector<uint8_t> host_stream;    // one layer between the store and the device
    std::vector<psb_codec_block> blocks;
    std::vector<uint32_t> host_offs;     // cross-segment children between the device and the staging
    // Multiplexor staging: per target segment, the offsets not yet written.
    uint64_t stage_cap = 0;
    std::vector<uint32_t> stage;
    std::vector<uint32_t> stage_len;
    bool files = false;                  // the stores are files (else host memory)
    psb_segmented_stats st{};

    ~Run() {
        if (enc) psb::encoder_destroy(enc);
        if (dec) psb::decoder_destroy(dec);
    }

    uint64_t states_in(uint64_t g) const { return std::min(seg_states, P->n_states - g * seg_states); }

    // Decodes segment g's layer from `store` into a cleared segment bitmap
    // (slot 0 or 1: the two layers of one segment are in flight together).
    // Nothing waits on the device: a bad offset sets scalars[3], read at the
    // end of the depth.
    int decode(psb::StoreImpl& store, uint64_t* bits, uint64_t g, int slot) {
        SG_CUDA(cudaMemsetAsync(bits, 0, seg_words * 8, s));
        const uint64_t bytes = psb::store_length(store, int(g));
        if (bytes == 0) return PSB_OK;
        if (host_stream.size() < bytes) host_stream.resize(bytes);
        psb::store_rewind(store, int(g));
        uint64_t got = 0;
        if (int rc = psb::store_read(store, int(g), host_stream.data(), bytes, &got)) return rc;
        if (got != bytes) return psb_set_error(PSB_ERR_IO, "segmented search: a layer came back short");
        uint32_t nb = 0;
        if (int rc = psb_frontier_index(host_stream.data(), bytes, nullptr, 0, &nb)) return rc;
        blocks.resize(nb);
        if (int rc = psb_frontier_index(host_stream.data(), bytes, blocks.data(), nb, &nb)) return rc;
        if (int rc = stream_buf[slot].grow(bytes)) return rc;
        if (int rc = block_tab[slot].grow(nb)) return rc;
        // Pageable sources: both copies have left host memory when the calls return.
        SG_CUDA(cudaMemcpyAsync(stream_buf[slot].p, host_stream.data(), bytes, cudaMemcpyHostToDevice, s));
        SG_CUDA(cudaMemcpyAsync(block_tab[slot].p, blocks.data(), nb * sizeof(psb_codec_block),
                                cudaMemcpyHostToDevice, s));
        st.h2d_bytes += bytes;
        return psb::frontier_decode_async(stream_buf[slot].p, host_stream.data(), blocks.data(), block_tab[slot].p,
                                          nb, bits, states_in(g), scalars.p + 3, dec, s);
    }

    // Encodes a segment bitmap holding `count` states as segment g's layer in `store`.
    int encode(const uint64_t* bits, uint64_t g, uint64_t count, psb::StoreImpl& store) {
        if (count == 0) return PSB_OK;
        uint64_t bytes = 0, n = 0;
        if (int rc = psb::encoder_plan(enc, bits, states_in(g), s, false, &bytes, &n)) return rc;
        if (n != count) return psb_set_error(PSB_ERR_DEVICE, "segmented search: layer count mismatch");
        if (int rc = stream_buf[0].grow(bytes)) return rc;
        if (int rc = psb::encoder_write(enc, stream_buf[0].p, s)) return rc;
        if (host_stream.size() < bytes) host_stream.resize(bytes);
        SG_CUDA(cudaMemcpyAsync(host_stream.data(), stream_buf[0].p, bytes, cudaMemcpyDeviceToHost, s));
        SG_CUDA(cudaStreamSynchronize(s));
        st.d2h_bytes += bytes;
        return psb::store_write(store, int(g), host_stream.data(), bytes);
    }

    // ORs the offsets segment g received (its chunks in `store`) into `bits`,
    // then drops them from the store.
    int receive(psb::StoreImpl& store, uint64_t g, uint64_t* bits) {
        const uint64_t bytes = psb::store_length(store, int(g));
        if (bytes == 0) return PSB_OK;
        if (host_offs.size() < bytes / 4) host_offs.resize(bytes / 4);
        psb::store_rewind(store, int(g));
        uint64_t n = 0;
        for (;;) {
            uint64_t got = 0;
            if (int rc = psb::store_read(store, int(g), host_offs.data() + n, bytes - n * 4, &got)) return rc;
            if (got == 0) break;
            n += got / 4;
        }
        if (int rc = offs.grow(n)) return rc;
        SG_CUDA(cudaMemcpyAsync(offs.p, host_offs.data(), n * 4, cudaMemcpyHostToDevice, s));
        st.h2d_bytes += n * 4;
        psb::seg_set_offsets<<<unsigned(std::min<uint64_t>((n + psb::kThreads - 1) / psb::kThreads, 148 * 16)),
                               psb::kThreads, 0, s>>>(bits, offs.p, n);
        SG_CUDA(cudaGetLastError());
        return psb::store_erase(store, int(g));
    }

    // Appends offsets for target segment t to its staging, writing full
    // stages to `store` (Multiplexor::Add, Common/Multiplexor.cpp:10-19).
    int stage_add(psb::StoreImpl& store, uint64_t t, const uint32_t* v, uint64_t n) {
        uint32_t* buf = stage.data() + t * stage_cap;
        while (n) {
            const uint64_t k = std::min<uint64_t>(n, stage_cap - stage_len[t]);
            std::memcpy(buf + stage_len[t], v, k * 4);
            stage_len[t] += uint32_t(k);
            v += k;
            n -= k;
            if (stage_len[t] == stage_cap) {
                if (int rc = psb::store_write(store, int(t), buf, stage_cap * 4)) return rc;
                stage_len[t] = 0;
            }
        }
        return PSB_OK;
    }
    int stage_flush(psb::StoreImpl& store) {  // Multiplexor::FlushAllSegments
        for (uint64_t t = 0; t < n_segments; t++) {
            if (!stage_len[t]) continue;
            if (int rc = psb::store_write(store, int(t), stage.data() + t * stage_cap, uint64_t(stage_len[t]) * 4))
                return rc;
            stage_len[t] = 0;
        }
        return PSB_OK;
    }

    // Expands the states of `bits` (segment g) chunk by chunk: with no store
    // it marks the children inside g in `next`; with one it stages the
    // offsets of the children outside g for their target segments.
    int expand(const uint64_t* bits, uint64_t g, psb::StoreImpl* cross_store) {
        const int cross = cross_store != nullptr;
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
        std::vector<unsigned int> h(cross ? n_segments : 0), start(cross ? n_segments : 0);
        for (uint64_t w = 0; w < seg_words; w += chunk_words) {
            a.word_lo = w;
            a.word_hi = std::min(seg_words, w + chunk_words);
            SG_CUDA(cudaMemsetAsync(scalars.p + 1, 0, 8, s));
            // one warp per 32 words
            const uint64_t warps = (a.word_hi - w + 31) / 32;
            const unsigned grid = unsigned(std::min<uint64_t>((warps * 32 + psb::kThreads - 1) / psb::kThreads, 148 * 8));
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
            SG_CUDA(cudaMemcpyAsync(h.data(), hist.p, n_segments * 4, cudaMemcpyDeviceToHost, s));
            SG_CUDA(cudaStreamSynchronize(s));
            unsigned int acc = 0;
            for (uint64_t t = 0; t < n_segments; t++) { start[t] = acc; acc += h[t]; }
            SG_CUDA(cudaMemcpyAsync(hist.p, start.data(), n_segments * 4, cudaMemcpyHostToDevice, s));
            if (int rc = offs.grow(n)) return rc;
            psb::seg_scatter<<<pg, psb::kThreads, 0, s>>>(kids.p, n, sb, hist.p, offs.p);
            SG_CUDA(cudaGetLastError());
            if (host_offs.size() < n) host_offs.resize(n);
            SG_CUDA(cudaMemcpyAsync(host_offs.data(), offs.p, n * 4, cudaMemcpyDeviceToHost, s));
            SG_CUDA(cudaStreamSynchronize(s));
            st.d2h_bytes += n * 4;
            for (uint64_t t = 0; t < n_segments; t++)
                if (h[t])
                    if (int rc = stage_add(*cross_store, t, host_offs.data() + start[t], h[t])) return rc;
        }
        SG_CUDA(cudaStreamSynchronize(s));
        return PSB_OK;
    }
};

}  // namespace

extern "C" int psb_bfs_segmented(const psb_puzzle* p, uint64_t initial, const psb_segmented_opts* opts,
                                 uint64_t* counts, uint32_t cap, uint32_t* n_depths, psb_segmented_stats* stats) {
    if (!p || !counts || !n_depths || cap == 0) return psb_set_error(PSB_ERR_ARG, "bad argument");
    if (opts && opts->struct_size != sizeof(psb_segmented_opts))
        return psb_set_error(PSB_ERR_ARG, "psb_segmented_opts.struct_size mismatch");
    if (initial >= p->n_states) return psb_set_error(PSB_ERR_ARG, "initial index >= IndexesCount()");
    const int sb = opts && opts->segment_bits ? opts->segment_bits : 32;
    if (sb < 10 || sb > 32) return psb_set_error(PSB_ERR_ARG, "segment_bits outside 10..32");
    std::vector<std::string> dirs;
    if (opts && opts->n_directories > 0) {
        if (!opts->directories) return psb_set_error(PSB_ERR_ARG, "directories is NULL");
        for (int i = 0; i < opts->n_directories; i++) {
            if (!opts->directories[i] || !*opts->directories[i]) return psb_set_error(PSB_ERR_ARG, "empty directory");
            dirs.emplace_back(opts->directories[i]);
        }
    }
    const int files_per_path = opts && opts->files_per_path >= 0 ? opts->files_per_path : 5;
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
    const uint64_t S = R.n_segments;
    R.stage_cap = std::max<uint64_t>(64, std::min<uint64_t>(kStageMax, kStageBudget / 4 / S));
    R.stage.assign(S * R.stage_cap, 0);
    R.stage_len.assign(S, 0);
    R.files = !dirs.empty();

    // The segment stores: three frontier layers (old, cur, new, rotating) and
    // the cross-segment children received for this depth and the next
    // (the reference's DiskBasedOptThreeBitBFS keeps the same five sets,
    // Common/DiskBasedOptThreeBitBFS.cpp:20-33).
    psb::StorePtr layer[3], xseg[2];
    for (int i = 0; i < 3; i++)
        if (int rc = psb::store_create(int(S), "layer" + std::to_string(i), dirs, files_per_path, &layer[i])) return rc;
    for (int i = 0; i < 2; i++)
        if (int rc = psb::store_create(int(S), "xseg" + std::to_string(i), dirs, files_per_path, &xseg[i])) return rc;
    std::vector<uint64_t> cnt_old(S, 0), cnt_cur(S, 0), cnt_new(S, 0);
    psb::StoreImpl *old_s = layer[0].get(), *cur_s = layer[1].get(), *new_s = layer[2].get();
    psb::StoreImpl *recv_s = xseg[0].get(), *next_s = xseg[1].get();
    auto store_bytes = [&]() {
        uint64_t n = 0;
        for (auto* x : {old_s, cur_s, new_s, recv_s, next_s}) n += psb::store_total(*x);
        return n;
    };

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
    if (!(R.dec = psb::decoder_create())) return psb_set_error(PSB_ERR_NOMEM, "segmented search: decoder");
    SG_CUDA(cudaMemsetAsync(R.scalars.p, 0, 4 * 8, R.s));

    // Depth 0: the initial state is segment g0's layer; its children in the
    // other segments are collected at once (SetInitialNode,
    // DiskBasedOptThreeBitBFS.cpp:34-53).
    const uint64_t g0 = initial >> sb;
    {
        SG_CUDA(cudaMemsetAsync(R.next.p, 0, R.seg_words * 8, R.s));
        const uint64_t off = initial - g0 * R.seg_states;
        const uint64_t word = uint64_t(1) << (off & 63);
        SG_CUDA(cudaMemcpyAsync(R.next.p + off / 64, &word, 8, cudaMemcpyHostToDevice, R.s));
        if (int rc = R.encode(R.next.p, g0, 1, *cur_s)) return rc;
        cnt_cur[g0] = 1;
        if (int rc = R.expand(R.next.p, g0, recv_s)) return rc;
        if (int rc = R.stage_flush(*recv_s)) return rc;
    }
    std::vector<uint64_t> res{1};
    const uint32_t max_depth = opts ? opts->max_depth : 0;
    const bool odd = p->odd != 0;
    for (;;) {
        if (max_depth && res.size() >= size_t(max_depth) + 1) break;
        uint64_t total = 0;
        for (uint64_t g = 0; g < S; g++) {
            cnt_new[g] = 0;
            if (cnt_cur[g] == 0 && psb::store_length(*recv_s, int(g)) == 0) {  // no state of depth d+1 can be in g
                if (int rc = psb::store_erase(*old_s, int(g))) return rc;
                continue;
            }
            SG_CUDA(cudaMemsetAsync(R.next.p, 0, R.seg_words * 8, R.s));
            if (int rc = R.receive(*recv_s, g, R.next.p)) return rc;
            if (int rc = R.decode(*cur_s, R.cur.p, g, 0)) return rc;
            if (cnt_cur[g])
                if (int rc = R.expand(R.cur.p, g, nullptr)) return rc;
            if (int rc = R.decode(*old_s, R.old.p, g, 1)) return rc;
            SG_CUDA(cudaMemsetAsync(R.scalars.p, 0, 8, R.s));
            psb::seg_finish<<<148 * 8, psb::kThreads, 0, R.s>>>(R.next.p, R.old.p, R.cur.p, R.seg_words, odd ? 1 : 0,
                                                               R.scalars.p);
            SG_CUDA(cudaGetLastError());
            unsigned long long c = 0;
            SG_CUDA(cudaMemcpyAsync(&c, R.scalars.p, 8, cudaMemcpyDeviceToHost, R.s));
            SG_CUDA(cudaStreamSynchronize(R.s));
            // g's depth d-1 layer is no longer needed (DeleteSegment of the old layer)
            if (int rc = psb::store_erase(*old_s, int(g))) return rc;
            total += c;
            cnt_new[g] = c;
            if (int rc = R.encode(R.next.p, g, c, *new_s)) return rc;
            if (c)
                if (int rc = R.expand(R.next.p, g, next_s)) return rc;
            const uint64_t held = store_bytes();
            (R.files ? R.st.peak_disk_bytes : R.st.peak_host_bytes) =
                std::max(R.files ? R.st.peak_disk_bytes : R.st.peak_host_bytes, held);
        }
        if (int rc = R.stage_flush(*next_s)) return rc;
        unsigned long long err[2] = {0, 0};
        SG_CUDA(cudaMemcpyAsync(err, R.scalars.p + 2, 16, cudaMemcpyDeviceToHost, R.s));
        SG_CUDA(cudaStreamSynchronize(R.s));
        if (err[0]) return psb_set_error(PSB_ERR_DEVICE, "segmented search produced a child index >= IndexesCount()");
        if (err[1]) return psb_set_error(PSB_ERR_DEVICE, "segmented search: a layer decoded outside its segment");
        if (total == 0) break;
        if (res.size() >= cap) return psb_set_error(PSB_ERR_CAPACITY, "more depths than counts_cap");
        res.push_back(total);
        // layers: old <- cur <- new (the emptied old store takes the next layer);
        // received children: the next step's
        std::swap(old_s, cur_s);
        std::swap(cur_s, new_s);
        cnt_old.swap(cnt_cur);
        cnt_cur.swap(cnt_new);
        std::swap(recv_s, next_s);
    }
    std::copy(res.begin(), res.end(), counts);
    *n_depths = uint32_t(res.size());
    if (stats && stats->struct_size >= sizeof(psb_segmented_stats)) {
        R.st.struct_size = stats->struct_size;
        R.st.segments = S;
        R.st.device_bytes = (R.next.cap + R.cur.cap + R.old.cap + R.kids.cap) * 8 + R.offs.cap * 4 +
                            R.stream_buf[0].cap + R.stream_buf[1].cap;
        R.st.peak_host_bytes += R.stage.size() * 4;
        R.st.total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        *stats = R.st;
    }
    return PSB_OK;
}
