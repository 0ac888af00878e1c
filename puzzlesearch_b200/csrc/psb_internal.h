// psb_internal.h -- definitions shared by the host-side translation units of
// libpsb200 (not part of the public ABI).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#include "psb_kernels.cuh"

struct psb_puzzle {
    int kind, a, b;
    int cells;  // permutation size (sliding, pancake)
    uint64_t n_states;
    int ops, branching, odd;
    psb::PuzzleKernels k;
    psb::PuzzleArgs pz;
};

// Records the calling thread's last error for psb_last_error(); returns code.
int psb_set_error(int code, const char* msg);

namespace psb {
// Level-end kernels, defined in psb_host.cu.
__global__ void finalize_three_bit(const ulonglong2* __restrict__ cur, ulonglong2* __restrict__ nw,
                                   ulonglong2* __restrict__ old, uint64_t n2, int odd, int zero_old,
                                   unsigned long long* count);
__global__ void finalize_classic(ulonglong2* __restrict__ nw, ulonglong2* __restrict__ closed, uint64_t n2,
                                 unsigned long long* count);
// Variants used by searches that may run bottom-up levels.
__global__ void finalize_three_bit_visited(const ulonglong2* __restrict__ cur, ulonglong2* __restrict__ nw,
                                           ulonglong2* __restrict__ old, ulonglong2* __restrict__ visited,
                                           uint64_t n2, int odd, int zero_old, unsigned long long* count);
__global__ void finalize_classic_clear(ulonglong2* __restrict__ nw, ulonglong2* __restrict__ closed,
                                       ulonglong2* __restrict__ open, uint64_t n2, unsigned long long* count);
__global__ void finalize_three_bit_flagged(const ulonglong2* __restrict__ cur, ulonglong2* __restrict__ nw,
                                           ulonglong2* __restrict__ old, ulonglong2* __restrict__ visited,
                                           uint64_t n2, const uint8_t* __restrict__ new_flags,
                                           const uint8_t* __restrict__ old_flags, uint64_t n_windows,
                                           uint32_t per_window, int odd, unsigned long long* count);
__global__ void retire_two_bit(ulonglong2* __restrict__ codes, uint64_t n2, uint32_t cur_code,
                               unsigned long long* count);

// Frontier encoder with device scratch kept between segments (psb_codec.cu).
struct SegmentEncoder;
SegmentEncoder* encoder_create();
void encoder_destroy(SegmentEncoder* e);
// Plans the reference's segment stream of the set bits of d_bits[0, n_bits)
// (n_bits <= 2^32): *count offsets in *bytes bytes; encoder_write then
// writes it to d_out (device, >= *bytes).  d_bits must stay unchanged
// until the write has run (both are ordered on stream s).  sums_ready: the
// chunk popcounts are already in encoder_chunk_sums' buffer.
int encoder_plan(SegmentEncoder* e, const uint64_t* d_bits, uint64_t n_bits, cudaStream_t s, bool sums_ready,
                 uint64_t* bytes, uint64_t* count);
int encoder_write(SegmentEncoder* e, uint8_t* d_out, cudaStream_t s);
// Frontier-search segments carry each state's operator bits: with `on`, the
// following plans write CompressedFrontierWriter's stream (StreamVInt blocks
// with bounds, Common/CompressedFrontier.cpp:63-70) whose nibble for offset v
// is state first_state + v of `nibbles` (a 4-bit array; NULL = all zero).
void encoder_set_ops(SegmentEncoder* e, bool on, const uint64_t* nibbles, uint64_t first_state);
// The encoder's chunk-sum buffer sized for an n_bits segment.
int encoder_chunk_sums(SegmentEncoder* e, uint64_t n_bits, unsigned long long** sums);
// Kernels the encoder launched since the last call.
uint64_t encoder_take_launches(SegmentEncoder* e);
// Segment store (psb_store.cu): the reference's Store over files in some
// directories, or over host memory when there are none.
class StoreImpl;
void store_destroy(StoreImpl* s);
struct StoreDeleter { void operator()(StoreImpl* s) const { store_destroy(s); } };
using StorePtr = std::unique_ptr<StoreImpl, StoreDeleter>;
int store_create(int max_segments, const std::string& name, const std::vector<std::string>& directories,
                 int files_per_path, StorePtr* out);
uint64_t store_length(const StoreImpl& s, int segment);
uint64_t store_total(const StoreImpl& s);
void store_rewind(StoreImpl& s, int segment);
int store_write(StoreImpl& s, int segment, const void* buf, uint64_t size);
int store_read(StoreImpl& s, int segment, void* buf, uint64_t cap, uint64_t* got);
int store_erase(StoreImpl& s, int segment);
int store_erase_all(StoreImpl& s);

// Decodes a segment stream (block table on the host, `h_blocks`, and on the
// device, `d_blocks`) into the cleared bitmap d_bits[0, n_bits) on stream s,
// without synchronising; an offset outside the segment sets *d_err.  The
// StreamVInt blocks are decoded in parallel chunks; `h_in`, the stream in
// host memory if the caller has it (else NULL), lets the host find the
// chunks.  The scratch grows on demand and is kept for the next call.
struct DecodeScratch;
DecodeScratch* decoder_create();
void decoder_destroy(DecodeScratch* d);
int frontier_decode_async(const uint8_t* d_in, const uint8_t* h_in, const psb_codec_block* h_blocks,
                          const psb_codec_block* d_blocks, uint32_t n_blocks, uint64_t* d_bits, uint64_t n_bits,
                          unsigned long long* d_err, DecodeScratch* scratch, cudaStream_t s);
// One-bit frontier bitmaps (ceil(n_states/64) words at out; first_state a
// multiple of 64) of a two-bit array (states with code `code`) and of a
// frontier-search array (states with an operator bit set, less `excl`),
// with their chunk popcounts in `sums` (from encoder_chunk_sums).  Two-bit
// extraction may be given the depth's active-window flags (NULL = none):
// chunks of unflagged windows count 0 and are not written.
int frontier_bits_two_bit(const uint64_t* codes, uint64_t first_state, uint64_t n_states, uint32_t code,
                          uint64_t* out, unsigned long long* sums, const uint8_t* flags, int window_bits,
                          uint64_t n_windows, cudaStream_t s);
int frontier_bits_nibbles(const uint64_t* nibbles, const uint64_t* excl, uint64_t first_state, uint64_t n_states,
                          uint64_t* out, unsigned long long* sums, cudaStream_t s);
}  // namespace psb
