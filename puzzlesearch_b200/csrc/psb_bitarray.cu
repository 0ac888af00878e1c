// psb_bitarray.cu -- device bit arrays: the reference's BitArray operations
// (Common/BitArray.h:69-169) on device memory, in the same layout (bit i of
// the array is bit i%64 of 64-bit word i/64).  The searches fuse these
// operations into their level and finalize kernels; these entry points expose
// them on their own for callers and for the reference's BitArray test.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>

#include "../../include/psb200.h"
#include "psb_internal.h"

namespace {

constexpr int kT = 256;
constexpr unsigned kGrid = 148 * 8;

uint64_t words_of(uint64_t n_bits) { return (n_bits + 63) / 64; }

// BitArray::Set(first + k*stride) for every such index below n_bits.  One
// thread per word ORs in the word's bits, so no atomics are needed.
__global__ void __launch_bounds__(kT) k_set_stride(uint64_t* __restrict__ w, uint64_t n_words, uint64_t n_bits,
                                                   uint64_t first, uint64_t stride) {
    for (uint64_t i = blockIdx.x * uint64_t(kT) + threadIdx.x; i < n_words; i += uint64_t(gridDim.x) * kT) {
        const uint64_t lo = i * 64, hi = lo + 64 < n_bits ? lo + 64 : n_bits;
        uint64_t k = lo <= first ? first : first + (lo - first + stride - 1) / stride * stride;
        uint64_t m = 0;
        for (; k < hi; k += stride) m |= uint64_t(1) << (k - lo);
        if (m) w[i] |= m;
    }
}

// Sum of the bit positions set in v: bit b of every position contributes 2^b.
__device__ __forceinline__ uint64_t position_sum(uint64_t v) {
    return uint64_t(__popcll(v & 0xAAAAAAAAAAAAAAAAull)) + 2ull * __popcll(v & 0xCCCCCCCCCCCCCCCCull) +
           4ull * __popcll(v & 0xF0F0F0F0F0F0F0F0ull) + 8ull * __popcll(v & 0xFF00FF00FF00FF00ull) +
           16ull * __popcll(v & 0xFFFF0000FFFF0000ull) + 32ull * __popcll(v & 0xFFFFFFFF00000000ull);
}

__device__ __forceinline__ uint64_t warp_sum64(uint64_t x) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xFFFFFFFFu, x, o);
    return x;
}

// BitArray::ScanBits / ScanBitsAndClear / ScanBitsAndClearWithExcl with the
// callback "count the index and add it to a sum" (wrapping mod 2^64, as a
// uint64_t accumulator does).
__global__ void __launch_bounds__(kT) k_scan(uint64_t* __restrict__ w, const uint64_t* __restrict__ excl,
                                             uint64_t n_words, int clear, unsigned long long* out) {
    uint64_t cnt = 0, sum = 0;
    for (uint64_t i = blockIdx.x * uint64_t(kT) + threadIdx.x; i < n_words; i += uint64_t(gridDim.x) * kT) {
        uint64_t v = w[i];
        if (v == 0) continue;
        if (clear) w[i] = 0;
        if (excl) v &= ~excl[i];
        const uint64_t c = __popcll(v);
        cnt += c;
        sum += i * 64 * c + position_sum(v);
    }
    cnt = warp_sum64(cnt);
    sum = warp_sum64(sum);
    if ((threadIdx.x & 31) == 0) {
        if (cnt) atomicAdd(&out[0], (unsigned long long)cnt);
        if (sum) atomicAdd(&out[1], (unsigned long long)sum);
    }
}

// BitArray::AndNotAndCount (BitArray.h:117-125).
__global__ void __launch_bounds__(kT) k_and_not_count(uint64_t* __restrict__ w, const uint64_t* __restrict__ excl,
                                                      uint64_t n_words, unsigned long long* out) {
    uint64_t cnt = 0;
    for (uint64_t i = blockIdx.x * uint64_t(kT) + threadIdx.x; i < n_words; i += uint64_t(gridDim.x) * kT) {
        const uint64_t v = w[i] & ~excl[i];
        w[i] = v;
        cnt += __popcll(v);
    }
    cnt = warp_sum64(cnt);
    if ((threadIdx.x & 31) == 0 && cnt) atomicAdd(&out[0], (unsigned long long)cnt);
}

// BitArray::Or (BitArray.h:103-107).
__global__ void __launch_bounds__(kT) k_or(uint64_t* __restrict__ w, const uint64_t* __restrict__ other,
                                           uint64_t n_words) {
    for (uint64_t i = blockIdx.x * uint64_t(kT) + threadIdx.x; i < n_words; i += uint64_t(gridDim.x) * kT)
        w[i] |= other[i];
}

unsigned grid_for(uint64_t n_words) {
    const uint64_t g = (n_words + kT - 1) / kT;
    return unsigned(g < kGrid ? (g ? g : 1) : kGrid);
}

int cuda_fail(cudaError_t e, const char* what) {
    char buf[256];
    snprintf(buf, sizeof buf, "%s: %s", what, cudaGetErrorString(e));
    return psb_set_error(e == cudaErrorMemoryAllocation ? PSB_ERR_NOMEM : PSB_ERR_CUDA, buf);
}

// Runs a reduction kernel into a two-counter device scratch and copies the
// counters back (the call returns after the stream has reached them).
template <class Launch>
int reduce_call(cudaStream_t s, uint64_t* h_out, Launch launch) {
    unsigned long long* d = nullptr;
    cudaError_t e = cudaMallocAsync(reinterpret_cast<void**>(&d), 16, s);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMallocAsync");
    unsigned long long h[2] = {0, 0};
    e = cudaMemsetAsync(d, 0, 16, s);
    if (e == cudaSuccess) {
        launch(d);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(h, d, 16, cudaMemcpyDeviceToHost, s);
    const cudaError_t f = cudaFreeAsync(d, s);
    if (e == cudaSuccess) e = f;
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(e, "bit-array reduction");
    h_out[0] = h[0];
    h_out[1] = h[1];
    return PSB_OK;
}

}  // namespace

extern "C" {

int psb_bits_set_stride(uint64_t* d_words, uint64_t n_bits, uint64_t first, uint64_t stride, void* stream) {
    if (!d_words || stride == 0) return psb_set_error(PSB_ERR_ARG, "bad argument");
    if (first >= n_bits) return PSB_OK;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const uint64_t nw = words_of(n_bits);
    k_set_stride<<<grid_for(nw), kT, 0, s>>>(d_words, nw, n_bits, first, stride);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? PSB_OK : cuda_fail(e, "k_set_stride");
}

int psb_bits_scan(uint64_t* d_words, const uint64_t* d_exclude, uint64_t n_bits, int clear, uint64_t* count,
                  uint64_t* index_sum, void* stream) {
    if (!d_words || !count || !index_sum) return psb_set_error(PSB_ERR_ARG, "bad argument");
    const uint64_t nw = words_of(n_bits);
    uint64_t out[2];
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (int rc = reduce_call(s, out, [&](unsigned long long* d) {
            k_scan<<<grid_for(nw), kT, 0, s>>>(d_words, d_exclude, nw, clear, d);
        }))
        return rc;
    *count = out[0];
    *index_sum = out[1];
    return PSB_OK;
}

int psb_bits_and_not_count(uint64_t* d_words, const uint64_t* d_exclude, uint64_t n_bits, uint64_t* count,
                           void* stream) {
    if (!d_words || !d_exclude || !count) return psb_set_error(PSB_ERR_ARG, "bad argument");
    const uint64_t nw = words_of(n_bits);
    uint64_t out[2];
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (int rc = reduce_call(s, out, [&](unsigned long long* d) {
            k_and_not_count<<<grid_for(nw), kT, 0, s>>>(d_words, d_exclude, nw, d);
        }))
        return rc;
    *count = out[0];
    return PSB_OK;
}

int psb_bits_or(uint64_t* d_words, const uint64_t* d_other, uint64_t n_bits, void* stream) {
    if (!d_words || !d_other) return psb_set_error(PSB_ERR_ARG, "bad argument");
    const uint64_t nw = words_of(n_bits);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    k_or<<<grid_for(nw), kT, 0, s>>>(d_words, d_other, nw);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? PSB_OK : cuda_fail(e, "k_or");
}

}  // extern "C"
