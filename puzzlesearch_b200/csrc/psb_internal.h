// psb_internal.h -- definitions shared by the host-side translation units of
// libpsb200 (not part of the public ABI).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

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
}  // namespace psb
