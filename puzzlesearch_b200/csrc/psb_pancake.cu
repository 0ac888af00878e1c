// Kernel table for the pancake puzzle (Puzzles/PancakeSimple.cpp), one
// instantiation per size: sizes 2..16 (PancakeSimple.cpp:26).
#include "psb_kernels.cuh"

namespace psb {

bool pancake_kernels(int n, PuzzleKernels* out) {
    switch (n) {
#define PSB_CASE(N) case N: *out = make_kernels<PancakeK<N>>(); return true;
        PSB_CASE(2) PSB_CASE(3) PSB_CASE(4) PSB_CASE(5) PSB_CASE(6) PSB_CASE(7) PSB_CASE(8) PSB_CASE(9)
        PSB_CASE(10) PSB_CASE(11) PSB_CASE(12) PSB_CASE(13) PSB_CASE(14) PSB_CASE(15) PSB_CASE(16)
#undef PSB_CASE
    }
    return false;
}

}  // namespace psb
