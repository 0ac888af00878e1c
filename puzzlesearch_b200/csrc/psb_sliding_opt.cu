// Kernel table for SlidingTilePuzzleOptimized's index
// (Puzzles/SlidingTilePuzzleOptimized.cpp), one instantiation per cell count
// of the boards the reference builds it for (2x2 .. 8x2, 3x3, 4x3, 5x3, 4x4,
// SlidingTilePuzzleOptimized.cpp:293-307); the width is a runtime argument,
// so 2x3 or 3x4 boards run too.
#include "psb_kernels.cuh"

namespace psb {

bool sliding_opt_kernels(int cells, PuzzleKernels* out) {
    switch (cells) {
#define PSB_CASE(N) case N: *out = make_kernels<SlidingOptK<N>>(); return true;
        PSB_CASE(4) PSB_CASE(6) PSB_CASE(8) PSB_CASE(9) PSB_CASE(10) PSB_CASE(12) PSB_CASE(14) PSB_CASE(15)
        PSB_CASE(16)
#undef PSB_CASE
    }
    return false;
}

}  // namespace psb
