// Kernel table for the sliding-tile puzzle (Puzzles/SlidingTilePuzzleSimple.cpp),
// one instantiation per cell count 2..16; the board width is a runtime argument.
#include "psb_kernels.cuh"

namespace psb {

bool sliding_kernels(int cells, PuzzleKernels* out) {
    switch (cells) {
#define PSB_CASE(N) case N: *out = make_kernels<SlidingK<N>>(); return true;
        PSB_CASE(2) PSB_CASE(3) PSB_CASE(4) PSB_CASE(5) PSB_CASE(6) PSB_CASE(7) PSB_CASE(8) PSB_CASE(9)
        PSB_CASE(10) PSB_CASE(11) PSB_CASE(12) PSB_CASE(13) PSB_CASE(14) PSB_CASE(15) PSB_CASE(16)
#undef PSB_CASE
    }
    return false;
}

}  // namespace psb
