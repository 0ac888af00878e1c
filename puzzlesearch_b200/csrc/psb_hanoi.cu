// Kernel table for four-peg Towers of Hanoi (Puzzles/FourPegHanoiSimple.cpp);
// the disk count and the symmetry flag are runtime arguments.
#include "psb_kernels.cuh"

namespace psb {

bool hanoi_kernels(PuzzleKernels* out) {
    *out = make_kernels<HanoiK>();
    return true;
}

}  // namespace psb
