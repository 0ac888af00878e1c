// psb_pancake_opt.cu -- kernel instances for PancakeOptimized's index
// (sizes 12..16; below 12 the index is PancakeSimple's and those kernels serve).
#include "psb_kernels.cuh"

namespace psb {

bool pancake_opt_kernels(int n, PuzzleKernels* out) {
    switch (n) {
#define PSB_CASE(N) case N: *out = make_kernels<PancakeOptK<N>>(); return true;
        PSB_CASE(12) PSB_CASE(13) PSB_CASE(14) PSB_CASE(15) PSB_CASE(16)
#undef PSB_CASE
    }
    return false;
}

}  // namespace psb
