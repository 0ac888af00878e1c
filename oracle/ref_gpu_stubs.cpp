// ref_gpu_stubs.cpp -- host-side stand-ins for the reference's CUDA entry
// points (test infrastructure only; built by oracle/build_ref.sh).
//
// The reference's SlidingTilePuzzleOptimized (Puzzles/SlidingTilePuzzleOptimized.cpp)
// is built into oracle/_ref for its Parse, ToString and IndexesCount, i.e. its
// index mapping.  Its Expand copies parents to a GPU and runs
// kernel_sliding_tile_optimized there (Puzzles/SlidingPuzzleGpu.cu); the
// reference's CUDA sources are not built here, and the tests never call that
// Expand.  Every entry point below throws instead.
#include "Puzzles/PuzzleGpu.h"
#include "Puzzles/SlidingPuzzleGpu.h"

#include <stdexcept>

namespace {
[[noreturn]] void no_gpu() { throw std::runtime_error("the reference's GPU expand is not built into the oracle"); }
}  // namespace

PuzzleGpu::Exec::~Exec() {}
void PuzzleGpu::Expand(std::vector<uint64_t>&, std::vector<int>&, std::vector<uint64_t>&, std::vector<int>&,
                       ExpandHint) { no_gpu(); }
PuzzleGpu::Exec* PuzzleGpu::AquireStream() { no_gpu(); }
void PuzzleGpu::ReleaseStream(Exec*) { no_gpu(); }
void PuzzleGpu::CombineIndexAndOpBits(std::vector<uint64_t>&, std::vector<int>&) { no_gpu(); }
void PuzzleGpu::SplitIndexAndOps(std::vector<uint64_t>&, std::vector<int>&) { no_gpu(); }
void CopyToGpu(const uint64_t*, uint64_t*, size_t, CuStream) { no_gpu(); }
void CopyFromGpu(const uint64_t*, uint64_t*, size_t, CuStream) { no_gpu(); }

template <int width, int height>
void GpuSlidingTilePuzzleOptimizedExpand(uint64_t*, uint64_t*, uint64_t, CuStream) { no_gpu(); }

// The shapes the reference instantiates (SlidingTilePuzzleOptimized.cpp:293-307).
template void GpuSlidingTilePuzzleOptimizedExpand<2, 2>(uint64_t*, uint64_t*, uint64_t, CuStream);
template void GpuSlidingTilePuzzleOptimizedExpand<3, 2>(uint64_t*, uint64_t*, uint64_t, CuStream);
template void GpuSlidingTilePuzzleOptimizedExpand<4, 2>(uint64_t*, uint64_t*, uint64_t, CuStream);
template void GpuSlidingTilePuzzleOptimizedExpand<5, 2>(uint64_t*, uint64_t*, uint64_t, CuStream);
template void GpuSlidingTilePuzzleOptimizedExpand<6, 2>(uint64_t*, uint64_t*, uint64_t, CuStream);
template void GpuSlidingTilePuzzleOptimizedExpand<7, 2>(uint64_t*, uint64_t*, uint64_t, CuStream);
template void GpuSlidingTilePuzzleOptimizedExpand<8, 2>(uint64_t*, uint64_t*, uint64_t, CuStream);
template void GpuSlidingTilePuzzleOptimizedExpand<3, 3>(uint64_t*, uint64_t*, uint64_t, CuStream);
template void GpuSlidingTilePuzzleOptimizedExpand<4, 3>(uint64_t*, uint64_t*, uint64_t, CuStream);
template void GpuSlidingTilePuzzleOptimizedExpand<5, 3>(uint64_t*, uint64_t*, uint64_t, CuStream);
template void GpuSlidingTilePuzzleOptimizedExpand<4, 4>(uint64_t*, uint64_t*, uint64_t, CuStream);
