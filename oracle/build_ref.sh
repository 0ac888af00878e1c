#!/usr/bin/env bash
# Builds the reference's own CPU path (lightln2/PuzzleSearch) from its sources
# into oracle/_ref/ -- test infrastructure only (a checker and the timed CPU
# baseline, never part of the product).
#
# The reference is MSVC C++; the only changes are mechanical, applied to a
# scratch copy under oracle/_ref/src (never committed):
#   * integer literal suffixes 1ui64 / 1ui32 / 1i64 -> ULL / U / LL
#   * std::chrono::high_resolution_clock -> steady_clock (MSVC aliases them)
#   * `*(__m128i*)(p) = v;` -> _mm_storeu_si128 (MSVC emits an unaligned store
#     for it; GCC assumes 16-byte alignment)
#   * `static` dropped from explicit template specializations (MSVC accepts it,
#     GCC does not)
#   * a forward declaration of SlidingTilePuzzleOptimized.cpp's Parity, which
#     MSVC finds at instantiation time and GCC's two-phase lookup does not
#   * a generated <intrin.h> mapping the MSVC intrinsics to GCC builtins, and
#     the AVX-512VL load/store intrinsics to their SSE2 / AVX2 equivalents so
#     the library runs on any x86-64-v3 host.
# SlidingTilePuzzleOptimized is built for its index mapping only: its GPU
# expand entry points are stand-ins that throw (oracle/ref_gpu_stubs.cpp).
# Outputs: oracle/_ref/libpsbref.so (C ABI from oracle/ref_capi.cpp),
#          oracle/_ref/psbref (CLI used for the CPU baseline timing) and
#          oracle/_ref/psbref_mt (multi-threaded level loop over the reference's
#          own expanders, for the large per-depth count fixtures).
set -euo pipefail
# The reference's source tree: the first argument, else $PSB_REFERENCE.
REF="${1:-${PSB_REFERENCE:-}}"
HERE="$(cd "$(dirname "$0")" && pwd)"
OUT="$HERE/_ref"
if [ -z "$REF" ]; then
    echo "usage: build_ref.sh <reference source tree> (or set PSB_REFERENCE); keeping any prebuilt $OUT" >&2
    exit 0
fi
if [ ! -d "$REF/Common" ]; then
    echo "build_ref: reference sources not found at $REF; keeping any prebuilt $OUT" >&2
    exit 0
fi
SRC="$OUT/src"
rm -rf "$SRC"
mkdir -p "$SRC/Common" "$SRC/Puzzles"
COMMON="Util.h Util.cpp Puzzle.h Puzzle.cpp Buffer.h Array.h BitArray.h InMemoryBFS.h
        InMemoryClassicBFS.cpp InMemoryTwoBitBFS.cpp InMemoryThreeBitBFS.cpp InMemoryFrontierSearch.cpp
        StreamVInt.h StreamVInt.cpp FrontierCompression.h FrontierCompression.cpp
        OpBitsCompression.h OpBitsCompression.cpp"
PUZZLES="PermutationMap.h PermutationMap.cpp SlidingTilePuzzleSimple.h SlidingTilePuzzleSimple.cpp
         PancakeSimple.h PancakeSimple.cpp FourPegHanoiSimple.h FourPegHanoiSimple.cpp
         PancakeOptimized.h PancakeOptimized.cpp FourPegHanoiOptimized.h FourPegHanoiOptimized.cpp
         PuzzleGpu.h GPU.h SlidingPuzzleGpu.h SlidingTilePuzzleOptimized.h SlidingTilePuzzleOptimized.cpp"
for f in $COMMON; do cp "$REF/Common/$f" "$SRC/Common/$f"; done
for f in $PUZZLES; do cp "$REF/Puzzles/$f" "$SRC/Puzzles/$f"; done
find "$SRC" -type f \( -name '*.h' -o -name '*.cpp' \) -print0 | xargs -0 sed -E -i \
    -e 's/([0-9A-Fa-fx])ui64/\1ULL/g' \
    -e 's/([0-9A-Fa-f])ui32/\1U/g' \
    -e 's/([0-9])i64/\1LL/g' \
    -e 's/high_resolution_clock/steady_clock/g' \
    -e 's/^__forceinline static int (_(En|De)codeTuple<[0-9]>)/__forceinline int \1/' \
    -e 's/\*\(__m128i\*\)\(([^)]*)\) = ([a-z_]+);/_mm_storeu_si128((__m128i*)(\1), \2);/g'
# MSVC resolves SlidingTilePuzzleOptimized's Parity at instantiation time;
# GCC's two-phase lookup needs it declared before ParseState uses it.
sed -i -e 's/^\(\s*\)constexpr int BLANK_POS = 15;/&\n\1template<int width, int height> bool Parity(struct VPuzzleState state);/' \
    "$SRC/Puzzles/SlidingTilePuzzleOptimized.cpp"

cat > "$SRC/intrin.h" <<'EOF'
/* Generated by oracle/build_ref.sh: the MSVC intrinsics live in msvc_compat.h. */
#pragma once
#include "msvc_compat.h"
EOF
cat > "$SRC/msvc_compat.h" <<'EOF'
/* Generated by oracle/build_ref.sh: force-included into every reference file. */
#pragma once
#include <algorithm>
#include <atomic>
#include <cstring>
#include <limits>
#include <memory>
#include <sstream>
#include <utility>
#include <immintrin.h>
#define _mm_loadu_epi8(p) _mm_loadu_si128((const __m128i*)(p))
#define _mm_loadu_epi32(p) _mm_loadu_si128((const __m128i*)(p))
#define _mm_storeu_epi8(p, v) _mm_storeu_si128((__m128i*)(p), (v))
#define _mm256_storeu_epi64(p, v) _mm256_storeu_si256((__m256i*)(p), (v))
#define __forceinline inline __attribute__((always_inline))
static inline unsigned long long __popcnt64(unsigned long long v) { return __builtin_popcountll(v); }
static inline unsigned int __popcnt(unsigned int v) { return __builtin_popcount(v); }
static inline unsigned char _BitScanForward64(unsigned long* idx, unsigned long long v) {
    if (!v) return 0; *idx = (unsigned long)__builtin_ctzll(v); return 1; }
static inline unsigned char _BitScanReverse64(unsigned long* idx, unsigned long long v) {
    if (!v) return 0; *idx = 63ul - (unsigned long)__builtin_clzll(v); return 1; }
EOF

CXX="${PSB_CXX:-/usr/bin/g++}"  # the system compiler: a CXX wrapper that links libstdc++ statically breaks loading next to numpy
# SlidingTilePuzzleOptimized's headers name CUDA runtime types (declarations
# only: its GPU entry points are stand-ins, oracle/ref_gpu_stubs.cpp).
CUDA_INC="${CUDA_HOME:-/usr/local/cuda}/include"
FLAGS="-std=c++20 -O3 -march=x86-64-v3 -fPIC -w -I$SRC -I$SRC/Common -I$CUDA_INC -include $SRC/msvc_compat.h"
SOURCES=""
for f in $COMMON $PUZZLES; do case "$f" in *.cpp)
    d=Common; [ -f "$SRC/Puzzles/$f" ] && d=Puzzles; SOURCES="$SOURCES $SRC/$d/$f";; esac; done
SOURCES="$SOURCES $HERE/ref_gpu_stubs.cpp"
$CXX $FLAGS -shared -o "$OUT/libpsbref.so" "$HERE/ref_capi.cpp" $SOURCES
$CXX $FLAGS -o "$OUT/psbref" "$HERE/ref_main.cpp" "$HERE/ref_capi.cpp" $SOURCES
$CXX $FLAGS -pthread -o "$OUT/psbref_mt" "$HERE/ref_mt_bfs.cpp" $SOURCES
echo "build_ref: built $OUT/libpsbref.so, $OUT/psbref and $OUT/psbref_mt"
