"""The Python puzzle class for a test spec [kind, a, b] (the oracle's kinds)."""
import puzzlesearch_b200 as psb


def make(spec):
    kind, a, b = spec
    if kind == "sliding":
        return psb.SlidingTilePuzzleSimple(a, b)
    if kind == "sliding_opt":
        return psb.SlidingTilePuzzleOptimized(a, b)
    if kind == "pancake":
        return psb.PancakeSimple(a)
    if kind == "pancake_opt":
        return psb.PancakeOptimized(a, bool(b))
    if kind == "hanoi4_opt":
        return psb.FourPegHanoiOptimized(a, bool(b))
    return psb.FourPegHanoiSimple(a, bool(b))
