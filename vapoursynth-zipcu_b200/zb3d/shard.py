"""Frame sharding across GPUs (one process per GPU, no data-path collective).

BM3D frames are independent given their source window, so a clip splits into
contiguous output ranges; a rank additionally reads the halo source frames its
windows reach (radius r for BM3D, 2r for BM3Dv2 with radius > 0, whose output
frame depends on the stacks of frames n-r..n+r) straight from the host.
"""
from __future__ import annotations


def output_range(nframes: int, world: int, rank: int):
    """[first, last) of the output frames of `rank` (balanced, contiguous)."""
    base, extra = divmod(nframes, world)
    first = rank * base + min(rank, extra)
    return first, first + base + (1 if rank < extra else 0)


def source_range(nframes: int, world: int, rank: int, radius: int = 0, v2: bool = False):
    """[first, last) of the source frames `rank` reads (its outputs plus halo)."""
    a, b = output_range(nframes, world, rank)
    if a == b:
        return a, a
    halo = 2 * radius if (v2 and radius > 0) else radius
    return max(a - halo, 0), min(b + halo, nframes)
