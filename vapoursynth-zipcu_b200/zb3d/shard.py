"""Frame sharding across GPUs (one process per GPU, no data-path collective).

BM3D frames are independent given their source window, so a clip splits into
contiguous output ranges; a rank additionally reads the halo source frames its
windows reach (radius r for BM3D, 2r for BM3Dv2 with radius > 0, whose output
frame depends on the stacks of frames n-r..n+r) straight from the host.

A rank filters the sub-clip of its source frames and keeps the outputs of its own
range: inside the sub-clip no window of those outputs reaches past the halo, so
they equal the full clip's outputs (the windows clamp at the sub-clip's ends only
where the full clip's do).
"""
from __future__ import annotations

from typing import Callable, Sequence


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


def run_rank(nframes: int, world: int, rank: int, source: Callable[[int], object],
             filter_clip: Callable[[Sequence], Callable[[int], object]], radius: int = 0,
             v2: bool = False) -> list:
    """This rank's output frames of a clip of `nframes`: source(g) gives source frame g,
    filter_clip(frames) filters a sub-clip of those frames and returns a function from a
    frame index of the sub-clip to its output.  Returns the outputs of output_range in
    order; concatenated over the ranks they are the outputs of the whole clip."""
    a, b = output_range(nframes, world, rank)
    if a == b:
        return []
    sa, sb = source_range(nframes, world, rank, radius, v2)
    out = filter_clip([source(g) for g in range(sa, sb)])
    return [out(n - sa) for n in range(a, b)]
