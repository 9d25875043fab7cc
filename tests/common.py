"""Shared helpers of the test-suite: seeded inputs laid out like the reference's
device buffers ([clip][plane][t][h][stride], vszipcu src/bm3d.cu:574)."""
from __future__ import annotations

import numpy as np

from zb3d import synth


def make_src(spec, seed_clip: int = 0, frame0: int = 0, motion: bool | None = None) -> np.ndarray:
    """float32 [clips][planes][tw][h][stride].  For final (Wiener) specs clip 0 is a
    lightly-noised 'basic estimate' and clip 1 the noisy clip."""
    tw = 2 * spec.radius + 1
    planes = 3 if spec.chroma else 1
    clips = 2 if spec.final else 1
    motion = spec.radius > 0 if motion is None else motion
    sig = max(spec.sigma[0], 1.0)
    out = np.zeros((clips, planes, tw, spec.h, spec.stride), np.float32)
    for p in range(planes):
        for t in range(tw):
            noisy = synth.noisy_plane(spec.w, spec.h, sig, clip=seed_clip, frame=frame0 + t, plane=p,
                                      motion=motion, stride=spec.stride)
            if spec.final:
                basic = synth.noisy_plane(spec.w, spec.h, sig / 4.0, clip=seed_clip + 50, frame=frame0 + t,
                                          plane=p, motion=motion, stride=spec.stride)
                clean = synth.clean_plane(spec.w, spec.h, seed_clip, frame0 + t, p, motion)
                basic[:, :spec.w] = 0.5 * basic[:, :spec.w] + 0.5 * clean
                out[0, p, t] = basic
                out[1, p, t] = noisy
            else:
                out[0, p, t] = noisy
    return out


def spec_id(s) -> str:
    return (f"{s.w}x{s.h}_bs{s.block_step}_R{s.bm_range}_r{s.radius}_f{s.final}_c{s.chroma}"
            f"_{s.bm_error}_{s.t2d}_E{s.extractor_exp}_m{s.proc_mask}")
