"""Generate the golden fixtures of the BM3D path from the reference itself.

Runs the reference's own kernels (vszipcu src/bm3d.cu, built into oracle/_ref by
oracle/build_ref.py and launched as src/bm3d.zig:375-401 does) on a GPU for a few
small seeded windows and stores, per case, the input window, the reference's
match lists (dump variant, taken after self inclusion, src/bm3d.cu:788) and its
output: the denoised planes (radius 0) or the stacked accumulators (radius > 0).

    python tests/golden/make_golden.py      (needs a CUDA GPU and oracle/_ref)

The CPU test-suite (tests/test_oracle_golden.py) checks the oracle against these
files, so the oracle stays pinned to the reference without a GPU.
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [os.path.join(ROOT, "vapoursynth-zipcu_b200"), os.path.join(ROOT, "oracle"),
                os.path.join(ROOT, "tests")]

import ref_configs as rc  # noqa: E402
from common import make_src  # noqa: E402


def golden_specs():
    s = rc.RefSpec
    return {
        "basic_bs8": s(w=72, h=56, stride=80, sigma=(10.0,) * 3),
        "basic_bs4": s(w=77, h=53, stride=80, sigma=(10.0,) * 3, block_step=4, bm_range=12),
        "final_bs4": s(w=77, h=53, stride=80, sigma=(10.0,) * 3, block_step=4, bm_range=12, final=1),
        "basic_bs3_small": s(w=45, h=37, stride=48, sigma=(3.0,) * 3, block_step=3, bm_range=5),
        "tiny_8x8": s(w=8, h=8, stride=16, sigma=(3.0,) * 3),
        "sad": s(w=72, h=56, stride=80, sigma=(3.0,) * 3, bm_error="sad"),
        "zssd": s(w=72, h=56, stride=80, sigma=(3.0,) * 3, bm_error="zssd"),
        "haar": s(w=72, h=56, stride=80, sigma=(3.0,) * 3, t2d="haar", t1d="haar"),
        "temporal_r1": s(w=64, h=48, stride=64, sigma=(15.0,) * 3, radius=1),
        "temporal_r2_final": s(w=64, h=48, stride=64, sigma=(15.0,) * 3, radius=2, final=1),
        "cbm3d": s(w=48, h=40, stride=48, sigma=(8.0, 6.0, 6.0), chroma=1, proc_mask=7),
    }


def main():
    import torch
    import refh
    from test_ref_pin import _run_ref
    assert torch.cuda.is_available(), "needs a GPU"
    names = golden_specs()
    for name, spec in names.items():
        src = make_src(spec)
        res, dst, dump = _run_ref(spec, src)
        out = dst if spec.radius == 0 else res
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), src=src, out=out, matches=dump,
                            spec=json.dumps(rc.spec_dict(spec)))
        print("wrote", name)


if __name__ == "__main__":
    main()
