"""The precision form of the collaborative filter (zb3d_args.filter_form = 1): the 2D DCT
of every group's patches on the tensor cores in split TF32 (csrc/zb3d_filter_tc.cu).

It is not bitwise. Its outputs are compared with the FP64 oracle (oracle/bm3d_oracle.c,
the reference's algorithm in double) and with the plain FP32 form, on the hard-threshold
and Wiener steps, radius 0, 1 and 2, and CBM3D. Both forms share the match lists.

The bounds, relative to the data range of about 1:
* radius 0, against the oracle: mean |error| < 2e-6 (measured 0.1-5.5e-7, the plain form
  0.1-4e-7) and max < 0.05, the plain form's own bound (tests/test_parity_gpu.py): a pixel
  can move by up to about 1e-2 where a coefficient sits within rounding of the hard
  threshold (measured max here 4.4e-5).
* stacked accumulators (radius > 0) and CBM3D against the plain form: mean relative
  difference < 1e-5 (measured 1.4e-7 to 9.5e-7).
"""
import numpy as np
import pytest

import oracle as orc
import ref_configs as rc
from common import make_src, spec_id
from gpu_common import run_product

pytestmark = pytest.mark.gpu

SPECS = [s for s in rc.parity_specs() if s.t2d == "dct" and s.t1d == "dct" and s.extractor_exp and
         s.bm_error == "ssd" and s.block_step in (4, 8)]
SPATIAL = [s for s in SPECS if s.radius == 0 and not s.chroma]
OTHER = [s for s in SPECS if s.radius > 0 or s.chroma]


@pytest.mark.parametrize("spec", SPATIAL, ids=[spec_id(s) for s in SPATIAL])
def test_precision_form_against_fp64_oracle(spec):
    src = make_src(spec)
    (plain,), lists = run_product(spec, src)
    (prec,), lists2 = run_product(spec, src, filter_form=1)
    assert (lists == lists2).all()
    cfg = orc.make_cfg(spec.w, spec.h, spec.stride, spec.scaled(), spec.block_step, spec.bm_range, spec.radius,
                       spec.ps_num, spec.ps_range, spec.chroma, spec.final, spec.bm_error, spec.t2d, spec.t1d,
                       extractor_exp=spec.extractor_exp)
    num, den, _ = orc.bm3d_pass(cfg, src)
    ref = num[0, 0] / den[0, 0]
    e_prec = np.abs(prec[0].astype(np.float64) - ref)
    e_plain = np.abs(plain[0].astype(np.float64) - ref)
    d = np.abs(prec[0].astype(np.float64) - plain[0])
    print(f"{spec_id(spec)}: vs FP64 precision mean {e_prec.mean():.2e} max {e_prec.max():.2e}, plain mean "
          f"{e_plain.mean():.2e} max {e_plain.max():.2e}; precision vs plain max {d.max():.2e}")
    assert np.isfinite(prec).all()
    assert e_prec.mean() < 2e-6 and e_prec.max() < 0.05


@pytest.mark.parametrize("spec", OTHER, ids=[spec_id(s) for s in OTHER])
def test_precision_form_against_plain_form(spec):
    src = make_src(spec)
    (plain,), _ = run_product(spec, src)
    (prec,), _ = run_product(spec, src, filter_form=1)
    planes = [p for p in range(prec.shape[0]) if not spec.chroma or (spec.proc_mask >> p) & 1]
    a = prec[planes].astype(np.float64)
    b = plain[planes].astype(np.float64)
    ok = np.isfinite(b)
    rel = np.abs(a - b)[ok].mean() / max(np.abs(b[ok]).mean(), 1e-30)
    print(f"{spec_id(spec)}: precision vs plain mean relative {rel:.2e}, max abs {np.abs(a - b)[ok].max():.2e}")
    assert np.isfinite(a[ok]).all() and rel < 1e-5


def test_precision_form_through_the_api_rejects_other_transforms():
    import zb3d
    from zb3d import synth
    clip = zb3d.Clip.from_frames([[synth.noisy_plane(64, 48, 10.0)]])
    with pytest.raises(zb3d.Error, match="filter_form"):
        zb3d.BM3D(clip, sigma=10.0, transform_2d_s="haar", filter_form=1)
    out = np.asarray(zb3d.BM3D(clip, sigma=10.0, block_step=4, bm_range=8, filter_form=1).get_frame(0)[0])
    assert np.isfinite(out).all()
