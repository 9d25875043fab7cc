"""Parity of the product kernels (sm_100a) with the reference's own kernels on
the same B200 and with the CPU oracle.

* Match lists: bit-exact against the reference's match dump (src/bm3d.cu:788)
  for every metric.  ssd/norm uses the GPU's approximate square root and
  reciprocal; the product writes the reference's final step (2 - 2 dot / D with
  the subtraction fused into the reciprocal) explicitly, so its distances, lists
  and outputs are the reference's bit for bit as well.
* Output: bitwise identical to the reference's output in deterministic mode
  (extractor_exp >= 3): same transforms, shrinkage and rounding; the product
  sums exactly in int64 fixed point, the reference in float atomics whose sums
  are exact while they stay below 2^24 quanta.  With extractor_exp = 0 the
  reference's float atomics round in arbitrary order, hence MAX_ABS_NONDET.
"""
import numpy as np
import pytest

import oracle as orc
import ref_configs as rc
import refh
from common import make_src, spec_id
from gpu_common import run_product
from test_ref_pin import _run_ref

SPECS = rc.parity_specs()
MAX_ABS = 0.0           # deterministic extractor (extractor_exp >= 3): bitwise
MAX_ABS_NONDET = 2e-5   # extractor_exp = 0: the reference's float atomics round in arbitrary order


def _cmp_out(spec, mine, ref_res, ref_dst):
    planes = 3 if spec.chroma else 1
    tol = MAX_ABS if spec.extractor_exp else MAX_ABS_NONDET
    worst = 0.0
    for p in range(planes):
        if spec.chroma and not (spec.proc_mask >> p) & 1:
            continue
        if spec.radius == 0:
            a = mine[p].astype(np.float64)
            b = ref_dst[p, :, :spec.w].astype(np.float64)
            if spec.chroma and spec.scaled()[p] < 1.1920929e-07:
                assert np.isnan(a).all() and np.isnan(b).all()
                continue
        else:
            a = mine[p].astype(np.float64)
            b = ref_res[p, :, :, :, :spec.w].astype(np.float64)
        d = np.abs(a - b)
        worst = max(worst, float(np.nanmax(d)))
        assert np.isfinite(a).all()
    print(f"{spec_id(spec)}: max|mine-ref| = {worst:.3e}")
    assert worst <= tol


@pytest.mark.gpu
@pytest.mark.parametrize("spec", SPECS, ids=[spec_id(s) for s in SPECS])
def test_product_matches_reference(spec):
    if not refh.available() or not refh.has_cubin(spec, True):
        pytest.skip("reference kernels not built (oracle/build_ref.py)")
    src = make_src(spec)
    res, dst, dump = _run_ref(spec, src)
    (mine,), lists = run_product(spec, src)
    mism = np.any(lists != dump, axis=(2, 3))
    assert not mism.any(), f"{int(mism.sum())}/{mism.size} blocks differ, first at {np.argwhere(mism)[:3].tolist()}"
    _cmp_out(spec, mine, res, dst)


@pytest.mark.gpu
@pytest.mark.parametrize("spec", SPECS[:6], ids=[spec_id(s) for s in SPECS[:6]])
def test_product_matches_oracle(spec):
    src = make_src(spec)
    (mine,), lists = run_product(spec, src)
    cfg = orc.make_cfg(spec.w, spec.h, spec.stride, spec.scaled(), spec.block_step, spec.bm_range, spec.radius,
                       spec.ps_num, spec.ps_range, spec.chroma, spec.final, spec.bm_error, spec.t2d, spec.t1d,
                       extractor_exp=spec.extractor_exp)
    num, den, m = orc.bm3d_pass(cfg, src)
    assert (lists == m).all()
    out = num[0, 0] / den[0, 0]
    err = np.abs(mine[0].astype(np.float64) - out)
    assert err.mean() < 1e-5 and err.max() < 0.05


@pytest.mark.gpu
def test_product_is_deterministic():
    spec = rc.parity_specs()[1]
    src = make_src(spec)
    outs, _ = run_product(spec, src, runs=3)
    for o in outs[1:]:
        assert np.array_equal(o.view(np.uint32), outs[0].view(np.uint32))
