"""Full-size workloads on the GPU against the reference's own kernels:
640x480 (sigma 3, block_step 8), the 1080p YUV420 two-pass job (sigma 10,
block_step 4, bm_range 12) and a 1080p VBM3D window (radius 2, sigma 15, moving
scene).  Match lists and outputs must be bitwise equal (extractor_exp = 3), and
the size-independent properties must hold: every list starts from the block
itself or contains it, indices stay inside the frame and the window, and two
runs are bitwise identical."""
import numpy as np
import pytest

import oracle as orc
import ref_configs as rc
import refh
from common import make_src
from gpu_common import run_product
from test_ref_pin import _run_ref

pytestmark = pytest.mark.gpu


def _need(spec):
    if not refh.available() or not refh.has_cubin(spec, True):
        pytest.skip("reference kernels not built")


def _check_lists(spec, lists):
    nby, nbx = lists.shape[:2]
    xs = np.minimum(np.arange(nbx) * spec.block_step, spec.w - 8)
    ys = np.minimum(np.arange(nby) * spec.block_step, spec.h - 8)
    X, Y = np.meshgrid(xs, ys)
    r = spec.radius
    has_self = ((lists[..., 0] == X[..., None]) & (lists[..., 1] == Y[..., None]) & (lists[..., 2] == r)).any(-1)
    assert has_self.all()
    assert (lists[..., 0] >= 0).all() and (lists[..., 0] <= spec.w - 8).all()
    assert (lists[..., 1] >= 0).all() and (lists[..., 1] <= spec.h - 8).all()
    assert (lists[..., 2] >= 0).all() and (lists[..., 2] <= 2 * r).all()


def _compare(spec, src):
    _need(spec)
    res, dst, dump = _run_ref(spec, src)
    outs, lists = run_product(spec, src, runs=2)
    assert np.array_equal(outs[0].view(np.uint32), outs[1].view(np.uint32)), "not deterministic"
    _check_lists(spec, lists)
    mism = np.any(lists != dump, axis=(2, 3))
    assert not mism.any(), f"{int(mism.sum())}/{mism.size} blocks differ"
    ref = dst[:, :, :spec.w] if spec.radius == 0 else res[..., :spec.w]
    assert np.array_equal(outs[0].view(np.uint32), np.ascontiguousarray(ref).view(np.uint32)), \
        f"max |diff| {np.nanmax(np.abs(outs[0] - ref))}"
    return outs[0], lists


def test_640x480_sigma3_against_reference_and_oracle():
    spec = rc.workload_specs()[0]
    src = make_src(spec)
    out, lists = _compare(spec, src)
    cfg = orc.make_cfg(spec.w, spec.h, spec.stride, spec.scaled(), spec.block_step, spec.bm_range,
                       extractor_exp=spec.extractor_exp)
    num, den, m = orc.bm3d_pass(cfg, src)
    assert np.array_equal(lists, m)
    err = np.abs(out[0].astype(np.float64) - num[0, 0] / den[0, 0])
    assert err.mean() < 1e-5 and err.max() < 0.05


@pytest.mark.parametrize("w,h", [(1920, 1080), (960, 540)])
def test_1080p_two_pass_plane_against_reference(w, h):
    basic = rc.RefSpec(w=w, h=h, stride=w, sigma=(10.0,) * 3, block_step=4, bm_range=12)
    final = rc.RefSpec(w=w, h=h, stride=w, sigma=(10.0,) * 3, block_step=4, bm_range=12, final=1)
    src = make_src(basic)
    out_b, _ = _compare(basic, src)
    src2 = np.stack([out_b[0][None, None], src[0, :, :, :, :w]])
    _compare(final, np.ascontiguousarray(src2))


def test_1080p_vbm3d_radius2_window_against_reference():
    spec = rc.workload_specs()[-1]
    assert spec.radius == 2
    src = make_src(spec, motion=True)
    _compare(spec, src)
