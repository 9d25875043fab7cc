"""CPU tests of the drop-in boundary: the C ABI loads and exports everything
include/zb3d.h declares, argument validation mirrors the reference's error
strings (vszipcu src/bm3d.zig:990-1256, 1391-1417), and the host-side helpers."""
import ctypes
import os
import re

import numpy as np
import pytest

import zb3d
from zb3d import _native as N

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_library_exports_every_declared_symbol():
    hdr = open(os.path.join(ROOT, "include", "zb3d.h")).read()
    # declarations: a line that starts with a return type, then the function name
    names = set(re.findall(r"^[a-z][a-z0-9_ ]*[ *]+(zb3d_[a-z0-9_]+)\s*\(", hdr, re.M))
    lib = N.lib()
    for n in sorted(names):
        assert hasattr(lib, n), n
    assert names == set(N.EXPORTS), sorted(names ^ set(N.EXPORTS))
    assert zb3d.version().startswith("zb3d")


def _info(w=64, h=48, fam=N.GRAY, st=N.FLOAT, bits=32, ss=(0, 0), frames=4):
    return N.VideoInfo(fam, st, bits, ss[0], ss[1], 1 if fam == N.GRAY else 3, w, h, frames)


def _create(info, v2=0, ref=None, **kw):
    keep = []
    a = zb3d._make_args(ref, keep=keep, **{k: kw.get(k) for k in (
        "sigma", "block_step", "bm_range", "radius", "ps_num", "ps_range", "chroma", "device_id", "num_streams",
        "extractor_exp", "bm_error_s", "transform_2d_s", "transform_1d_s", "zero_init", "fast_fused", "match_form",
        "filter_form")})
    err = N.err_buf()
    h = N.lib().zb3d_create(ctypes.byref(info), ctypes.byref(a), v2, err, len(err))
    if h:
        N.lib().zb3d_free(h)
    return err.value.decode()


class _R:
    def __init__(self, i):
        self.i = i

    def info(self):
        return self.i


CASES = [
    (dict(info=_info(st=N.INTEGER, bits=8)), "BM3D: only constant format 32 bit float input supported."),
    (dict(info=_info(w=0)), "BM3D: only constant format 32 bit float input supported."),
    (dict(ref=_R(_info(fam=N.YUV))), 'BM3D: "ref" must be of the same format as "clip".'),
    (dict(ref=_R(_info(w=32))), 'BM3D: "ref" must be of the same dimensions as "clip".'),
    (dict(ref=_R(_info(frames=9))), 'BM3D: "ref" must be of the same number of frames as "clip".'),
    (dict(sigma=[-1.0]), 'BM3D: "sigma" must be non-negative.'),
    (dict(sigma=[float("nan")]), 'BM3D: "sigma" must be non-negative.'),
    (dict(block_step=[9]), 'BM3D: "block_step" must be in range [1, 8].'),
    (dict(block_step=[4, 0]), 'BM3D: "block_step" must be in range [1, 8].'),
    (dict(bm_range=[0]), 'BM3D: "bm_range" must be positive.'),
    (dict(ps_num=[9]), 'BM3D: "ps_num" must be in range [1, 8].'),
    (dict(ps_range=[0]), 'BM3D: "ps_range" must be positive.'),
    (dict(radius=-1), 'BM3D: "radius" must be non-negative.'),
    (dict(radius=17), 'BM3D: "radius" must be <= 16.'),
    (dict(chroma=1), 'BM3D: clip format must be YUV444 when "chroma" is true.'),
    (dict(chroma=1, info=_info(fam=N.YUV, ss=(1, 1))), 'BM3D: clip format must be YUV444 when "chroma" is true.'),
    (dict(bm_error_s=["ssdx"]), 'BM3D: invalid "bm_error_s".'),
    (dict(transform_2d_s=["dct", "fft"]), 'BM3D: invalid "transform_2d_s".'),
    (dict(transform_1d_s=["bior1.6"]), 'BM3D: invalid "transform_1d_s".'),
    (dict(device_id=-1), "BM3D: invalid device ID."),
    (dict(num_streams=0), "BM3D: num_streams must be 1..32."),
    (dict(num_streams=33), "BM3D: num_streams must be 1..32."),
    (dict(sigma=[0.0]), "BM3D: all planes have sigma < FLT_EPSILON (nothing to process)."),
    (dict(info=_info(w=7)), "BM3D: every processed plane must be at least 8x8."),
    (dict(info=_info(w=30, h=30, fam=N.YUV, ss=(2, 2))), "BM3D: every processed plane must be at least 8x8."),
    # additions with no reference counterpart
    (dict(match_form=2), 'BM3D: "match_form" must be 0 or 1.'),
    (dict(filter_form=2), 'BM3D: "filter_form" must be 0 or 1.'),
    (dict(filter_form=1, transform_2d_s=["haar"]), 'BM3D: "filter_form" 1 needs the DCT in both dimensions.'),
    (dict(filter_form=1, transform_1d_s=["wht"]), 'BM3D: "filter_form" 1 needs the DCT in both dimensions.'),
]


@pytest.mark.parametrize("kw,msg", CASES, ids=[c[1][:40] + str(i) for i, c in enumerate(CASES)])
def test_create_errors_mirror_reference(kw, msg):
    info = kw.pop("info", _info())
    ref = kw.pop("ref", None)
    assert _create(info, 0, ref=ref, **kw) == msg


def test_case_insensitive_strings_and_fallback_pass_validation():
    # valid arguments get as far as device selection (no GPU here, or a GPU: no error text)
    msg = _create(_info(fam=N.YUV, ss=(1, 1)), 0, sigma=[3.0, 2.0], bm_error_s=["SSD/Norm", "zSAD"],
                  transform_2d_s=["BIOR1.5"], transform_1d_s=["Haar", "WHT"], block_step=[4, 8], radius=2)
    assert msg in ("", "BM3D: invalid device ID.")


def test_vaggregate_create_errors():
    lib = N.lib()

    def make(clip, src, planes):
        arr = (ctypes.c_int * max(len(planes), 1))(*planes)
        err = N.err_buf()
        h = lib.zb3d_vaggregate_create(ctypes.byref(clip), ctypes.byref(src), arr, len(planes), err, len(err))
        if h:
            lib.zb3d_vaggregate_free(h)
        return err.value.decode(), bool(h)

    src = _info(h=48)
    assert make(_info(h=48 * 6), _info(st=N.INTEGER, bits=16), [0])[0] == 'VAggregate: "src" must be 32 bit float.'
    assert make(_info(h=48 * 6, frames=3), src, [0])[0] == \
        'VAggregate: "clip" must have the same format and frame count as "src".'
    assert make(_info(h=48 * 4), src, [0])[0] == \
        'VAggregate: "clip" is not a BM3D stacked clip of "src" (radius >= 1).'
    assert make(_info(h=48 * 7), src, [0])[0] == \
        'VAggregate: "clip" is not a BM3D stacked clip of "src" (radius >= 1).'
    assert make(_info(h=48 * (4 * 17 + 2)), src, [0])[0] == "VAggregate: radius too large."
    assert make(_info(h=48 * 6), src, [3])[0] == 'VAggregate: "planes" must be 0..2.'
    assert make(_info(h=48 * 6), src, [])[0] == 'VAggregate: "planes" is required.'
    assert make(_info(h=48 * 10), src, [0]) == ("", True)


def test_agg_z_matches_oracle():
    import oracle as orc
    lib = N.lib()
    for r in range(0, 4):
        for nf in (1, 2, 5, 9):
            for n in range(nf):
                for i in range(2 * r + 1):
                    assert lib.zb3d_agg_z(i, n, nf, r) == orc.agg_z(i, n, nf, r)


def test_bm3dv2_passes_through_when_nothing_is_processed():
    frames = [[np.random.default_rng(i).random((16, 24), dtype=np.float32)] for i in range(2)]
    clip = zb3d.Clip.from_frames(frames)
    assert zb3d.BM3Dv2(clip, sigma=0.0) is clip
    assert zb3d.BM3Dv2(clip, sigma=[1e-9]) is clip


def test_bm3d_raises_vs_error_text():
    frames = [[np.zeros((16, 24), np.float32)]]
    clip = zb3d.Clip.from_frames(frames)
    with pytest.raises(zb3d.Error, match=r'"block_step" must be in range \[1, 8\]'):
        zb3d.BM3D(clip, block_step=0)
    with pytest.raises(zb3d.Error, match="must be YUV444"):
        zb3d.BM3D(clip, chroma=1)


def test_processed_planes_rule():
    assert zb3d._processed_planes(None, 3) == [True, True, True]
    assert zb3d._processed_planes([3.0, 0.0], 3) == [True, False, False]
    assert zb3d._processed_planes([0.0, 2.0], 3) == [False, True, True]


def test_pilot_abi_argument_checks_need_no_gpu():
    """The learned pilot's C entry points validate their arguments before any CUDA call."""
    lib = N.lib()
    # CTA cap of the tensor-core convolution: 1..4
    for bad in (0, 5, -1):
        assert lib.zb3d_pilot_tc_ctas_per_sm(bad) == -1
    for ok in (1, 2, 3, 4):
        assert lib.zb3d_pilot_tc_ctas_per_sm(ok) == 0
    fake = 0x10000  # 16-byte aligned, never dereferenced: every call below fails its checks first
    h, w = 32, 48
    # image strides shorter than an image are refused
    assert lib.zb3d_pilot_pack_input_blocked(fake, h * w - 1, fake, 2, h, w, 4.0, fake, None) == -1
    assert lib.zb3d_pilot_conv3x3_tc(fake, 2, h, w, 32, fake, None, 16, 0, None, fake, fake, h * w - 1, 0, None,
                                     None) == -1
    assert lib.zb3d_pilot_conv3x3_tc(fake, 2, h, w, 32, fake, None, 16, 0, None, fake, fake, 0, h * w - 1, None,
                                     None) == -1
    # misaligned operands and unsupported layer shapes are refused
    assert lib.zb3d_pilot_conv3x3_tc(fake + 4, 1, h, w, 32, fake, None, 32, 1, fake, None, None, 0, 0, None,
                                     None) == -1
    assert lib.zb3d_pilot_conv3x3_tc(fake, 1, h, w, 24, fake, None, 32, 1, fake, None, None, 0, 0, None, None) == -1
    assert lib.zb3d_pilot_conv3x3_tc(fake, 1, h, w, 64, fake, None, 64, 1, fake, None, None, 0, 0, None, None) == -1
    # empty batches are a no-op
    assert lib.zb3d_pilot_pack_input_blocked(fake, 0, fake, 0, h, w, 4.0, fake, None) == 0
    assert lib.zb3d_pilot_conv3x3_tc(fake, 0, h, w, 32, fake, None, 32, 1, fake, None, None, 0, 0, None, None) == 0


def test_dct2d_tf32_argument_checks_need_no_gpu():
    """The precision-form transform rejects bad arguments before any CUDA call."""
    from zb3d import _native as N
    lib = N.lib()
    assert lib.zb3d_dct2d_tf32(None, None, 0, 1, None, None) == 0    # nothing to do
    assert lib.zb3d_dct2d_tf32(None, None, 5, 1, None, None) == 1    # missing buffers
    assert lib.zb3d_dct2d_tf32(None, None, -1, 1, None, None) == 1   # negative count
    assert lib.zb3d_dct2d_tf32(16, 20, 5, 1, 32, None) == 1          # output not 16-byte aligned


def test_batch_entry_points_check_their_jobs_before_any_cuda_call():
    """zb3d_process_batch refuses an empty job list and jobs without a filter or buffers."""
    lib = N.lib()
    err = N.err_buf()
    assert lib.zb3d_process_batch(None, 0, None, err, len(err)) == -1
    assert "no jobs" in err.value.decode()
    jobs = (N.BatchJob * 2)(N.BatchJob(None, 0x10000, 0x10000), N.BatchJob(None, 0x10000, 0x10000))
    assert lib.zb3d_process_batch_ex(jobs, 2, None, 0, 0, err, len(err)) == -1
    assert "job 0 has no filter" in err.value.decode()
