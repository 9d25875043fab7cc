"""The public API (zb3d.BM3D / BM3Dv2 / VAggregate on host frames, through the
C ABI's get_frame) against the reference's own kernels on the same GPU.

* two-pass BM3Dv2 on YUV420 equals, plane by plane, the reference kernel run
  as basic then final pass (bitwise, deterministic mode);
* BM3D with radius > 0 emits the reference's stacked accumulators for the
  clamped window of every frame (src/bm3d.zig:684-699), bitwise;
* BM3Dv2 radius > 0 equals the reference's vaggregate over those stacks, and
  the fused and composed forms are byte-identical (vszipcu README.md:77-79);
* CBM3D (YUV444, chroma=1); concurrent get_frame calls; frame-range errors.
"""
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

import oracle as orc  # noqa: F401  (keeps the oracle importable in this module's process)
import ref_configs as rc
import refh
import zb3d
from zb3d import _native as N
from zb3d import synth

pytestmark = pytest.mark.gpu


def _ref_window(spec, src_np, dump=False):
    from test_ref_pin import _run_ref
    return _run_ref(spec, src_np, dump=dump)


def _need(spec):
    if not refh.available() or not refh.has_cubin(spec):
        pytest.skip("reference kernels not built")


def _gray_clip(w, h, n, sigma, motion=False):
    return zb3d.Clip.from_frames([[synth.noisy_plane(w, h, sigma, frame=f, motion=motion)[:, :w]] for f in range(n)])


def test_host_path_equals_device_path():
    from gpu_common import run_product
    from common import make_src
    spec = rc.parity_specs()[1]
    src = make_src(spec)
    (dev,), _ = run_product(spec, src)
    clip = zb3d.Clip.from_frames([[src[0, 0, 0, :, :spec.w]]])
    out = zb3d.BM3D(clip, sigma=10.0, block_step=4, bm_range=12, extractor_exp=3).get_frame(0)[0]
    assert np.array_equal(out, dev[0])


def test_two_pass_yuv420_equals_reference_kernels():
    w, h, sigma = 96, 64, 10.0
    frames = [[synth.noisy_plane(w >> (p > 0), h >> (p > 0), sigma, frame=f, plane=p)[:, :w >> (p > 0)]
               for p in range(3)] for f in range(2)]
    clip = zb3d.Clip.from_frames(frames, family=N.YUV, subsampling=(1, 1))
    kw = dict(sigma=[sigma] * 3, block_step=4, bm_range=12, extractor_exp=3)
    basic = zb3d.BM3Dv2(clip, **kw)
    final = zb3d.BM3Dv2(clip, ref=basic, **kw)
    for n in range(2):
        got_b, got_f = basic.get_frame(n), final.get_frame(n)
        for p in range(3):
            pw, ph = w >> (p > 0), h >> (p > 0)
            sb = rc.RefSpec(w=pw, h=ph, stride=pw, sigma=(sigma,) * 3, block_step=4, bm_range=12)
            sf = rc.RefSpec(w=pw, h=ph, stride=pw, sigma=(sigma,) * 3, block_step=4, bm_range=12, final=1)
            _need(sb)
            _need(sf)
            noisy = frames[n][p]
            _, rb, _ = _ref_window(sb, noisy[None, None, None])
            assert np.array_equal(rb[0], got_b[p]), (n, p)
            _, rf, _ = _ref_window(sf, np.stack([got_b[p], noisy])[:, None, None])
            assert np.array_equal(rf[0], got_f[p]), (n, p)


@pytest.mark.parametrize("final", [0, 1])
def test_temporal_stacks_vaggregate_and_fused(final):
    import torch
    w, h, r, nf, sigma = 64, 48, 1, 5, 15.0
    clip = _gray_clip(w, h, nf, sigma, motion=True)
    ref = _gray_clip(w, h, nf, sigma / 4, motion=True) if final else None
    kw = dict(sigma=sigma, radius=r, extractor_exp=3)
    spec = rc.RefSpec(w=w, h=h, stride=w, sigma=(sigma,) * 3, radius=r, final=final)
    _need(spec)
    stacked = zb3d.BM3D(clip, ref=ref, **kw)
    assert stacked.height == h * 2 * (2 * r + 1)
    # sigma falls back plane to plane, so all three planes count as processed (src/bm3d.zig:1013-1017)
    assert stacked.get_props(0) == {"BM3D_V_radius": r, "BM3D_V_process": [1, 1, 1]}
    ref_stacks = {}
    for n in range(nf):
        idx = [min(max(n - r + t, 0), nf - 1) for t in range(2 * r + 1)]
        win = np.stack([clip.get_frame(i)[0] for i in idx])[None, None]
        if final:
            win = np.concatenate([np.stack([ref.get_frame(i)[0] for i in idx])[None, None], win])
        res, _, _ = _ref_window(spec, win)
        ref_stacks[n] = res[0]
        got = stacked.get_frame(n)[0].reshape(2 * r + 1, 2, h, w)
        assert np.array_equal(got, res[0]), n
    composed = zb3d.BM3Dv2(clip, ref=ref, **kw)
    fused = zb3d.BM3Dv2(clip, ref=ref, fast_fused=1, **kw)
    vagg = refh.RefVagg(w, h, w, r, 1)
    for n in range(nf):
        a, b = composed.get_frame(n)[0], fused.get_frame(n)[0]
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), n
        stacks = [torch.from_numpy(ref_stacks[min(max(n - r + i, 0), nf - 1)]).cuda() for i in range(2 * r + 1)]
        zs = [orc.agg_z(i, n, nf, r) for i in range(2 * r + 1)]
        dst = torch.zeros((h, w), dtype=torch.float32, device="cuda")
        vagg.run(dst.data_ptr(), [s.data_ptr() for s in stacks], zs, 1)
        torch.cuda.synchronize()
        assert np.array_equal(dst.cpu().numpy(), a), n
    vagg.close()


def test_cbm3d_yuv444_equals_reference():
    w, h, sig = 48, 40, (8.0, 6.0, 6.0)
    frames = [[synth.noisy_plane(w, h, 8.0, frame=0, plane=p)[:, :w] for p in range(3)]]
    clip = zb3d.Clip.from_frames(frames, family=N.YUV)
    out = zb3d.BM3D(clip, sigma=list(sig), chroma=1, extractor_exp=3).get_frame(0)
    spec = rc.RefSpec(w=w, h=h, stride=w, sigma=sig, chroma=1, proc_mask=7)
    _need(spec)
    _, dst, _ = _ref_window(spec, np.stack(frames[0])[None, :, None])
    for p in range(3):
        assert np.array_equal(out[p], dst[p]), p


def test_concurrent_get_frame_matches_serial():
    clip = _gray_clip(80, 64, 8, 10.0)
    f = zb3d.BM3D(clip, sigma=10.0, block_step=4, num_streams=4, extractor_exp=3)
    serial = [f.get_frame(n)[0].copy() for n in range(8)]
    g = zb3d.BM3D(clip, sigma=10.0, block_step=4, num_streams=4, extractor_exp=3)
    with ThreadPoolExecutor(6) as ex:
        par = list(ex.map(lambda n: g.get_frame(n)[0], range(8)))
    for a, b in zip(serial, par):
        assert np.array_equal(a, b)


def test_unprocessed_planes_are_copied_and_errors_raise():
    w, h = 64, 48
    frames = [[synth.noisy_plane(w >> (p > 0), h >> (p > 0), 5.0, frame=0, plane=p)[:, :w >> (p > 0)]
               for p in range(3)]]
    clip = zb3d.Clip.from_frames(frames, family=N.YUV, subsampling=(1, 1))
    out = zb3d.BM3Dv2(clip, sigma=[5.0, 0.0]).get_frame(0)
    assert not np.array_equal(out[0], frames[0][0])
    assert np.array_equal(out[1], frames[0][1]) and np.array_equal(out[2], frames[0][2])
    with pytest.raises(zb3d.Error):
        zb3d.BM3Dv2(clip, sigma=5.0).get_frame(3)


def test_pinned_and_pageable_frames_take_the_same_path_to_the_same_bytes():
    """Page-locked caller frames are DMA'd directly (zb3d_get_frame's direct path),
    pageable ones go through the slot's staging buffer: both give the same bytes,
    for inputs (clip and ref) and outputs."""
    import ctypes
    w, h, sigma = 200, 120, 10.0
    frames = [[synth.noisy_plane(w >> (p > 0), h >> (p > 0), sigma, frame=f, plane=p)[:, :w >> (p > 0)]
               for p in range(3)] for f in range(2)]
    kw = dict(sigma=[sigma] * 3, block_step=4, bm_range=12, extractor_exp=3)
    outs = []
    for pinned in (False, True):
        clip = zb3d.Clip.from_frames(frames, family=N.YUV, subsampling=(1, 1), pinned=pinned)
        basic = zb3d.BM3Dv2(clip, **kw)
        final = zb3d.BM3Dv2(clip, ref=basic, **kw)
        outs.append([[np.array(p) for p in final.get_frame(n)] for n in range(2)])
    for n in range(2):
        for p in range(3):
            assert np.array_equal(outs[0][n][p], outs[1][n][p])
    # pageable output buffers through the C ABI: the staging download path
    clip = zb3d.Clip.from_frames(frames, family=N.YUV, subsampling=(1, 1), pinned=True)
    nf = zb3d._create(1, clip, None, **{k: kw.get(k) for k in ("sigma", "block_step", "bm_range", "extractor_exp")},
                      radius=None, ps_num=None, ps_range=None, chroma=None, device_id=None, num_streams=None,
                      bm_error_s=None, transform_2d_s=None, transform_1d_s=None, zero_init=None, fast_fused=None)
    keep = []
    cf = (N.Frame * 1)(zb3d._frame_struct(clip.get_frame(0), keep))
    planes = [np.zeros(np.shape(frames[0][p]), np.float32) for p in range(3)]
    fo = N.FrameOut()
    for p, a in enumerate(planes):
        fo.ptr[p] = a.ctypes.data
        fo.stride[p] = a.strides[0]
    err = N.err_buf()
    assert N.lib().zb3d_get_frame(nf.h, 0, cf, None, ctypes.byref(fo), err, len(err)) == 0, err.value
    ref = zb3d.BM3Dv2(clip, **kw).get_frame(0)
    for p in range(3):
        assert np.array_equal(planes[p], ref[p])


def test_large_pageable_planes_split_over_copy_threads():
    """1920x1080 planes are staged by several copy threads (row chunks of at least 1 MiB):
    pageable input and output planes, mixed with page-locked ones, give the pinned bytes."""
    import ctypes
    w, h, sigma = 1920, 1080, 10.0
    plane = synth.noisy_plane(w, h, sigma, clip=9, frame=0)
    kw = dict(sigma=sigma, block_step=4, bm_range=12)
    pinned = zb3d.BM3Dv2(zb3d.Clip.from_frames([[plane]], pinned=True), **kw).get_frame(0)[0]
    clip = zb3d.Clip.from_frames([[plane]])
    nf = zb3d._create(1, clip, None, sigma=sigma, block_step=4, bm_range=12, radius=None, ps_num=None,
                      ps_range=None, chroma=None, device_id=None, num_streams=None, extractor_exp=None,
                      bm_error_s=None, transform_2d_s=None, transform_1d_s=None, zero_init=None, fast_fused=None)
    keep = []
    cf = (N.Frame * 1)(zb3d._frame_struct(clip.get_frame(0), keep))
    out = np.zeros((h, w + 3), np.float32)  # pageable, row stride not the plane width
    fo = N.FrameOut()
    fo.ptr[0] = out.ctypes.data
    fo.stride[0] = out.strides[0]
    err = N.err_buf()
    assert N.lib().zb3d_get_frame(nf.h, 0, cf, None, ctypes.byref(fo), err, len(err)) == 0, err.value
    assert np.array_equal(out[:, :w], np.asarray(pinned))


def test_graph_replay_equals_direct_launches():
    """Device entry points capture a window's launches into a CUDA graph on first use and
    replay it; profiling forces direct launches.  All three give the same bytes."""
    import torch
    from zb3d.device import DeviceFilter
    w, h = 320, 200
    f = DeviceFilter(w, h, family=N.YUV, subsampling=(1, 1), num_streams=1, sigma=[10.0] * 3, block_step=4,
                     bm_range=12, extractor_exp=3)
    src = np.zeros(f.src_elems, np.float32)
    for e, lay in enumerate(f.entries):
        src[lay.src_offset:lay.src_offset + lay.src_elems].reshape(lay.height, lay.pitch)[:, :lay.width] = \
            synth.noisy_plane(lay.width, lay.height, 10.0, plane=e)
    d_src = torch.from_numpy(src).cuda()
    outs = []
    for profile in (False, False, True):
        f.profile(profile)
        d_dst = torch.full((f.dst_elems,), float("nan"), dtype=torch.float32, device="cuda")
        f.run(d_src.data_ptr(), d_dst.data_ptr())
        torch.cuda.synchronize()
        outs.append(d_dst.cpu().numpy())
    f.profile(False)
    f.profile_collect()
    f.close()
    assert np.array_equal(outs[0].view(np.uint32), outs[1].view(np.uint32))
    assert np.array_equal(outs[0].view(np.uint32), outs[2].view(np.uint32))
