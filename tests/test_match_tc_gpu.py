"""The tensor-core matching form (zb3d_match_tc.cu) against the FP32 scan.

1. The pass-1 distances of tile (0, 0), read back from tensor memory, equal
   |b - c0|^2 - 2 (mu - c0) S - 2 (a - mu).(b - c0) = SSD - |a - c0|^2 within the
   bound eps the kernel uses, and every window candidate of every block is read.
   This pins the operand layouts (the expanded-row operand B, the norm table),
   descriptors and TMEM lanes on the hardware and checks the error bound the
   exactness argument rests on.
2. Match lists (and outputs) of match_form=1 are bit-identical to match_form=0
   over block steps, ranges, noise levels, partial tiles, the clamped last block
   column and temporal windows.
"""
import ctypes

import numpy as np
import pytest

from zb3d import _native as N
from zb3d import synth
from zb3d.device import DeviceFilter, unpack_list

pytestmark = pytest.mark.gpu

def _tile_geom(w, h, bs, R):
    nbx = (w - 8 + bs - 1) // bs + 1
    nby = (h - 8 + bs - 1) // bs + 1
    nvx, nvy = min(8, nbx), min(16, nby)
    bx = [min(bs * k, w - 8) for k in range(nvx)]
    by = [min(bs * k, h - 8) for k in range(nvy)]
    ux0, uy0 = max(bx[0] - R, 0), max(by[0] - R, 0)
    nuc = min(bx[-1] + R, w - 8) - ux0 + 1
    nur = min(by[-1] + R, h - 8) - uy0 + 1
    return bx, by, ux0, uy0, nuc, nur, 56  # flat candidates f = row * 56 + column


def _expected(plane, w, h, bs, R):
    """float64 d(m, f) for tile (0, 0), the kernel's eps per block, window masks."""
    bx, by, ux0, uy0, nuc, nur, stride = _tile_geom(w, h, bs, R)
    img = plane[:, :w].astype(np.float64)
    P = np.lib.stride_tricks.sliding_window_view(img, (8, 8))
    mus = [img[y:y + 8, x:x + 8].mean() for y in by for x in bx]
    c0 = float(np.float32(np.mean(np.float32(mus))))
    cand = P[uy0:uy0 + nur, ux0:ux0 + nuc].reshape(nur, nuc, 64)
    bh = cand - c0
    pn = (bh ** 2).sum(-1)
    sm = np.abs(bh.sum(-1)).max()
    out = {}
    for m in range(128):
        bxl, byl = m % 8, m // 8
        if bxl >= len(bx) or byl >= len(by):
            continue
        xb, yb = bx[bxl], by[byl]
        a = img[yb:yb + 8, xb:xb + 8].reshape(64)
        e = ((cand - a) ** 2).sum(-1)
        ah2 = ((a - c0) ** 2).sum()
        d = e - ah2
        win = np.zeros((nur, nuc), bool)
        win[max(yb - R, 0) - uy0:min(yb + R, h - 8) - uy0 + 1, max(xb - R, 0) - ux0:min(xb + R, w - 8) - ux0 + 1] = True
        rows = np.where(win.any(1))[0]
        pm = pn[rows].max()
        an = np.sqrt(((a - a.mean()) ** 2).sum())
        nu = a.mean() - c0
        eps = 1.01 * 2.0 ** -9 * an * np.sqrt(pm) + 2.0 ** -15 * (2 * an * np.sqrt(pm) + 2 * abs(nu) * sm + pm + ah2 + 1)
        out[m] = (d, win, eps)
    return out, (ux0, uy0, nuc, nur, stride)


def _probe(plane, w, h, bs, R):
    import torch
    cols = N.lib().zb3d_tc_probe_cols(w, h, bs, R)
    assert cols > 0
    d_plane = torch.from_numpy(np.ascontiguousarray(plane)).cuda()
    nbx = (w - 8 + bs - 1) // bs + 1
    nby = (h - 8 + bs - 1) // bs + 1
    d_list = torch.zeros((nby, nbx, 8, 2), dtype=torch.int32, device="cuda")
    d_dist = torch.full((128, cols), float("nan"), dtype=torch.float32, device="cuda")
    st = (ctypes.c_ulonglong * 4)()
    err = N.err_buf()
    rc = N.lib().zb3d_tc_probe(d_plane.data_ptr(), w, h, plane.shape[1], bs, R, d_list.data_ptr(),
                               d_dist.data_ptr(), None, st, err, len(err))
    assert rc == 0, err.value.decode()
    return d_dist.cpu().numpy(), unpack_list(d_list.cpu().numpy()), tuple(st)


@pytest.mark.parametrize("w,h,bs,R,sigma", [(96, 96, 4, 12, 10.0), (200, 150, 4, 12, 3.0), (77, 61, 3, 9, 20.0)])
def test_tc_distances_within_bound(w, h, bs, R, sigma):
    plane = synth.noisy_plane(w, h, sigma, clip=7)
    dist, _, _ = _probe(plane, w, h, bs, R)
    exp, (ux0, uy0, nuc, nur, stride) = _expected(plane, w, h, bs, R)
    worst = 0.0
    for m, (d, win, eps) in exp.items():
        row = dist[m][:nur * stride].reshape(nur, stride)[:, :nuc]
        assert not np.isnan(row[win]).any(), f"block {m}: window candidates not read"
        err = np.abs(row[win] - d[win])
        worst = max(worst, float((err / eps).max()))
        assert (err <= eps).all(), f"block {m}: |d - exact| {err.max():.3g} > eps {eps:.3g}"
    print(f"max |d - exact| / eps = {worst:.3f}")


def _lists(w, h, bs, R, sigma, form, radius=0, clip=0, motion=False):
    import torch
    tw = 2 * radius + 1
    f = DeviceFilter(w, h, family=N.GRAY, num_frames=tw, sigma=[sigma], block_step=bs, bm_range=R,
                     radius=radius, num_streams=1, match_form=form)
    lay = f.entries[0]
    src = np.zeros(f.src_elems, np.float32)
    view = src[lay.src_offset:lay.src_offset + lay.src_elems].reshape(1, 1, tw, h, lay.pitch)
    for t in range(tw):
        view[0, 0, t, :, :w] = synth.noisy_plane(w, h, sigma, clip=clip, frame=t, motion=motion)
    d_src = torch.from_numpy(src).cuda()
    nbx = (w - 8 + bs - 1) // bs + 1
    nby = (h - 8 + bs - 1) // bs + 1
    d_list = torch.zeros((nby, nbx, 8, 2), dtype=torch.int32, device="cuda")
    f.match(0, d_src.data_ptr(), d_list.data_ptr())
    torch.cuda.synchronize()
    stats = f.match_stats() if form == 1 else None
    d_dst = torch.zeros(f.dst_elems, dtype=torch.float32, device="cuda")
    f.run(d_src.data_ptr(), d_dst.data_ptr())
    torch.cuda.synchronize()
    out = d_dst.cpu().numpy()
    f.close()
    return d_list.cpu().numpy(), out, stats


CASES = [
    (1920, 1080, 4, 12, 10.0),   # the two-pass workload's luma plane
    (960, 540, 4, 12, 10.0),     # its chroma planes
    (640, 480, 4, 12, 3.0),
    (333, 211, 4, 12, 25.0),     # partial tiles, clamped last block column and row
    (300, 200, 2, 13, 10.0),
    (300, 200, 3, 9, 5.0),
    (256, 160, 4, 5, 10.0),
    (130, 90, 1, 6, 10.0),
]


@pytest.mark.parametrize("w,h,bs,R,sigma", CASES)
def test_tc_lists_and_outputs_equal_fp32_scan(w, h, bs, R, sigma):
    l0, o0, _ = _lists(w, h, bs, R, sigma, 0)
    l1, o1, st = _lists(w, h, bs, R, sigma, 1)
    tiles, blocks, reranked, fallbacks = st
    nb = l0.shape[0] * l0.shape[1]
    assert blocks == nb and tiles > 0, st
    mism = np.any(l0 != l1, axis=(2, 3))
    assert not mism.any(), f"{int(mism.sum())}/{mism.size} blocks differ"
    assert np.array_equal(o0.view(np.uint32), o1.view(np.uint32))
    # the bound is tight enough that almost every block is settled by the tensor cores (a
    # failed self-check would send whole tiles to the FP32 scan)
    assert fallbacks <= 0.01 * blocks, st
    print(f"{w}x{h} bs{bs} R{R} sigma{sigma}: {reranked / max(blocks - fallbacks, 1):.1f} re-ranked per block, "
          f"{fallbacks / blocks:.2%} fallback")


def test_tc_temporal_window_equal_fp32_scan():
    l0, o0, _ = _lists(480, 270, 4, 12, 15.0, 0, radius=2, clip=3, motion=True)
    l1, o1, _ = _lists(480, 270, 4, 12, 15.0, 1, radius=2, clip=3, motion=True)
    assert np.array_equal(l0, l1)
    assert np.array_equal(o0.view(np.uint32), o1.view(np.uint32))


def test_tc_out_of_range_tiles_fall_back():
    # pixels beyond the FP16 sizing (|x| > 4) send their tiles to the FP32 scan
    w, h = 160, 128
    l0, _, _ = _lists(w, h, 4, 12, 10.0, 0, clip=11)
    import torch
    f = DeviceFilter(w, h, family=N.GRAY, num_frames=1, sigma=[10.0], block_step=4, bm_range=12,
                     num_streams=1, match_form=1)
    lay = f.entries[0]
    src = np.zeros(f.src_elems, np.float32)
    view = src[lay.src_offset:lay.src_offset + lay.src_elems].reshape(h, lay.pitch)
    img = synth.noisy_plane(w, h, 10.0, clip=11)
    img[40:48, 50:60] = 9.0
    view[:, :w] = img
    d_src = torch.from_numpy(src).cuda()
    nbx, nby = (w - 8 + 3) // 4 + 1, (h - 8 + 3) // 4 + 1
    d_list = torch.zeros((nby, nbx, 8, 2), dtype=torch.int32, device="cuda")
    f.match(0, d_src.data_ptr(), d_list.data_ptr())
    torch.cuda.synchronize()
    st = f.match_stats()
    f.close()
    assert st[3] > 0
    # and the lists still equal the FP32 scan of the same frame
    f0 = DeviceFilter(w, h, family=N.GRAY, num_frames=1, sigma=[10.0], block_step=4, bm_range=12,
                      num_streams=1, match_form=0)
    d_list0 = torch.zeros_like(d_list)
    f0.match(0, d_src.data_ptr(), d_list0.data_ptr())
    torch.cuda.synchronize()
    f0.close()
    assert torch.equal(d_list, d_list0)


def test_autotuner_picks_a_valid_form_caches_it_and_stays_exact(tmp_path, monkeypatch):
    import torch
    cache = tmp_path / "tune.txt"
    monkeypatch.setenv("ZB3D_TUNE_CACHE", str(cache))
    w, h = 480, 272
    plane = synth.noisy_plane(w, h, 10.0, clip=5)

    def lists_for(**kw):
        f = DeviceFilter(w, h, family=N.GRAY, num_frames=1, sigma=[10.0], block_step=4, bm_range=12,
                         num_streams=1, **kw)
        lay = f.entries[0]
        src = np.zeros(f.src_elems, np.float32)
        src[lay.src_offset:lay.src_offset + lay.src_elems].reshape(h, lay.pitch)[:, :w] = plane
        d_src = torch.from_numpy(src).cuda()
        nbx, nby = (w - 8 + 3) // 4 + 1, (h - 8 + 3) // 4 + 1
        d_list = torch.zeros((nby, nbx, 8, 2), dtype=torch.int32, device="cuda")
        f.match(0, d_src.data_ptr(), d_list.data_ptr())
        torch.cuda.synchronize()
        t = f.tuning(0)
        f.close()
        return d_list.cpu().numpy(), t

    l_auto, (form, rows) = lists_for()
    assert form in (0, 1) and rows in (2, 4)
    text = cache.read_text()
    assert f" {form} {rows}" in text and "_w480_h272_" in text
    _, again = lists_for()
    assert again == (form, rows)
    assert cache.read_text() == text  # served from the cache, not re-timed
    l0, _ = lists_for(match_form=0)
    l1, t1 = lists_for(match_form=1)
    assert t1[0] == 1
    assert np.array_equal(l_auto, l0) and np.array_equal(l_auto, l1)
