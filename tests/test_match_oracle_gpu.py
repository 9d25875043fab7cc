"""Match lists of the FP32 matchers against the CPU oracle's exact lists (oracle.match, which
test_ref_pin.py pins to the reference kernels), on paths the parity configurations do not
reach:

* the packed tile's half-plane layout sized at run time (bm_range > 15 at block_step 4 and
  8), with ragged widths (the clamped last block column) and both the default CTA shape and
  the one the autotuner picks (2, 4 or 8 block rows);
* the temporal search with per-frame lists of 2 entries (ps_num 1 and 2) and of 8 entries
  (ps_num 3 and 5), over moving frames.
"""
import numpy as np
import pytest

import oracle as orc
from zb3d import _native as N
from zb3d import synth
from zb3d.device import DeviceFilter, unpack_list

pytestmark = pytest.mark.gpu

CASES = [
    # w, h, block_step, bm_range, radius, ps_num, sigma
    (320, 200, 4, 16, 0, 2, 10.0),
    (333, 211, 4, 20, 0, 2, 25.0),
    (320, 208, 8, 24, 0, 2, 10.0),
    (301, 157, 8, 17, 0, 2, 5.0),
    (160, 120, 8, 9, 2, 1, 15.0),
    (160, 120, 8, 9, 2, 2, 15.0),
    (150, 110, 4, 7, 1, 3, 15.0),
    (160, 120, 8, 9, 2, 5, 15.0),
]


@pytest.mark.parametrize("autotune", ["0", "1"])
@pytest.mark.parametrize("w,h,bs,R,radius,ps_num,sigma", CASES)
def test_match_lists_equal_oracle(w, h, bs, R, radius, ps_num, sigma, autotune, monkeypatch, tmp_path):
    import torch
    monkeypatch.setenv("ZB3D_AUTOTUNE", autotune)
    monkeypatch.setenv("ZB3D_TUNE_CACHE", str(tmp_path / "tune.txt"))
    tw = 2 * radius + 1
    f = DeviceFilter(w, h, family=N.GRAY, num_frames=tw, sigma=[sigma], block_step=bs, bm_range=R, radius=radius,
                     ps_num=ps_num, ps_range=4, num_streams=1, match_form=0)
    lay = f.entries[0]
    planes = [synth.noisy_plane(w, h, sigma, clip=3, frame=t, motion=True, stride=lay.pitch) for t in range(tw)]
    src = np.zeros(f.src_elems, np.float32)
    view = src[lay.src_offset:lay.src_offset + lay.src_elems].reshape(tw, h, lay.pitch)
    for t in range(tw):
        view[t] = planes[t]
    d_src = torch.from_numpy(src).cuda()
    nbx = (w - 8 + bs - 1) // bs + 1
    nby = (h - 8 + bs - 1) // bs + 1
    d_list = torch.zeros((nby, nbx, 8, 2), dtype=torch.int32, device="cuda")
    f.match(0, d_src.data_ptr(), d_list.data_ptr())
    torch.cuda.synchronize()
    got = unpack_list(d_list.cpu().numpy())
    form, rows = f.tuning(0)
    f.close()

    cfg = orc.make_cfg(w, h, lay.pitch, [sigma / 255.0], bs, R, radius, ps_num, 4)
    want = orc.match(cfg, planes)
    bad = np.any(got != want, axis=(2, 3))
    assert not bad.any(), (f"{bad.sum()} of {bad.size} blocks differ (form {form}, {rows} rows per CTA); "
                           f"first {np.argwhere(bad)[:4].tolist()}")
