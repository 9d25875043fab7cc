"""zb3d_bm3d_plane_noalloc, the entry point for callers that cannot allocate
device memory while they run (its scratch is a fixed array inside the library),
called through the C ABI and compared with the regular device path
(zb3d_process_entry_device) on consecutive calls: the shared scratch must not
carry anything from one call into the next.  Collected last on purpose."""
import ctypes

import numpy as np
import pytest

from zb3d import _native as N
from zb3d import synth
from zb3d.device import DeviceFilter

pytestmark = pytest.mark.gpu

KW = dict(block_step=4, bm_range=12, extractor_exp=3)


def _regular(w, h, sigma, final, src_host, block_step=4):
    import torch
    kw = dict(KW, block_step=block_step)
    f = DeviceFilter(w, h, num_frames=1, ref=bool(final), sigma=[sigma], num_streams=1, **kw)
    lay = f.entries[0]
    d_src = torch.from_numpy(src_host.reshape(-1)).cuda()
    d_dst = torch.full((lay.dst_elems,), float("nan"), dtype=torch.float32, device="cuda")
    f.run_entry(0, d_src.data_ptr(), d_dst.data_ptr())
    torch.cuda.synchronize()
    out = d_dst.cpu().numpy().reshape(h, lay.pitch)
    pitch = lay.pitch
    f.close()
    return out, pitch


def _noalloc(w, h, pitch, sigma, final, src_host, block_step=4):
    import torch
    d_src = torch.from_numpy(src_host.reshape(-1)).cuda()
    d_dst = torch.full((h * pitch,), float("nan"), dtype=torch.float32, device="cuda")
    err = N.err_buf()
    rc = N.lib().zb3d_bm3d_plane_noalloc(d_src.data_ptr(), d_dst.data_ptr(), w, h, pitch, int(final), sigma,
                                         block_step, KW["bm_range"], KW["extractor_exp"], None, err, len(err))
    assert rc == 0, err.value.decode()
    torch.cuda.synchronize()
    return d_dst.cpu().numpy().reshape(h, pitch)


def _plane(w, h, pitch, sigma, frame):
    p = np.zeros((h, pitch), np.float32)
    p[:, :w] = synth.noisy_plane(w, h, sigma, frame=frame)[:, :w]
    return p


def test_noalloc_matches_regular_path_on_consecutive_calls():
    sigma = 10.0
    # call 1: basic estimate of a 320x240 plane
    w, h = 320, 240
    pitch = (w + 31) // 32 * 32
    noisy = _plane(w, h, pitch, sigma, 0)
    reg_b, rp = _regular(w, h, sigma, 0, noisy)
    assert rp == pitch
    got_b = _noalloc(w, h, pitch, sigma, 0, noisy)
    assert np.array_equal(got_b[:, :w], reg_b[:, :w])
    # call 2: Wiener pass on top of it (the scratch still holds call 1's sums)
    two = np.stack([np.where(np.isnan(got_b), 0, got_b), noisy])
    reg_f, _ = _regular(w, h, sigma, 1, two)
    got_f = _noalloc(w, h, pitch, sigma, 1, two)
    assert np.array_equal(got_f[:, :w], reg_f[:, :w])
    # call 3: another frame of another size
    w2, h2 = 200, 136
    pitch2 = (w2 + 31) // 32 * 32
    noisy2 = _plane(w2, h2, pitch2, sigma, 5)
    reg_2, _ = _regular(w2, h2, sigma, 0, noisy2)
    got_2 = _noalloc(w2, h2, pitch2, sigma, 0, noisy2)
    assert np.array_equal(got_2[:, :w2], reg_2[:, :w2])


def _repitch(p, w, pitch):
    """The same plane(s) at another row pitch (padding zero)."""
    out = np.zeros(p.shape[:-1] + (pitch,), np.float32)
    out[..., :w] = p[..., :w]
    return out


@pytest.mark.parametrize("block_step", [4, 3])
def test_noalloc_ragged_width_and_odd_pitch(block_step):
    """A 77x53 plane: at block_step 4 the last block column is clamped (x = w - 8), and
    block_step 3 runs the generic matcher.  The caller's pitch (83 floats) is not one the
    regular path would choose; outputs do not depend on the pitch, so they must equal the
    regular path's at its own pitch."""
    sigma = 10.0
    w, h = 77, 53
    reg_pitch = (w + 31) // 32 * 32
    noisy = _plane(w, h, reg_pitch, sigma, 3)
    reg_b, _ = _regular(w, h, sigma, 0, noisy, block_step)
    got_b = _noalloc(w, h, 83, sigma, 0, _repitch(noisy, w, 83), block_step)
    assert np.array_equal(got_b[:, :w], reg_b[:, :w])
    two = np.stack([np.where(np.isnan(reg_b), 0, reg_b), noisy])
    reg_f, _ = _regular(w, h, sigma, 1, two, block_step)
    got_f = _noalloc(w, h, 83, sigma, 1, _repitch(two, w, 83), block_step)
    assert np.array_equal(got_f[:, :w], reg_f[:, :w])


def test_noalloc_leaves_a_zero_sigma_plane_unprocessed():
    """sigma below FLT_EPSILON: the plane is not filtered (as BM3D skips it) and the output
    is the noisy plane, also in the Wiener pass over a flat basic estimate."""
    w, h = 64, 40
    pitch = 64
    flat = np.full((h, pitch), 0.5, np.float32)
    noisy = _plane(w, h, pitch, 10.0, 7)
    got = _noalloc(w, h, pitch, 0.0, 1, np.stack([flat, noisy]))
    assert np.array_equal(got[:, :w], noisy[:, :w])
    got0 = _noalloc(w, h, pitch, 0.0, 0, noisy)
    assert np.array_equal(got0[:, :w], noisy[:, :w])


def test_noalloc_rejects_planes_beyond_its_scratch():
    import torch
    w, h = 1920, 1080  # 2.07 M pitched pixels > 1 M
    d = torch.zeros(16, dtype=torch.float32, device="cuda")
    err = N.err_buf()
    rc = N.lib().zb3d_bm3d_plane_noalloc(d.data_ptr(), d.data_ptr(), w, h, w, 0, 10.0, 4, 12, 3, None, err,
                                         len(err))
    assert rc == -1
    assert "too large for the built-in scratch" in err.value.decode()
    err = N.err_buf()
    rc = N.lib().zb3d_bm3d_plane_noalloc(d.data_ptr(), d.data_ptr(), 64, 48, 32, 0, 10.0, 4, 12, 3, None, err,
                                         len(err))
    assert rc == -1 and "invalid arguments" in err.value.decode()
