"""zb3d_process_batch: one persistent launch over the plane entries of many windows.

* The outputs of a batch of uneven jobs equal, byte for byte, each job run on its own
  through zb3d_process_device. The jobs cover luma and chroma planes of different sizes,
  block_step 4 and 8, a ragged width (clamped last block column), CBM3D, the Wiener step
  with a reference clip, and an entry the batch kernel does not take (SAD matching).
* Bounded waits: with the first entry's filter chunks waiting for one match tile more
  than exists, the call reports that they gave up, and the next batch on the same device
  is correct again.
* The same batch captured once as a CUDA graph (zb3d_batch_create) and replayed: equal
  outputs on every replay, status clear.
"""
import pytest

import zb3d
from zb3d import _native as N
from zb3d import synth
from zb3d.device import Batch, DeviceFilter, process_batch

pytestmark = pytest.mark.gpu


def _job(torch, w, h, family, seed, ref=False, **kw):
    sub = (1, 1) if family == N.YUV and not kw.get("chroma") else (0, 0)
    f = DeviceFilter(w, h, family=family, subsampling=sub, num_streams=1, ref=ref, **kw)
    src = torch.zeros(f.src_elems, dtype=torch.float32, device="cuda")
    for lay in f.entries:
        v = src[lay.src_offset:lay.src_offset + lay.src_elems].view(lay.nclips, lay.nplanes, lay.height, lay.pitch)
        for c in range(lay.nclips):
            for i in range(lay.nplanes):
                p = lay.plane[i]
                v[c, i, :, :lay.width] = torch.from_numpy(
                    synth.noisy_plane(lay.width, lay.height, 12.0 - 4.0 * c, clip=seed, frame=c, plane=p))
    return f, src


def _jobs(torch):
    specs = [
        (320, 240, N.GRAY, 1, False, dict(sigma=[10.0], block_step=4, bm_range=12)),
        (200, 120, N.YUV, 2, False, dict(sigma=[8.0, 6.0, 6.0], block_step=8, bm_range=9)),
        (77, 53, N.GRAY, 3, False, dict(sigma=[12.0], block_step=4, bm_range=7)),
        (96, 64, N.YUV, 4, False, dict(sigma=[10.0, 7.0, 7.0], block_step=8, bm_range=9, chroma=1)),
        (160, 96, N.GRAY, 5, True, dict(sigma=[10.0], block_step=4, bm_range=12, extractor_exp=3)),
        (128, 80, N.GRAY, 6, False, dict(sigma=[9.0], block_step=4, bm_range=8, bm_error_s="sad")),
    ]
    out = []
    for w, h, fam, seed, ref, kw in specs:
        f, src = _job(torch, w, h, fam, seed, ref=ref, **kw)
        out.append((f, src, torch.full((f.dst_elems,), -1.0, dtype=torch.float32, device="cuda")))
    return out


def _planes(f, buf):
    for lay in f.entries:
        yield lay, buf[lay.dst_offset:lay.dst_offset + lay.dst_elems].view(-1, lay.height, lay.pitch)[..., :lay.width]


def test_batch_equals_each_window_alone():
    import torch
    jobs = _jobs(torch)
    alone = []
    for f, src, _ in jobs:
        d = torch.full((f.dst_elems,), -1.0, dtype=torch.float32, device="cuda")
        f.run(src.data_ptr(), d.data_ptr())
        alone.append(d)
    torch.cuda.synchronize()
    for rep in range(2):  # the second call reuses the batch scratch
        for _, _, d in jobs:
            d.fill_(-1.0)
        torch.cuda.synchronize()
        process_batch([(f, s.data_ptr(), d.data_ptr()) for f, s, d in jobs])
        for (f, _, d), a in zip(jobs, alone):
            for (lay, x), (_, y) in zip(_planes(f, d), _planes(f, a)):
                assert torch.equal(x, y), (rep, lay.width, lay.height)


def test_batch_waits_run_out_and_report_it():
    import torch
    jobs = _jobs(torch)[:3]
    torch.cuda.synchronize()
    with pytest.raises(zb3d.Error, match="gave up waiting"):
        process_batch([(f, s.data_ptr(), d.data_ptr()) for f, s, d in jobs], wait_polls=1 << 12,
                      unsatisfiable=True)
    # the device is usable afterwards and the next batch is complete and correct
    alone = []
    for f, src, _ in jobs:
        d = torch.empty(f.dst_elems, dtype=torch.float32, device="cuda")
        f.run(src.data_ptr(), d.data_ptr())
        alone.append(d)
    torch.cuda.synchronize()
    process_batch([(f, s.data_ptr(), d.data_ptr()) for f, s, d in jobs])
    for (f, _, d), a in zip(jobs, alone):
        for (lay, x), (_, y) in zip(_planes(f, d), _planes(f, a)):
            assert torch.equal(x, y), (lay.width, lay.height)


def test_batch_graph_replays_equal_each_window_alone():
    import torch
    jobs = _jobs(torch)
    alone = []
    for f, src, _ in jobs:
        d = torch.full((f.dst_elems,), -1.0, dtype=torch.float32, device="cuda")
        f.run(src.data_ptr(), d.data_ptr())
        alone.append(d)
    torch.cuda.synchronize()
    b = Batch([(f, s.data_ptr(), d.data_ptr()) for f, s, d in jobs])
    st = torch.cuda.Stream()
    try:
        for rep in range(3):
            for _, _, d in jobs:
                d.fill_(-1.0)
            torch.cuda.synchronize()
            b.launch(st.cuda_stream)
            st.synchronize()
            b.status()
            for (f, _, d), a in zip(jobs, alone):
                for (lay, x), (_, y) in zip(_planes(f, d), _planes(f, a)):
                    assert torch.equal(x, y), (rep, lay.width, lay.height)
    finally:
        b.close()
