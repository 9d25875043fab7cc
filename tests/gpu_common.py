"""GPU helpers of the test-suite: run the product kernels and the reference
kernels on the same window."""
from __future__ import annotations

import numpy as np

from zb3d import _native as N
from zb3d.device import DeviceFilter, unpack_list


def metric_name(m: str) -> str:
    return "ssd/norm" if m == "ssd_norm" else m


def transform_name(t: str) -> str:
    return "bior1.5" if t == "bior1_5" else t


def product_filter(spec, **over) -> DeviceFilter:
    fam = N.YUV if spec.chroma else N.GRAY
    sig = list(spec.sigma) if spec.chroma else [spec.sigma[0]]
    kw = dict(sigma=sig, block_step=spec.block_step, bm_range=spec.bm_range, radius=spec.radius,
              ps_num=spec.ps_num, ps_range=spec.ps_range, chroma=spec.chroma,
              extractor_exp=spec.extractor_exp, bm_error_s=metric_name(spec.bm_error),
              transform_2d_s=transform_name(spec.t2d), transform_1d_s=transform_name(spec.t1d), num_streams=1)
    kw.update(over)
    return DeviceFilter(spec.w, spec.h, family=fam, num_frames=2 * spec.radius + 1, ref=bool(spec.final), **kw)


def to_product_layout(f: DeviceFilter, src_ref_layout: np.ndarray) -> np.ndarray:
    """[clips][planes][tw][h][stride] (reference pitch) -> product entry layout."""
    out = np.zeros(f.src_elems, np.float32)
    lay = f.entries[0]
    c, p, t, h, _ = src_ref_layout.shape
    view = out[lay.src_offset:lay.src_offset + lay.src_elems].reshape(c, p, t, h, lay.pitch)
    view[..., :lay.width] = src_ref_layout[..., :lay.width]
    return out


def run_product(spec, src_np, runs: int = 1, **over):
    import torch
    f = product_filter(spec, **over)
    lay = f.entries[0]
    d_src = torch.from_numpy(to_product_layout(f, src_np)).cuda()
    outs = []
    for _ in range(runs):
        d_dst = torch.full((f.dst_elems,), float("nan"), dtype=torch.float32, device="cuda")
        f.run(d_src.data_ptr(), d_dst.data_ptr())
        torch.cuda.synchronize()
        outs.append(d_dst.cpu().numpy())
    nbx = (spec.w - 8 + spec.block_step - 1) // spec.block_step + 1
    nby = (spec.h - 8 + spec.block_step - 1) // spec.block_step + 1
    d_list = torch.zeros((nby, nbx, 8, 2), dtype=torch.int32, device="cuda")
    f.match(0, d_src.data_ptr(), d_list.data_ptr())
    torch.cuda.synchronize()
    lists = unpack_list(d_list.cpu().numpy())
    planes = lay.nplanes
    tw = 2 * spec.radius + 1
    shaped = []
    for o in outs:
        seg = o[lay.dst_offset:lay.dst_offset + lay.dst_elems]
        if spec.radius == 0:
            shaped.append(seg.reshape(planes, spec.h, lay.pitch)[..., :spec.w])
        else:
            shaped.append(seg.reshape(planes, tw, 2, spec.h, lay.pitch)[..., :spec.w])
    f.close()
    return shaped, lists
