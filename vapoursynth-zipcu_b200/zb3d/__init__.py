"""zb3d: B200-native BM3D / BM3Dv2 / VAggregate.

Python mirror of the vszipcu plugin functions of this path
(``core.vszipcu.BM3D``, ``BM3Dv2``, ``VAggregate``; vszipcu src/plugin.zig:84-98):
same argument names, defaults, per-plane fallback rule and error strings, over a
small clip abstraction in place of VapourSynth nodes (VapourSynth itself is not
required).  Every frame is computed by the native library (CUDA, sm_100a) through
the C ABI of include/zb3d.h; there is no CPU path.

    clip = Clip.from_frames(frames, family=YUV, subsampling=(1, 1))
    basic = BM3Dv2(clip, sigma=10, block_step=4, bm_range=12)
    final = BM3Dv2(clip, ref=basic, sigma=10, block_step=4, bm_range=12)
    y, u, v = final.get_frame(0)
"""
from __future__ import annotations

import ctypes
import threading
from collections import OrderedDict
from typing import Callable, Optional, Sequence

import numpy as np

from . import _native as N

__all__ = ["Clip", "Error", "BM3D", "BM3Dv2", "VAggregate", "Pilot", "GRAY", "YUV", "RGB", "version",
           "pinned_empty"]

GRAY, RGB, YUV = N.GRAY, N.RGB, N.YUV
FLT_EPSILON = np.float32(1.19209290e-7)


class Error(Exception):
    """Raised where VapourSynth would raise vs.Error (create-time or frame errors)."""


class _PinnedBlock:
    """A page-locked host block from the library's pool (zb3d_host_alloc), exposed
    to numpy; returned to the pool when the last array using it goes away."""

    def __init__(self, shape):
        n = int(np.prod(shape)) * 4
        self.ptr = N.lib().zb3d_host_alloc(max(n, 4))
        if not self.ptr:
            raise MemoryError(f"zb3d_host_alloc({n}) failed")
        self.__array_interface__ = {"shape": tuple(shape), "typestr": "<f4", "data": (self.ptr, False),
                                    "version": 3}

    def __del__(self):
        try:
            N.lib().zb3d_host_free(self.ptr)
        except Exception:
            pass


def pinned_empty(shape) -> np.ndarray:
    """float32 array in page-locked host memory: frames in it reach the device by DMA
    alone (no staging copy)."""
    return np.asarray(_PinnedBlock(shape))


def version() -> str:
    return N.lib().zb3d_version().decode()


class Clip:
    """A clip of float32 planar frames.  ``get_frame(n)`` returns a list of 2-D
    numpy arrays (one per plane, shape (height, width) of that plane)."""

    def __init__(self, width: int, height: int, num_frames: int, family: int = GRAY,
                 subsampling=(0, 0), frame_fn: Optional[Callable[[int], list]] = None,
                 props_fn: Optional[Callable[[int], dict]] = None, sample_type: int = N.FLOAT,
                 bits: int = 32, cache: int = 16):
        self.width, self.height, self.num_frames = width, height, num_frames
        self.family = family
        self.subsampling = tuple(subsampling)
        self.num_planes = 1 if family == GRAY else 3
        self.sample_type, self.bits = sample_type, bits
        self._frame_fn = frame_fn
        self._props_fn = props_fn
        self._cache: "OrderedDict[int, list]" = OrderedDict()
        self._cache_size = cache
        self._lock = threading.Lock()

    @classmethod
    def from_frames(cls, frames: Sequence[Sequence[np.ndarray]], family: int = GRAY, subsampling=(0, 0),
                    pinned: bool = False) -> "Clip":
        """A clip over in-memory frames.  With ``pinned`` each plane is copied once into
        page-locked memory, which the filters then read by DMA."""
        if pinned:
            seen: dict = {}

            def pin(p):
                key = id(p)
                if key not in seen:
                    a = pinned_empty(np.shape(p))
                    a[...] = p
                    seen[key] = (p, a)
                return seen[key][1]

            frames = [[pin(p) for p in f] for f in frames]
        frames = [[np.ascontiguousarray(p, dtype=np.float32) for p in f] for f in frames]
        h, w = frames[0][0].shape
        return cls(w, h, len(frames), family, subsampling, frame_fn=lambda n: frames[n], cache=0)

    def info(self) -> N.VideoInfo:
        return N.VideoInfo(self.family, self.sample_type, self.bits, self.subsampling[0], self.subsampling[1],
                           self.num_planes, self.width, self.height, self.num_frames)

    def plane_shape(self, p: int):
        if p == 0:
            return self.height, self.width
        return self.height >> self.subsampling[1], self.width >> self.subsampling[0]

    def get_frame(self, n: int) -> list:
        if not 0 <= n < self.num_frames:
            raise Error(f"frame {n} out of range")
        with self._lock:
            if n in self._cache:
                self._cache.move_to_end(n)
                return self._cache[n]
        f = self._frame_fn(n)
        if self._cache_size:
            with self._lock:
                self._cache[n] = f
                while len(self._cache) > self._cache_size:
                    self._cache.popitem(last=False)
        return f

    def get_props(self, n: int) -> dict:
        return self._props_fn(n) if self._props_fn else {}


def _frame_struct(planes, keep: list) -> N.Frame:
    fr = N.Frame()
    for p, a in enumerate(planes[:3]):
        a = np.ascontiguousarray(a, dtype=np.float32)
        keep.append(a)
        fr.ptr[p] = a.ctypes.data
        fr.stride[p] = a.strides[0]
    return fr


class Pilot:
    """A learned pilot network loaded through the C ABI (zb3d_pilot_load) from a ZB3DPLT1
    weights file (default: the shipped 32 ch x 7 layer net with its gate).  Pass it as
    ``BM3Dv2(clip, sigma=..., pilot=p)`` to run both steps in one filter with the pilot as
    step 1 wherever its gate accepts the plane's sigma (the plain step 1 elsewhere).  The
    filters keep a reference to it."""

    def __init__(self, path: Optional[str] = None, device_id: int = 0):
        if path is None:
            import os
            path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "pilot_bs4_r12.zb3dp")
        err = N.err_buf()
        self.h = N.lib().zb3d_pilot_load(path.encode(), int(device_id), err, len(err))
        if not self.h:
            raise Error(err.value.decode())
        self.path, self.device_id = path, int(device_id)
        w, l, g = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        N.lib().zb3d_pilot_describe(self.h, ctypes.byref(w), ctypes.byref(l), ctypes.byref(g))
        self.width, self.layers = w.value, l.value
        self.gate = []  # (sigma, plane width, plane height, two-pass delta dB)
        for i in range(g.value):
            s, d, pw, ph = ctypes.c_float(), ctypes.c_float(), ctypes.c_int(), ctypes.c_int()
            N.lib().zb3d_pilot_gate_level(self.h, i, ctypes.byref(s), ctypes.byref(pw), ctypes.byref(ph),
                                          ctypes.byref(d))
            self.gate.append((s.value, pw.value, ph.value, d.value))

    def accepts(self, sigma: float, width: int, height: int) -> bool:
        """Whether the gate accepts the pilot for a width x height plane at this sigma."""
        return bool(N.lib().zb3d_pilot_accepts(self.h, float(sigma), int(width), int(height)))

    def __del__(self):
        try:
            if self.h:
                N.lib().zb3d_pilot_free(self.h)
                self.h = None
        except Exception:
            pass


def _per_plane(v, ctype):
    if v is None:
        return None, 0
    vals = list(v) if isinstance(v, (list, tuple, np.ndarray)) else [v]
    arr = (ctype * max(len(vals), 1))(*vals)
    return arr, len(vals)


def _strings(v):
    if v is None:
        return None, 0
    vals = list(v) if isinstance(v, (list, tuple)) else [v]
    enc = [s.encode() if isinstance(s, str) else bytes(s) for s in vals]
    return (ctypes.c_char_p * len(enc))(*enc), len(enc)


class _NativeFilter:
    def __init__(self, handle, free_fn):
        self.h = handle
        self._free = free_fn

    def __del__(self):
        try:
            if self.h:
                self._free(self.h)
                self.h = None
        except Exception:
            pass


def _make_args(ref, sigma, block_step, bm_range, radius, ps_num, ps_range, chroma, device_id, num_streams,
               extractor_exp, bm_error_s, transform_2d_s, transform_1d_s, zero_init, fast_fused, keep,
               match_form=None, pilot=None, filter_form=None):
    a = N.Args()
    N.lib().zb3d_args_init(ctypes.byref(a))
    if ref is not None:
        ri = ref.info()
        keep.append(ri)
        a.ref = ctypes.pointer(ri)
    for name, val, ct in (("sigma", sigma, ctypes.c_float), ("block_step", block_step, ctypes.c_int),
                          ("bm_range", bm_range, ctypes.c_int), ("ps_num", ps_num, ctypes.c_int),
                          ("ps_range", ps_range, ctypes.c_int)):
        arr, n = _per_plane(val, ct)
        if arr is not None:
            keep.append(arr)
            setattr(a, name, ctypes.cast(arr, type(getattr(a, name))))
            setattr(a, "n_" + name, n)
    for name, val in (("bm_error_s", bm_error_s), ("transform_2d_s", transform_2d_s),
                      ("transform_1d_s", transform_1d_s)):
        arr, n = _strings(val)
        if arr is not None:
            keep.append(arr)
            setattr(a, name, ctypes.cast(arr, ctypes.POINTER(ctypes.c_char_p)))
            setattr(a, "n_" + name, n)
    for name, val in (("radius", radius), ("chroma", chroma), ("device_id", device_id),
                      ("num_streams", num_streams), ("extractor_exp", extractor_exp),
                      ("zero_init", zero_init), ("fast_fused", fast_fused), ("match_form", match_form),
                      ("filter_form", filter_form)):
        if val is not None:
            setattr(a, name, int(val))
    if pilot is not None:
        keep.append(pilot)
        a.pilot = pilot.h
    return a


def _create(v2, clip, ref, **kw):
    keep: list = []
    a = _make_args(ref, keep=keep, **kw)
    ci = clip.info()
    err = N.err_buf()
    h = N.lib().zb3d_create(ctypes.byref(ci), ctypes.byref(a), v2, err, len(err))
    if not h:
        raise Error(err.value.decode())
    nf = _NativeFilter(h, N.lib().zb3d_free)
    nf.pilot = kw.get("pilot")  # the filter must not outlive its pilot
    return nf


def _filter_clip(nf: _NativeFilter, clip: Clip, ref: Optional[Clip]) -> Clip:
    lib = N.lib()
    out = N.VideoInfo()
    lib.zb3d_output_info(nf.h, ctypes.byref(out))
    r = ctypes.c_int()
    proc = (ctypes.c_int * 3)()
    lib.zb3d_output_props(nf.h, ctypes.byref(r), proc)
    radius, process = r.value, [bool(x) for x in proc]
    stacked = out.height != clip.height

    def frame(n):
        first, last = ctypes.c_int(), ctypes.c_int()
        lib.zb3d_frame_range(nf.h, n, ctypes.byref(first), ctypes.byref(last))
        keep: list = []
        cnt = last.value - first.value + 1
        cf = (N.Frame * cnt)(*[_frame_struct(clip.get_frame(i), keep) for i in range(first.value, last.value + 1)])
        rf = None
        if ref is not None:
            rf = (N.Frame * cnt)(*[_frame_struct(ref.get_frame(i), keep) for i in range(first.value, last.value + 1)])
        src = clip.get_frame(n)
        planes = []
        for p in range(clip.num_planes):
            h, w = clip.plane_shape(p)
            if stacked:
                h = h * out.height // clip.height
            planes.append(pinned_empty((h, w)) if (process[p] or stacked)
                          else np.array(src[p], dtype=np.float32, copy=True))
        fo = N.FrameOut()
        for p, a in enumerate(planes):
            fo.ptr[p] = a.ctypes.data
            fo.stride[p] = a.strides[0]
        err = N.err_buf()
        if lib.zb3d_get_frame(nf.h, n, cf, rf, ctypes.byref(fo), err, len(err)) != 0:
            raise Error(err.value.decode() or "BM3D: process frame failed.")
        return planes

    props = (lambda n: {"BM3D_V_radius": radius, "BM3D_V_process": [int(x) for x in process]}) if stacked else None
    c = Clip(out.width, out.height, out.num_frames, clip.family, clip.subsampling, frame_fn=frame, props_fn=props)
    c._native = nf
    return c


def BM3D(clip: Clip, ref: Optional[Clip] = None, sigma=None, block_step=None, bm_range=None, radius=None,
         ps_num=None, ps_range=None, chroma=None, device_id=None, num_streams=None, extractor_exp=None,
         bm_error_s=None, transform_2d_s=None, transform_1d_s=None, zero_init=None, fast_fused=None,
         match_form=None, filter_form=None) -> Clip:
    """vszipcu BM3D (src/bm3d.zig:965): with radius > 0 it returns the stacked
    accumulator clip (height * 2 * (2r+1)) that VAggregate consumes.  fast_fused is
    accepted and ignored, as in the reference (src/plugin.zig:83).  match_form (not
    in the reference): 0 (default) = FP32 scan of every candidate, 1 = tensor-core
    distance bound + exact FP32 re-rank; both give the same lists.  filter_form (not in the
    reference): 0 (default) = FP32 transforms, bit for bit the reference's; 1 = the precision
    form, 2D transforms on the tensor cores in split TF32 (FP32-level error, not bitwise)."""
    nf = _create(0, clip, ref, sigma=sigma, block_step=block_step, bm_range=bm_range, radius=radius,
                 ps_num=ps_num, ps_range=ps_range, chroma=chroma, device_id=device_id, num_streams=num_streams,
                 extractor_exp=extractor_exp, bm_error_s=bm_error_s, transform_2d_s=transform_2d_s,
                 transform_1d_s=transform_1d_s, zero_init=zero_init, fast_fused=None, match_form=match_form,
                 filter_form=filter_form)
    return _filter_clip(nf, clip, ref)


def _processed_planes(sigma, num_planes):
    proc = [True, True, True]
    vals = None if sigma is None else (list(sigma) if isinstance(sigma, (list, tuple, np.ndarray)) else [sigma])
    for i in range(3):
        if vals is not None and i < len(vals):
            proc[i] = not (np.float32(vals[i]) < FLT_EPSILON)
        elif i > 0:
            proc[i] = proc[i - 1]
    return proc[:num_planes]


def BM3Dv2(clip: Clip, ref: Optional[Clip] = None, sigma=None, block_step=None, bm_range=None, radius=None,
           ps_num=None, ps_range=None, chroma=None, device_id=None, num_streams=None, extractor_exp=None,
           bm_error_s=None, transform_2d_s=None, transform_1d_s=None, zero_init=None, fast_fused=None,
           match_form=None, pilot: Optional[Pilot] = None, filter_form=None) -> Clip:
    """vszipcu BM3Dv2 (src/bm3d.zig:1432-1501): pass-through when no plane is
    processed; radius 0 = BM3D; radius > 0 = BM3D + VAggregate, or the fused
    device path with fast_fused (same output bytes).  match_form as in BM3D.
    pilot (not in the reference; a Pilot, radius 0, no ref): the two-pass result
    BM3Dv2(clip, ref=<step 1>) in one filter, with the pilot as step 1 where its gate
    accepts the plane's sigma and the plain step 1 elsewhere."""
    proc = _processed_planes(sigma, clip.num_planes)
    if not any(proc):
        return clip
    if pilot is not None:
        nf = _create(1, clip, ref, sigma=sigma, block_step=block_step, bm_range=bm_range, radius=radius,
                     ps_num=ps_num, ps_range=ps_range, chroma=chroma, device_id=device_id, num_streams=num_streams,
                     extractor_exp=extractor_exp, bm_error_s=bm_error_s, transform_2d_s=transform_2d_s,
                     transform_1d_s=transform_1d_s, zero_init=zero_init, fast_fused=None, match_form=match_form,
                     pilot=pilot, filter_form=filter_form)
        return _filter_clip(nf, clip, None)
    kw = dict(sigma=sigma, block_step=block_step, bm_range=bm_range, radius=radius, ps_num=ps_num,
              ps_range=ps_range, chroma=chroma, device_id=device_id, num_streams=num_streams,
              extractor_exp=extractor_exp, bm_error_s=bm_error_s, transform_2d_s=transform_2d_s,
              transform_1d_s=transform_1d_s, zero_init=zero_init, match_form=match_form, filter_form=filter_form)
    r = 0 if radius is None else int(radius)
    if r > 0 and fast_fused:
        nf = _create(1, clip, ref, fast_fused=1, **kw)
        return _filter_clip(nf, clip, ref)
    stacked = BM3D(clip, ref, **kw)
    if r == 0:
        return stacked
    return VAggregate(stacked, clip, [i for i, p in enumerate(proc) if p])


def VAggregate(clip: Clip, src: Clip, planes) -> Clip:
    """vszipcu VAggregate (src/bm3d.zig:1372): temporal aggregation of a BM3D
    stacked clip, on the GPU (ascending FP32 sums, IEEE division)."""
    lib = N.lib()
    pl = list(planes) if isinstance(planes, (list, tuple)) else [planes]
    arr = (ctypes.c_int * max(len(pl), 1))(*pl)
    ci, si = clip.info(), src.info()
    err = N.err_buf()
    h = lib.zb3d_vaggregate_create(ctypes.byref(ci), ctypes.byref(si), arr, len(pl), err, len(err))
    if not h:
        raise Error(err.value.decode())
    nf = _NativeFilter(h, lib.zb3d_vaggregate_free)
    proc = [p in pl for p in range(3)]

    def frame(n):
        first, last = ctypes.c_int(), ctypes.c_int()
        lib.zb3d_vaggregate_frame_range(nf.h, n, ctypes.byref(first), ctypes.byref(last))
        keep: list = []
        cnt = last.value - first.value + 1
        st = (N.Frame * cnt)(*[_frame_struct(clip.get_frame(i), keep) for i in range(first.value, last.value + 1)])
        s = src.get_frame(n)
        planes_out = []
        for p in range(src.num_planes):
            hh, ww = src.plane_shape(p)
            planes_out.append(np.empty((hh, ww), np.float32) if proc[p] else np.array(s[p], np.float32, copy=True))
        fo = N.FrameOut()
        for p, a in enumerate(planes_out):
            fo.ptr[p] = a.ctypes.data
            fo.stride[p] = a.strides[0]
        e2 = N.err_buf()
        if lib.zb3d_vaggregate_get_frame(nf.h, n, st, ctypes.byref(fo), e2, len(e2)) != 0:
            raise Error(e2.value.decode())
        return planes_out

    c = Clip(src.width, src.height, src.num_frames, src.family, src.subsampling, frame_fn=frame)
    c._native = nf
    return c
