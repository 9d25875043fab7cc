"""Device-resident driver of one BM3D filter window (inputs already in HBM).

Thin wrapper over zb3d_process_device / zb3d_match_device: buffers are passed as
raw device addresses (e.g. ``tensor.data_ptr()``), streams as raw handles.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _native as N
from . import Error, _make_args


class DeviceFilter:
    """BM3D over device buffers laid out per entry: src [clips][planes][tw][h][pitch],
    dst [planes][h][pitch] (stacked [planes][tw][2][h][pitch] when radius > 0)."""

    def __init__(self, width, height, family=N.GRAY, subsampling=(0, 0), num_frames=1, ref=False, **kw):
        lib = N.lib()
        nplanes = 1 if family == N.GRAY else 3
        self.info = N.VideoInfo(family, N.FLOAT, 32, subsampling[0], subsampling[1], nplanes, width, height,
                                num_frames)
        keep: list = []

        class _Ref:
            def __init__(s, i):
                s._i = i

            def info(s):
                return s._i

        a = _make_args(_Ref(self.info) if ref else None, keep=keep, **self._defaults(kw))
        err = N.err_buf()
        self.h = lib.zb3d_create(ctypes.byref(self.info), ctypes.byref(a), 0, err, len(err))
        if not self.h:
            raise Error(err.value.decode())
        self.entries = []
        for e in range(lib.zb3d_num_entries(self.h)):
            lay = N.EntryLayout()
            lib.zb3d_entry_layout_get(self.h, e, ctypes.byref(lay))
            self.entries.append(lay)
        self.src_elems = lib.zb3d_src_elems(self.h)
        self.dst_elems = lib.zb3d_dst_elems(self.h)

    @staticmethod
    def _defaults(kw):
        names = ("sigma", "block_step", "bm_range", "radius", "ps_num", "ps_range", "chroma", "device_id",
                 "num_streams", "extractor_exp", "bm_error_s", "transform_2d_s", "transform_1d_s", "zero_init",
                 "fast_fused", "match_form", "filter_form")
        return {n: kw.get(n) for n in names}

    def run(self, src_ptr: int, dst_ptr: int, stream: int = 0):
        err = N.err_buf()
        if N.lib().zb3d_process_device(self.h, src_ptr, dst_ptr, stream or None, err, len(err)) != 0:
            raise Error(err.value.decode())

    def run_entry(self, e: int, src_ptr: int, dst_ptr: int, stream: int = 0):
        err = N.err_buf()
        if N.lib().zb3d_process_entry_device(self.h, e, src_ptr, dst_ptr, stream or None, err, len(err)) != 0:
            raise Error(err.value.decode())

    def profile(self, on: bool = True):
        N.lib().zb3d_profile_enable(self.h, int(on))

    def profile_collect(self):
        """(match_ms, match_launches, filter_ms, filter_launches) since the last collect."""
        mm, fm = ctypes.c_double(), ctypes.c_double()
        mn, fn = ctypes.c_int(), ctypes.c_int()
        N.lib().zb3d_profile_collect(self.h, ctypes.byref(mm), ctypes.byref(mn), ctypes.byref(fm), ctypes.byref(fn))
        return mm.value, mn.value, fm.value, fn.value

    def tuning(self, e: int = 0):
        """(form, rows) the autotuner chose for entry e."""
        form, rows = ctypes.c_int(), ctypes.c_int()
        if N.lib().zb3d_entry_tuning(self.h, e, ctypes.byref(form), ctypes.byref(rows)) != 0:
            raise Error("no such entry")
        return form.value, rows.value

    def match_stats(self, reset: bool = False):
        """Tensor-core form counters: (tiles, blocks, re-ranked candidates, fallback blocks)."""
        out = (ctypes.c_ulonglong * 4)()
        if N.lib().zb3d_match_stats(self.h, out, int(reset)) != 0:
            raise Error("zb3d_match_stats failed")
        return tuple(int(v) for v in out)

    def match(self, e: int, src_ptr: int, list_ptr: int, stream: int = 0):
        err = N.err_buf()
        if N.lib().zb3d_match_device(self.h, e, src_ptr, list_ptr, stream or None, err, len(err)) != 0:
            raise Error(err.value.decode())

    def close(self):
        if self.h:
            N.lib().zb3d_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def unpack_list(raw: np.ndarray) -> np.ndarray:
    """[..., 8, 2] int32 (x, y | z << 24) -> [..., 8, 3] (x, y, z)."""
    x = raw[..., 0]
    y = raw[..., 1] & 0xFFFFFF
    z = (raw[..., 1].astype(np.int64) >> 24) & 0xFF
    return np.stack([x, y, z.astype(np.int32)], axis=-1)


def process_batch(jobs, stream: int = 0, wait_polls: int = 0, unsatisfiable: bool = False):
    """One window of each job in one call (zb3d_process_batch): jobs = [(DeviceFilter, src_ptr,
    dst_ptr), ...].  Synchronous; raises Error with the library's reason on failure."""
    arr = (N.BatchJob * len(jobs))(*[N.BatchJob(f.h, s, d) for f, s, d in jobs])
    err = N.err_buf()
    rc = N.lib().zb3d_process_batch_ex(arr, len(jobs), stream or None, int(wait_polls), int(bool(unsatisfiable)),
                                       err, len(err))
    if rc != 0:
        raise Error(err.value.decode())


class Batch:
    """A batch captured once as a CUDA graph (zb3d_batch_create): jobs = [(DeviceFilter, src_ptr,
    dst_ptr), ...].  launch() replays it on a stream asynchronously; status() after the stream
    was synchronised raises Error if a filter chunk of the last launch gave up waiting."""

    def __init__(self, jobs):
        arr = (N.BatchJob * len(jobs))(*[N.BatchJob(f.h, s, d) for f, s, d in jobs])
        err = N.err_buf()
        self.h = N.lib().zb3d_batch_create(arr, len(jobs), err, len(err))
        if not self.h:
            raise Error(err.value.decode())
        self._filters = [f for f, _, _ in jobs]  # the filters outlive the batch

    def launch(self, stream: int = 0):
        err = N.err_buf()
        if N.lib().zb3d_batch_launch(self.h, stream or None, err, len(err)) != 0:
            raise Error(err.value.decode())

    def status(self):
        err = N.err_buf()
        if N.lib().zb3d_batch_status(self.h, err, len(err)) != 0:
            raise Error(err.value.decode())

    def close(self):
        if self.h:
            N.lib().zb3d_batch_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
