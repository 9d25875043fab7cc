"""ctypes binding of libzb3d.so (include/zb3d.h).

The library is built in-tree next to this file (``python -m zb3d.build``).  There
is no fallback: if it is missing or fails to load, import-time use raises.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libzb3d.so")

UNSET = -2147483647 - 1
GRAY, RGB, YUV = 1, 2, 3
INTEGER, FLOAT = 0, 1

c_int, c_float, c_size_t, c_void_p, c_char_p = ctypes.c_int, ctypes.c_float, ctypes.c_size_t, ctypes.c_void_p, ctypes.c_char_p


class VideoInfo(ctypes.Structure):
    _fields_ = [("color_family", c_int), ("sample_type", c_int), ("bits_per_sample", c_int),
                ("subsampling_w", c_int), ("subsampling_h", c_int), ("num_planes", c_int),
                ("width", c_int), ("height", c_int), ("num_frames", c_int)]


class Args(ctypes.Structure):
    _fields_ = [
        ("ref", ctypes.POINTER(VideoInfo)),
        ("sigma", ctypes.POINTER(c_float)), ("n_sigma", c_int),
        ("block_step", ctypes.POINTER(c_int)), ("n_block_step", c_int),
        ("bm_range", ctypes.POINTER(c_int)), ("n_bm_range", c_int),
        ("radius", c_int),
        ("ps_num", ctypes.POINTER(c_int)), ("n_ps_num", c_int),
        ("ps_range", ctypes.POINTER(c_int)), ("n_ps_range", c_int),
        ("chroma", c_int), ("device_id", c_int), ("num_streams", c_int), ("extractor_exp", c_int),
        ("bm_error_s", ctypes.POINTER(c_char_p)), ("n_bm_error_s", c_int),
        ("transform_2d_s", ctypes.POINTER(c_char_p)), ("n_transform_2d_s", c_int),
        ("transform_1d_s", ctypes.POINTER(c_char_p)), ("n_transform_1d_s", c_int),
        ("zero_init", c_int), ("fast_fused", c_int), ("match_form", c_int),
        ("pilot", c_void_p), ("filter_form", c_int),
    ]


class Frame(ctypes.Structure):
    _fields_ = [("ptr", c_void_p * 3), ("stride", ctypes.c_ssize_t * 3)]


class FrameOut(ctypes.Structure):
    _fields_ = [("ptr", c_void_p * 3), ("stride", ctypes.c_ssize_t * 3)]


class BatchJob(ctypes.Structure):
    _fields_ = [("filter", c_void_p), ("d_src", c_void_p), ("d_dst", c_void_p)]


class EntryLayout(ctypes.Structure):
    _fields_ = [("nplanes", c_int), ("plane", c_int * 3), ("width", c_int), ("height", c_int), ("pitch", c_int),
                ("tw", c_int), ("nclips", c_int), ("src_offset", c_size_t), ("src_elems", c_size_t),
                ("dst_offset", c_size_t), ("dst_elems", c_size_t)]


EXPORTS = {
    "zb3d_args_init": (None, [ctypes.POINTER(Args)]),
    "zb3d_create": (c_void_p, [ctypes.POINTER(VideoInfo), ctypes.POINTER(Args), c_int, c_char_p, c_size_t]),
    "zb3d_output_info": (None, [c_void_p, ctypes.POINTER(VideoInfo)]),
    "zb3d_frame_range": (None, [c_void_p, c_int, ctypes.POINTER(c_int), ctypes.POINTER(c_int)]),
    "zb3d_output_props": (None, [c_void_p, ctypes.POINTER(c_int), ctypes.POINTER(c_int)]),
    "zb3d_get_frame": (c_int, [c_void_p, c_int, ctypes.POINTER(Frame), ctypes.POINTER(Frame),
                               ctypes.POINTER(FrameOut), c_char_p, c_size_t]),
    "zb3d_free": (None, [c_void_p]),
    "zb3d_num_entries": (c_int, [c_void_p]),
    "zb3d_entry_layout_get": (c_int, [c_void_p, c_int, ctypes.POINTER(EntryLayout)]),
    "zb3d_src_elems": (c_size_t, [c_void_p]),
    "zb3d_dst_elems": (c_size_t, [c_void_p]),
    "zb3d_process_device": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_char_p, c_size_t]),
    "zb3d_process_entry_device": (c_int, [c_void_p, c_int, c_void_p, c_void_p, c_void_p, c_char_p, c_size_t]),
    "zb3d_profile_enable": (None, [c_void_p, c_int]),
    "zb3d_profile_collect": (c_int, [c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(c_int),
                                     ctypes.POINTER(ctypes.c_double), ctypes.POINTER(c_int)]),
    "zb3d_bm3d_plane_noalloc": (c_int, [c_void_p, c_void_p, c_int, c_int, c_int, c_int, c_float, c_int, c_int,
                                        c_int, c_void_p, c_char_p, c_size_t]),
    "zb3d_match_device": (c_int, [c_void_p, c_int, c_void_p, c_void_p, c_void_p, c_char_p, c_size_t]),
    "zb3d_match_stats": (c_int, [c_void_p, ctypes.POINTER(ctypes.c_ulonglong), c_int]),
    "zb3d_entry_tuning": (c_int, [c_void_p, c_int, ctypes.POINTER(c_int), ctypes.POINTER(c_int)]),
    "zb3d_tc_probe_cols": (c_int, [c_int, c_int, c_int, c_int]),
    "zb3d_tc_probe": (c_int, [c_void_p, c_int, c_int, c_int, c_int, c_int, c_void_p, c_void_p, c_void_p,
                              ctypes.POINTER(ctypes.c_ulonglong), c_char_p, c_size_t]),
    "zb3d_vaggregate_device": (c_int, [ctypes.POINTER(c_void_p), ctypes.POINTER(c_int), c_int, c_int, c_int,
                                       c_int, c_int, ctypes.c_uint, c_void_p, c_void_p]),
    "zb3d_vaggregate_create": (c_void_p, [ctypes.POINTER(VideoInfo), ctypes.POINTER(VideoInfo),
                                          ctypes.POINTER(c_int), c_int, c_char_p, c_size_t]),
    "zb3d_vaggregate_output_info": (None, [c_void_p, ctypes.POINTER(VideoInfo)]),
    "zb3d_vaggregate_frame_range": (None, [c_void_p, c_int, ctypes.POINTER(c_int), ctypes.POINTER(c_int)]),
    "zb3d_vaggregate_get_frame": (c_int, [c_void_p, c_int, ctypes.POINTER(Frame), ctypes.POINTER(FrameOut),
                                          c_char_p, c_size_t]),
    "zb3d_vaggregate_free": (None, [c_void_p]),
    "zb3d_agg_z": (c_int, [c_int, c_int, c_int, c_int]),
    "zb3d_version": (c_char_p, []),
    "zb3d_pilot_conv3x3": (c_int, [c_void_p, c_int, c_int, c_int, c_int, c_void_p, c_void_p, c_int, c_int,
                                   c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    "zb3d_pilot_conv3x3_tc": (c_int, [c_void_p, c_int, c_int, c_int, c_int, c_void_p, c_void_p, c_int, c_int,
                                      c_void_p, c_void_p, c_void_p, ctypes.c_longlong, ctypes.c_longlong, c_void_p,
                                      c_void_p]),
    "zb3d_pilot_tc_ctas_per_sm": (c_int, [c_int]),
    "zb3d_dct2d_tf32": (c_int, [c_void_p, c_void_p, ctypes.c_longlong, c_int, c_void_p, c_void_p]),
    "zb3d_pilot_pack_input_blocked": (c_int, [c_void_p, ctypes.c_longlong, c_void_p, c_int, c_int, c_int, c_float,
                                              c_void_p, c_void_p]),
    "zb3d_pilot_conv3x3_wgrad": (c_int, [c_void_p, c_void_p, c_int, c_int, c_int, c_int, c_int, c_void_p,
                                         c_void_p, c_void_p]),
    "zb3d_pilot_pack_input": (c_int, [c_void_p, c_void_p, c_int, c_int, c_int, c_float, c_void_p, c_void_p]),
    "zb3d_pilot_mse_grad": (c_int, [c_void_p, c_void_p, ctypes.c_longlong, c_float, c_void_p, c_void_p, c_void_p]),
    "zb3d_pilot_adam": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, ctypes.c_longlong, c_float, c_float, c_float,
                                c_float, c_int, c_float, c_void_p, c_void_p, c_void_p]),
    "zb3d_pilot_flip_weights": (c_int, [c_void_p, c_int, c_int, c_void_p, c_void_p]),
    "zb3d_pilot_to_bf16": (c_int, [c_void_p, ctypes.c_longlong, c_void_p, c_void_p]),
    "zb3d_pilot_load": (c_void_p, [c_char_p, c_int, c_char_p, c_size_t]),
    "zb3d_pilot_from_memory": (c_void_p, [c_void_p, c_size_t, c_int, c_char_p, c_size_t]),
    "zb3d_pilot_free": (None, [c_void_p]),
    "zb3d_pilot_describe": (None, [c_void_p, ctypes.POINTER(c_int), ctypes.POINTER(c_int), ctypes.POINTER(c_int)]),
    "zb3d_pilot_gate_level": (c_int, [c_void_p, c_int, ctypes.POINTER(c_float), ctypes.POINTER(c_int),
                                      ctypes.POINTER(c_int), ctypes.POINTER(c_float)]),
    "zb3d_pilot_accepts": (c_int, [c_void_p, c_float, c_int, c_int]),
    "zb3d_pilot_workspace_bytes": (c_size_t, [c_void_p, c_int, c_int]),
    "zb3d_pilot_run": (c_int, [c_void_p, c_void_p, c_int, c_int, c_int, c_float, c_void_p, c_int, c_void_p,
                               c_void_p, c_void_p]),
    "zb3d_process_batch": (c_int, [c_void_p, c_int, c_void_p, c_char_p, c_size_t]),
    "zb3d_process_batch_ex": (c_int, [c_void_p, c_int, c_void_p, ctypes.c_uint, c_int, c_char_p, c_size_t]),
    "zb3d_batch_create": (c_void_p, [c_void_p, c_int, c_char_p, c_size_t]),
    "zb3d_batch_launch": (c_int, [c_void_p, c_void_p, c_char_p, c_size_t]),
    "zb3d_batch_status": (c_int, [c_void_p, c_char_p, c_size_t]),
    "zb3d_batch_free": (None, [c_void_p]),
    "zb3d_host_alloc": (c_void_p, [c_size_t]),
    "zb3d_host_free": (None, [c_void_p]),
}

_lib = None


def lib() -> ctypes.CDLL:
    """The loaded native library; raises if it was not built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"zb3d: native library missing ({LIB_PATH}); build it with `python -m zb3d.build`")
        l = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in EXPORTS.items():
            fn = getattr(l, name)
            fn.restype = res
            fn.argtypes = args
        _lib = l
    return _lib


def err_buf():
    return ctypes.create_string_buffer(1024)
