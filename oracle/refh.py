"""Front end of the reference-kernel harness.  TEST INFRASTRUCTURE ONLY.

Runs the reference's own BM3D kernels (compiled by ``oracle/build_ref.py`` from
vszipcu src/bm3d.cu into ``oracle/_ref/*.cubin``) on the GPU, on torch-owned
device memory, replaying the reference host's launch sequence
(src/bm3d.zig:375-401 and :589-630).
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")

import sys  # noqa: E402
sys.path.insert(0, HERE)
import ref_configs as rc  # noqa: E402

_lib = None


def available() -> bool:
    return os.path.exists(os.path.join(REF_DIR, "libzb3d_refh.so"))


def lib():
    global _lib
    if _lib is None:
        _lib = ctypes.CDLL(os.path.join(REF_DIR, "libzb3d_refh.so"))
        _lib.refh_load.restype = ctypes.c_void_p
        _lib.refh_load.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int]
        _lib.refh_unload.argtypes = [ctypes.c_void_p]
        _lib.refh_set_dump.argtypes = [ctypes.c_void_p, ctypes.c_ulonglong, ctypes.c_char_p, ctypes.c_int]
        _lib.refh_set_dump_err.argtypes = [ctypes.c_void_p, ctypes.c_ulonglong, ctypes.c_char_p, ctypes.c_int]
        _lib.refh_bm3d.argtypes = [ctypes.c_void_p, ctypes.c_ulonglong, ctypes.c_ulonglong, ctypes.c_ulonglong,
                                   ctypes.c_size_t, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                   ctypes.c_int, ctypes.c_ulonglong, ctypes.c_char_p, ctypes.c_int]
        _lib.refh_vagg.argtypes = [ctypes.c_void_p, ctypes.c_ulonglong, ctypes.POINTER(ctypes.c_ulonglong),
                                   ctypes.POINTER(ctypes.c_int), ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                   ctypes.c_int, ctypes.c_ulonglong, ctypes.c_char_p, ctypes.c_int]
    return _lib


def cubin_path(spec, dump=False) -> str:
    return os.path.join(REF_DIR, rc.cubin_name(spec, dump))


def has_cubin(spec, dump=False) -> bool:
    return os.path.exists(cubin_path(spec, dump))


class RefKernel:
    """One loaded reference specialisation."""

    def __init__(self, spec, dump=False, path=None):
        self.spec = spec
        self.dump = dump
        err = ctypes.create_string_buffer(512)
        p = path or cubin_path(spec, dump)
        self.h = lib().refh_load(p.encode(), err, 512)
        if not self.h:
            raise RuntimeError(f"reference kernel load failed ({p}): {err.value.decode()}")

    def close(self):
        if self.h:
            lib().refh_unload(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_dump(self, dptr: int):
        err = ctypes.create_string_buffer(512)
        if lib().refh_set_dump(self.h, dptr, err, 512):
            raise RuntimeError(err.value.decode())

    def set_dump_err(self, dptr: int):
        """Also store each list slot's distance (float[nby][nbx][8]); 0 turns it off."""
        err = ctypes.create_string_buffer(512)
        if lib().refh_set_dump_err(self.h, dptr, err, 512):
            raise RuntimeError(err.value.decode())

    def run(self, res_ptr: int, src_ptr: int, dst_ptr: int, res_bytes: int, stream: int = 0):
        s = self.spec
        err = ctypes.create_string_buffer(512)
        agg_planes = 3 if s.chroma else 1
        r = lib().refh_bm3d(self.h, res_ptr, src_ptr, dst_ptr, res_bytes, s.w, s.h, s.block_step, s.warps,
                            agg_planes, stream, err, 512)
        if r:
            raise RuntimeError(err.value.decode())


class RefVagg:
    def __init__(self, w, h, stride, radius, proc_mask):
        err = ctypes.create_string_buffer(512)
        p = os.path.join(REF_DIR, rc.vagg_cubin_name(w, h, stride, radius, proc_mask))
        self.w, self.hgt, self.radius = w, h, radius
        self.h = lib().refh_load(p.encode(), err, 512)
        if not self.h:
            raise RuntimeError(f"reference vaggregate load failed ({p}): {err.value.decode()}")

    def run(self, dst_ptr: int, ptrs, zs, nplanes: int, stream: int = 0):
        tw = len(ptrs)
        P = (ctypes.c_ulonglong * tw)(*ptrs)
        Z = (ctypes.c_int * tw)(*zs)
        err = ctypes.create_string_buffer(512)
        r = lib().refh_vagg(self.h, dst_ptr, P, Z, tw, self.w, self.hgt, nplanes, stream, err, 512)
        if r:
            raise RuntimeError(err.value.decode())

    def close(self):
        if self.h:
            lib().refh_unload(self.h)
            self.h = None
