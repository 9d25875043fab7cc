"""ctypes front end of the CPU oracle (``liboracle.so``).  TEST INFRASTRUCTURE ONLY.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline and
reference arms import this module.  See bm3d_oracle.c for what it restates.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BM = {"ssd": 0, "sad": 1, "zssd": 2, "zsad": 3, "ssd_norm": 4, "ssd/norm": 4}
TR = {"dct": 0, "haar": 1, "wht": 2, "bior1_5": 3, "bior1.5": 3}


class OcCfg(ctypes.Structure):
    _fields_ = [
        ("w", ctypes.c_int), ("h", ctypes.c_int), ("stride", ctypes.c_int),
        ("nplanes", ctypes.c_int), ("radius", ctypes.c_int), ("final_", ctypes.c_int),
        ("chroma", ctypes.c_int), ("sigma", ctypes.c_float * 3),
        ("bs", ctypes.c_int), ("range", ctypes.c_int), ("ps_num", ctypes.c_int), ("ps_range", ctypes.c_int),
        ("bm_error", ctypes.c_int), ("t2d", ctypes.c_int), ("t1d", ctypes.c_int),
        ("nthreads", ctypes.c_int), ("extractor", ctypes.c_float),
    ]


_lib = None


def build() -> str:
    path = os.path.join(HERE, "liboracle.so")
    src = os.path.join(HERE, "bm3d_oracle.c")
    if not os.path.exists(path) or os.path.getmtime(path) < os.path.getmtime(src):
        subprocess.check_call(["make", "-s", "-C", HERE, "liboracle.so"])
    return path


def lib():
    global _lib
    if _lib is None:
        _lib = ctypes.CDLL(build())
        _lib.oracle_bm3d_pass.restype = ctypes.c_int
        _lib.oracle_match.restype = ctypes.c_int
        _lib.oracle_distance.restype = ctypes.c_float
        _lib.oracle_agg_z.restype = ctypes.c_int
    return _lib


def make_cfg(w, h, stride, sigma_scaled, block_step=8, bm_range=9, radius=0, ps_num=2, ps_range=4,
             chroma=0, final=0, bm_error="ssd", t2d="dct", t1d="dct", nthreads=None,
             extractor_exp=0) -> OcCfg:
    c = OcCfg()
    c.w, c.h, c.stride = w, h, stride
    c.nplanes = 3 if chroma else 1
    c.radius, c.final_, c.chroma = radius, int(final), int(chroma)
    s = list(sigma_scaled) + [sigma_scaled[-1]] * (3 - len(sigma_scaled))
    for i in range(3):
        c.sigma[i] = s[i]
    c.bs, c.range, c.ps_num, c.ps_range = block_step, bm_range, ps_num, ps_range
    c.bm_error, c.t2d, c.t1d = BM[bm_error], TR[t2d], TR[t1d]
    c.nthreads = nthreads or os.cpu_count() or 1
    c.extractor = 0.0 if extractor_exp == 0 else 2.0 ** extractor_exp
    return c


def _ptrs(planes):
    arrs = [np.ascontiguousarray(p, dtype=np.float32) for p in planes]
    arr = (ctypes.c_void_p * len(arrs))(*[a.ctypes.data for a in arrs])
    return arr, arrs


def bm3d_pass(cfg: OcCfg, src: np.ndarray, want_matches: bool = True):
    """src: float32 [clips][planes][tw][h][stride].  Returns (num, den, matches):
    num/den FP64 [planes][tw][h][w], matches int32 [nby][nbx][8][3] (x, y, z)."""
    tw = 2 * cfg.radius + 1
    nclips = 2 if cfg.final_ else 1
    assert src.shape == (nclips, cfg.nplanes, tw, cfg.h, cfg.stride), src.shape
    planes = [src[c, p, t] for c in range(nclips) for p in range(cfg.nplanes) for t in range(tw)]
    arr, keep = _ptrs(planes)
    num = np.zeros((cfg.nplanes, tw, cfg.h, cfg.w), np.float64)
    den = np.zeros_like(num)
    nbx = (cfg.w - 8 + cfg.bs - 1) // cfg.bs + 1
    nby = (cfg.h - 8 + cfg.bs - 1) // cfg.bs + 1
    m = np.zeros((nby, nbx, 8, 3), np.int32) if want_matches else None
    r = lib().oracle_bm3d_pass(ctypes.byref(cfg), arr, num.ctypes.data_as(ctypes.c_void_p),
                               den.ctypes.data_as(ctypes.c_void_p),
                               m.ctypes.data_as(ctypes.c_void_p) if m is not None else None)
    if r < 0:
        raise MemoryError("oracle_bm3d_pass")
    del keep
    return num, den, m


def match(cfg: OcCfg, mplanes) -> np.ndarray:
    """Match lists only (FP32 exact order); mplanes = tw matching planes [h][stride]."""
    arr, keep = _ptrs(mplanes)
    nbx = (cfg.w - 8 + cfg.bs - 1) // cfg.bs + 1
    nby = (cfg.h - 8 + cfg.bs - 1) // cfg.bs + 1
    m = np.zeros((nby, nbx, 8, 3), np.int32)
    lib().oracle_match(ctypes.byref(cfg), arr, m.ctypes.data_as(ctypes.c_void_p))
    del keep
    return m


def distance(metric: str, a: np.ndarray, b: np.ndarray) -> float:
    a = np.ascontiguousarray(a, np.float32)
    b = np.ascontiguousarray(b, np.float32)
    return lib().oracle_distance(BM[metric], a.ctypes.data_as(ctypes.c_void_p),
                                 b.ctypes.data_as(ctypes.c_void_p), a.shape[1])


def agg_z(i: int, n: int, nframes: int, radius: int) -> int:
    return lib().oracle_agg_z(i, n, nframes, radius)


def vaggregate_plane(stacks, w, h, stride, radius, n, nframes) -> np.ndarray:
    """VAggregate of one plane: stacks[i] = stacked accumulator plane of frame
    clamp(n-r+i), float32 [2*tw*h][stride]."""
    arr, keep = _ptrs(stacks)
    dst = np.zeros((h, stride), np.float32)
    lib().oracle_vaggregate_plane(dst.ctypes.data_as(ctypes.c_void_p), arr, w, h, stride, radius, n, nframes)
    del keep
    return dst


def finish(num: np.ndarray, den: np.ndarray) -> np.ndarray:
    """num/den of the centre slot in FP64 (radius 0 output)."""
    with np.errstate(invalid="ignore", divide="ignore"):
        return num / den
