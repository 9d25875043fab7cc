"""Build recipe of libzb3d.so (sm_100a), in-tree next to this file.

    python -m zb3d.build        (from vapoursynth-zipcu_b200/)

zb3d_kernels.cu and zb3d_match_tc.cu are compiled with -use_fast_math (the
reference kernel's floating-point mode), zb3d_vagg.cu without it (IEEE sums and division, no
flush-to-zero), the host in C++17; nvcc links them into one shared library.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(os.path.dirname(PKG), "include")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(HERE, "libzb3d.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", f"-I{INCLUDE}", f"-I{CSRC}"]

UNITS = [
    ("zb3d_kernels.cu", ARCH + ["-use_fast_math"]),
    ("zb3d_match_tc.cu", ARCH + ["-use_fast_math"]),
    ("zb3d_vagg.cu", ARCH),
    ("zb3d_pilot.cu", ARCH),
    ("zb3d_pilot_tc.cu", ARCH),
    ("zb3d_dct_tc.cu", ARCH),
    ("zb3d_filter_tc.cu", ARCH),
    ("zb3d_host.cpp", ARCH),
    ("zb3d_pilot_net.cpp", ARCH),
    ("zb3d_noalloc.cu", ARCH),
]
HEADERS = ["zb3d_args.h", "zb3d_match.cuh", "zb3d_transforms.cuh", "zb3d_tcgen05.cuh"]


def _stale(out, deps):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, ptxas_info: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(INCLUDE, "zb3d.h")]
    objs = []
    procs = []
    for src, flags in UNITS:
        path = os.path.join(CSRC, src)
        obj = os.path.join(BUILD, src + ".o")
        objs.append(obj)
        if _stale(obj, [path] + hdrs) or ptxas_info:
            cmd = [NVCC] + COMMON + flags + (["-Xptxas", "-v"] if ptxas_info and src.endswith(".cu") else [])
            cmd += ["-c", path, "-o", obj]
            if verbose:
                print(" ".join(cmd))
            procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)))
    for src, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src}:\n{out}")
        if out and (verbose or ptxas_info):
            print(out)
    if _stale(LIB, objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
        if verbose:
            print(" ".join(cmd))
        subprocess.check_call(cmd)
    return LIB


if __name__ == "__main__":
    print(build(verbose=True, ptxas_info="--ptxas" in sys.argv))
