"""Build the reference BM3D kernels into ``oracle/_ref/``.  TEST INFRASTRUCTURE ONLY.

Recipe: the reference's own sources are read where they lie (``src/bm3d.cu`` and
``src/bm3d_vagg.cu`` under the mounted reference tree), prefixed with the
reference's ``#define`` block, and compiled with NVRTC using the reference's own
options (vszipcu src/bm3d.zig:20-31, cudaz/src/nvrtc.zig:137-211):

    bm3d.cu       -arch=sm_100 -use_fast_math -std=c++17 -modify-stack-limit=false
    bm3d_vagg.cu  -arch=sm_100 -std=c++17 -modify-stack-limit=false

For the match-index pins a second variant stores the final match list of each
reference block: a copy of ``bm3d.cu`` written into ``oracle/_ref/gen/`` (never
into the reference tree) gets ``__device__`` dump pointers (indices, and optionally
the list's distances) and one store block inserted right after the self-inclusion
step (src/bm3d.cu:788).

Outputs go only to ``oracle/_ref/`` (git-ignored; it travels with the tree to the
GPU machine, where the reference sources do not exist).
"""
from __future__ import annotations

import ctypes
import os
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import ref_configs as rc  # noqa: E402

# the reference source tree (its src/bm3d.cu); there is no default location
REF_ROOT = os.environ.get("ZB3D_REFERENCE_ROOT", "")
OUT = os.path.join(HERE, "_ref")
GEN = os.path.join(OUT, "gen")

_DUMP_DECL = "\n#ifdef ZB_REF_DUMP\n__device__ int *zb_ref_dump;\n__device__ float *zb_ref_dump_err;\n#endif\n"
_DUMP_STORE = """
#ifdef ZB_REF_DUMP
    {
        const int zb_bx = 4 * gid + lane_id / 8;
        const long long zb_slot = ((long long)blockIdx.y * ZB_REF_NBX + zb_bx) * 8 + sub_lane_id;
        int *zb_p = zb_ref_dump + zb_slot * 3;
        zb_p[0] = index8_x;
        zb_p[1] = index8_y;
        zb_p[2] = index8_z;
        if (zb_ref_dump_err) zb_ref_dump_err[zb_slot] = errors8;
    }
#endif
"""
_ANCHOR = "    float denoising_patch[64];"


def _nvrtc():
    for name in ("libnvrtc.so.12", "libnvrtc.so"):
        for d in ("/usr/local/cuda/lib64", ""):
            try:
                return ctypes.CDLL(os.path.join(d, name) if d else name)
            except OSError:
                continue
    raise RuntimeError("NVRTC not found")


def nvrtc_compile(src: str, name: str, opts: list[str]) -> bytes:
    lib = _nvrtc()
    prog = ctypes.c_void_p()
    r = lib.nvrtcCreateProgram(ctypes.byref(prog), src.encode(), name.encode(), 0, None, None)
    if r != 0:
        raise RuntimeError(f"nvrtcCreateProgram failed: {r}")
    try:
        arr = (ctypes.c_char_p * len(opts))(*[o.encode() for o in opts])
        r = lib.nvrtcCompileProgram(prog, len(opts), arr)
        if r != 0:
            n = ctypes.c_size_t()
            lib.nvrtcGetProgramLogSize(prog, ctypes.byref(n))
            buf = ctypes.create_string_buffer(n.value)
            lib.nvrtcGetProgramLog(prog, buf)
            raise RuntimeError(f"{name}: NVRTC compile failed:\n{buf.value.decode(errors='replace')}")
        n = ctypes.c_size_t()
        lib.nvrtcGetCUBINSize(prog, ctypes.byref(n))
        buf = ctypes.create_string_buffer(n.value)
        lib.nvrtcGetCUBIN(prog, buf)
        return buf.raw
    finally:
        lib.nvrtcDestroyProgram(ctypes.byref(prog))


def _bm3d_source(dump: bool) -> str:
    with open(os.path.join(REF_ROOT, "src", "bm3d.cu")) as f:
        text = f.read()
    if not dump:
        return text
    if _ANCHOR not in text:
        raise RuntimeError("dump anchor not found in the reference bm3d.cu")
    text = text.replace(_ANCHOR, _DUMP_STORE + _ANCHOR, 1)
    return _DUMP_DECL + text


BM3D_OPTS = ["-arch=sm_100", "-use_fast_math", "-std=c++17", "-modify-stack-limit=false"]
VAGG_OPTS = ["-arch=sm_100", "-std=c++17", "-modify-stack-limit=false"]


def build(force: bool = False, jobs: int = 8, verbose: bool = True) -> int:
    if not REF_ROOT:
        raise RuntimeError("build_ref: set ZB3D_REFERENCE_ROOT to the reference source tree (the directory "
                           "holding src/bm3d.cu)")
    if not os.path.isfile(os.path.join(REF_ROOT, "src", "bm3d.cu")):
        if verbose:
            print(f"build_ref: reference sources not found under {REF_ROOT}; skipped")
        return 0
    os.makedirs(GEN, exist_ok=True)
    srcs = {False: _bm3d_source(False), True: _bm3d_source(True)}
    with open(os.path.join(GEN, "bm3d_dump.cu"), "w") as f:
        f.write(srcs[True])
    with open(os.path.join(REF_ROOT, "src", "bm3d_vagg.cu")) as f:
        vsrc = f.read()
    todo = []
    for s in rc.all_specs():
        for dump in (False, True):
            path = os.path.join(OUT, rc.cubin_name(s, dump))
            if force or not os.path.exists(path):
                todo.append((rc.define_block(s, dump) + srcs[dump], "bm3d.cu", BM3D_OPTS, path))
    for v in rc.vagg_specs():
        path = os.path.join(OUT, rc.vagg_cubin_name(*v))
        if force or not os.path.exists(path):
            todo.append((rc.vagg_define_block(*v) + vsrc, "bm3d_vagg.cu", VAGG_OPTS, path))

    def one(job):
        src, name, opts, path = job
        img = nvrtc_compile(src, name, opts)
        tmp = path + ".tmp"
        with open(tmp, "wb") as f:
            f.write(img)
        os.replace(tmp, path)
        return path

    with ThreadPoolExecutor(max_workers=jobs) as ex:
        for p in ex.map(one, todo):
            if verbose:
                print("built", os.path.relpath(p, HERE))
    return len(todo)


if __name__ == "__main__":
    n = build(force="--force" in sys.argv)
    print(f"build_ref: {n} cubins compiled")
