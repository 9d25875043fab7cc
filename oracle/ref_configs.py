"""Specialisations of the reference BM3D kernel that the GPU parity tests and the
bench run.  TEST INFRASTRUCTURE ONLY.

The reference compiles one kernel per filter configuration: every size, sigma and
option is a ``#define`` baked in by NVRTC (vszipcu src/bm3d.zig:793-823, floats
printed as hexfloat).  ``define_block`` reproduces that block byte for byte in
meaning, ``cubin_name`` names the cubin that ``oracle/build_ref.py`` writes for it
into ``oracle/_ref/``.
"""
from __future__ import annotations

import hashlib
import struct
from dataclasses import dataclass, field, asdict

BM_ERRORS = ("ssd", "sad", "zssd", "zsad", "ssd_norm")
TRANSFORMS = ("dct", "haar", "wht", "bior1_5")

# f32(2.7 * 0.75 * 64 / 255) and f32(0.75 * 64 / 255) exactly as the reference
# host stores them (src/bm3d.zig:1020-1023).
HARD_FACTOR_BITS = 0x3F021BB6
WIENER_FACTOR_BITS = 0x3E40C0C1


def f32(x: float) -> float:
    return struct.unpack("<f", struct.pack("<f", x))[0]


def f32_from_bits(b: int) -> float:
    return struct.unpack("<f", struct.pack("<I", b))[0]


def scaled_sigma(sigma: float, final: bool) -> float:
    """sigma * factor in f32 (src/bm3d.zig:1019-1024)."""
    fac = f32_from_bits(WIENER_FACTOR_BITS if final else HARD_FACTOR_BITS)
    return f32(f32(sigma) * fac)


def hexf(x: float) -> str:
    return float.hex(f32(x)) + "f"


@dataclass(frozen=True)
class RefSpec:
    """One reference kernel specialisation (the ModKey plus the per-filter defines)."""
    w: int
    h: int
    stride: int
    sigma: tuple = (3.0, 3.0, 3.0)      # unscaled, 8-bit scale
    block_step: int = 8
    bm_range: int = 9
    radius: int = 0
    ps_num: int = 2
    ps_range: int = 4
    chroma: int = 0
    final: int = 0
    extractor_exp: int = 3
    proc_mask: int = 1
    bm_error: str = "ssd"
    t2d: str = "dct"
    t1d: str = "dct"
    warps: int = 2

    def scaled(self):
        return tuple(scaled_sigma(s, bool(self.final)) for s in self.sigma)

    def extractor(self) -> float:
        return 0.0 if self.extractor_exp == 0 else 2.0 ** self.extractor_exp

    def nbx(self) -> int:
        return (self.w - 8 + self.block_step - 1) // self.block_step + 1

    def nby(self) -> int:
        return (self.h - 8 + self.block_step - 1) // self.block_step + 1


def define_block(s: RefSpec, dump: bool = False) -> str:
    sy, su, sv = s.scaled()
    lines = [
        f"#define WIDTH {s.w}",
        f"#define HEIGHT {s.h}",
        f"#define STRIDE {s.stride}",
        f"#define SIGMA_Y {hexf(sy)}",
        f"#define SIGMA_U {hexf(su)}",
        f"#define SIGMA_V {hexf(sv)}",
        f"#define BLOCK_STEP {s.block_step}",
        f"#define BM_RANGE {s.bm_range}",
        f"#define RADIUS {s.radius}",
        f"#define PS_NUM {s.ps_num}",
        f"#define PS_RANGE {s.ps_range}",
        f"#define TEMPORAL {1 if s.radius > 0 else 0}",
        f"#define CHROMA {s.chroma}",
        f"#define FINAL {s.final}",
        f"#define EXTRACTOR {hexf(s.extractor())}",
        f"#define WARPS {s.warps}",
        f"#define PROC_MASK {s.proc_mask}",
        f"#define BM_ERROR {s.bm_error}",
        f"#define TRANSFORM_2D {s.t2d}",
        f"#define TRANSFORM_1D {s.t1d}",
    ]
    if dump:
        lines.append("#define ZB_REF_DUMP 1")
        lines.append(f"#define ZB_REF_NBX {s.nbx()}")
    return "\n".join(lines) + "\n"


def vagg_define_block(w: int, h: int, stride: int, radius: int, proc_mask: int) -> str:
    return (f"#define WIDTH {w}\n#define HEIGHT {h}\n#define STRIDE {stride}\n"
            f"#define RADIUS {radius}\n#define PROC_MASK {proc_mask}\n")


def cubin_name(s: RefSpec, dump: bool = False) -> str:
    key = hashlib.sha1(define_block(s, dump).encode()).hexdigest()[:16]
    return f"bm3d_{'dump_' if dump else ''}{key}.cubin"


def vagg_cubin_name(w: int, h: int, stride: int, radius: int, proc_mask: int) -> str:
    key = hashlib.sha1(vagg_define_block(w, h, stride, radius, proc_mask).encode()).hexdigest()[:16]
    return f"vagg_{key}.cubin"


def pitch_for(w: int) -> int:
    """Row pitch (elements) used by the tests: 64-byte rows like a VapourSynth frame."""
    return (w + 15) // 16 * 16


# --------------------------------------------------------------------------
# The cases.  Small ones are also run by the CPU oracle in seconds.
# --------------------------------------------------------------------------
def _small(**kw):
    base = dict(w=72, h=56, stride=pitch_for(72))
    base.update(kw)
    return RefSpec(**base)


def parity_specs():
    specs = []
    # spatial, default-ish parameters, basic and final
    for final in (0, 1):
        specs.append(_small(final=final, sigma=(10.0,) * 3))
        specs.append(_small(w=77, h=53, stride=pitch_for(77), block_step=4, bm_range=12,
                            final=final, sigma=(10.0,) * 3))
    # generic block steps, tiny frames, non-deterministic extractor
    for bs in (1, 2, 3, 5, 6, 7):
        specs.append(_small(w=45, h=37, stride=pitch_for(45), block_step=bs, bm_range=5))
    specs.append(_small(w=8, h=8, stride=16))
    specs.append(_small(w=9, h=17, stride=16, block_step=4))
    specs.append(_small(w=20, h=12, stride=32, block_step=8, bm_range=3))
    specs.append(_small(extractor_exp=0))
    # distance metrics and transforms
    for m in BM_ERRORS[1:]:
        specs.append(_small(bm_error=m))
    for t in TRANSFORMS[1:]:
        specs.append(_small(t2d=t, t1d=t))
        specs.append(_small(t2d=t, t1d=t, final=1))
    # temporal (the window frames are passed explicitly)
    for r in (1, 2):
        for final in (0, 1):
            specs.append(_small(w=64, h=48, stride=64, radius=r, final=final, sigma=(15.0,) * 3))
    specs.append(_small(w=64, h=48, stride=64, radius=1, block_step=4, bm_range=6, ps_num=3, ps_range=2))
    # CBM3D (YUV444, matching on Y)
    for final in (0, 1):
        specs.append(_small(w=48, h=40, stride=48, chroma=1, proc_mask=7, final=final,
                            sigma=(8.0, 6.0, 6.0)))
    specs.append(_small(w=48, h=40, stride=48, chroma=1, proc_mask=5, sigma=(8.0, 0.0, 6.0)))
    specs.append(_small(w=48, h=40, stride=48, chroma=1, proc_mask=7, radius=1, sigma=(8.0, 6.0, 6.0)))
    # ssd/norm on more blocks: approximate square root and reciprocal in both kernels
    specs.append(_small(w=256, h=192, stride=256, block_step=4, bm_range=12, bm_error="ssd_norm", sigma=(10.0,) * 3))
    specs.append(_small(w=200, h=150, stride=224, block_step=8, bm_range=9, bm_error="ssd_norm", final=1))
    return specs


def workload_specs():
    """Full-size workloads: 640x480 (sigma 3, bs 8) and the 1080p YUV420 two-pass job."""
    out = []
    out.append(RefSpec(w=640, h=480, stride=640, sigma=(3.0,) * 3, block_step=8, bm_range=9))
    for final in (0, 1):
        out.append(RefSpec(w=1920, h=1080, stride=1920, sigma=(10.0,) * 3, block_step=4, bm_range=12, final=final))
        out.append(RefSpec(w=960, h=540, stride=960, sigma=(10.0,) * 3, block_step=4, bm_range=12, final=final))
    # 1080p VBM3D radius 2 (fused), sigma 15, default block_step / range
    out.append(RefSpec(w=1920, h=1080, stride=1920, sigma=(15.0,) * 3, radius=2))
    return out


def api_specs():
    """Whole-plane cases of the public-API tests (YUV420 two-pass planes)."""
    out = []
    for final in (0, 1):
        for (w, h) in ((96, 64), (48, 32)):
            out.append(RefSpec(w=w, h=h, stride=w, sigma=(10.0,) * 3, block_step=4, bm_range=12, final=final))
    return out


def vagg_specs():
    out = []
    for s in parity_specs() + workload_specs():
        if s.radius > 0:
            out.append((s.w, s.h, s.stride, s.radius, s.proc_mask if s.chroma else 1))
    return sorted(set(out))


def all_specs():
    seen, out = set(), []
    for s in parity_specs() + workload_specs() + api_specs():
        if s not in seen:
            seen.add(s)
            out.append(s)
    return out


def spec_dict(s: RefSpec) -> dict:
    return asdict(s)
