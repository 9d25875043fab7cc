#!/usr/bin/env python3
"""Throughput benchmark of the zb3d BM3D path on B200.

Workload (the metric's configuration): plain two-pass BM3Dv2 on YUV420PS
1920x1080 luma / 960x540 chroma, sigma=[10,10,10], block_step=4, bm_range=12,
radius=0, dct/dct, extractor_exp=3.  Pass 1 (hard threshold) makes the basic
estimate, pass 2 (Wiener) uses it as `ref`; all three planes, every frame.
Frames are seeded synthetic (gradient + 20 rectangles + sinusoidal texture +
N(0, 10/255) noise), 64 per GPU.  A step is that two-pass job over 8 frames.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

`value` is luma megapixels per second of the whole job with inputs resident in
HBM (CUDA events on the launching streams, max over ranks).  `e2e` is the same
job through the public API (zb3d.BM3Dv2 on host frames: pinned staging, H2D,
kernels, D2H inside the timed region).  Multi-GPU runs shard frames across
ranks (no collective on the data path) and report weak scaling.

`--impl reference` times the CPU restatement of the path (the reference ships
no CPU BM3D) on the host's cores over a bounded frame sample.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import sys
import threading
import time
from typing import Optional
from concurrent.futures import ThreadPoolExecutor

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "vapoursynth-zipcu_b200"))

import numpy as np  # noqa: E402

W, H = 1920, 1080
SIGMA = 10.0
BLOCK_STEP, BM_RANGE, EXTRACTOR_EXP = 4, 12, 3
FRAMES_PER_GPU = 64
BATCH = 8
DISTINCT = 8            # distinct synthetic frames, replicated into FRAMES_PER_GPU device buffers
METRIC = "BM3Dv2 1080p Mpix/s: plain vs BF16+learned-pilot form at ΔPSNR≤0.05 dB"
WORKLOAD = ("plain two-pass BM3Dv2, YUV420PS 1920x1080 / 960x540, sigma [10,10,10], block_step 4, "
            "bm_range 12, radius 0, dct/dct, extractor_exp 3")
KW = dict(sigma=[SIGMA] * 3, block_step=BLOCK_STEP, bm_range=BM_RANGE, extractor_exp=EXTRACTOR_EXP)
FORM_KEYS = {0: "fp32_scan", 1: "tensor_core"}
FORM_NAMES = {0: "plain FP32: every candidate's SSD in the reference's order, match lists bit-exact",
              1: "tensor-core: tcgen05 FP16 distance bound, exact FP32 re-rank, match lists bit-exact"}


def plane_dims():
    return [(W, H), (W // 2, H // 2), (W // 2, H // 2)]


def synth_frames(clip: int, count: int, first: int = 0):
    """Frames first .. first + count - 1 of a synthetic clip (three planes each)."""
    from zb3d import synth
    out = []
    for f in range(first, first + count):
        out.append([synth.noisy_plane(w, h, SIGMA, clip=clip, frame=f, plane=p)
                    for p, (w, h) in enumerate(plane_dims())])
    return out


def warm_until(torch, step, warmup: int, min_s: float = 0.3) -> int:
    """Untimed warm-up: `step` at least `warmup` times, then until `min_s` seconds of
    synchronised wall time have passed, so that the SM clocks have left their idle level
    (they take a few hundred ms to rise) before a short timed region starts.  Returns the
    number of steps run."""
    t0 = time.perf_counter()
    n = 0
    while n < warmup or time.perf_counter() - t0 < min_s:
        step()
        n += 1
        if n >= warmup:
            torch.cuda.synchronize()
    return n


def match_flops(w, h, bs, rng):
    """Algorithmic FLOPs of one block-matching launch: 192 per candidate (64 sub,
    64 mul, 64 add per 8x8 distance) over every reference block's clipped window."""
    xs = [min(bs * k, w - 8) for k in range((w - 8 + bs - 1) // bs + 1)]
    ys = [min(bs * k, h - 8) for k in range((h - 8 + bs - 1) // bs + 1)]
    cols = sum(min(x + rng, w - 8) - max(x - rng, 0) + 1 for x in xs)
    rows = sum(min(y + rng, h - 8) - max(y - rng, 0) + 1 for y in ys)
    return 192.0 * cols * rows


class ClockSampler:
    """SM clock and throttle reasons sampled through NVML every 10 ms during the
    timed region."""
    REASONS = {0x4: "sw_power_cap", 0x8: "hw_slowdown", 0x20: "sw_thermal_slowdown",
               0x40: "hw_thermal_slowdown", 0x80: "hw_power_brake_slowdown"}

    def __init__(self, index: int):
        self.index = index
        self.samples = []
        self.mask = 0
        self.max_mhz = None
        self._stop = threading.Event()
        self._t = None
        self._nvml = None
        self._h = None

    def _loop(self):
        nv, h = self._nvml, self._h
        while True:  # at least one sample, however short the timed region
            try:
                self.samples.append(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM))
                self.mask |= nv.nvmlDeviceGetCurrentClocksEventReasons(h)
            except Exception:
                pass
            if self._stop.wait(0.01):
                break

    def start(self):
        # NVML set-up (slow on first use) happens here, before the timed region starts
        try:
            import pynvml as nv
            nv.nvmlInit()
            self._h = nv.nvmlDeviceGetHandleByIndex(self.index)
            self.max_mhz = nv.nvmlDeviceGetMaxClockInfo(self._h, nv.NVML_CLOCK_SM)
            self._nvml = nv
        except Exception:
            self._nvml = None
            return
        self._t = threading.Thread(target=self._loop, daemon=True)
        self._t.start()

    def stop(self):
        if not self._t:
            return None
        self._stop.set()
        self._t.join()
        if not self.samples:
            return None
        return {"sm_mhz": statistics.median(self.samples), "sm_max_mhz": self.max_mhz,
                "reasons": sorted(v for k, v in self.REASONS.items() if self.mask & k),
                "samples": len(self.samples), "source": "NVML, 10 ms"}


# ---------------------------------------------------------------------------
# our implementation, device-resident
# ---------------------------------------------------------------------------
class DevicePipeline:
    """Two-pass BM3Dv2 on device buffers.  Per frame and plane one buffer holds
    [basic | noisy]: pass 1 reads the noisy half and writes the basic half, pass 2
    reads both (ref = basic) and writes the output plane; nothing is copied."""

    def __init__(self, torch, nstreams: int = 2):
        from zb3d import _native as N
        from zb3d.device import DeviceFilter
        self.torch = torch
        self.ns = nstreams
        self.basic = [DeviceFilter(W, H, family=N.YUV, subsampling=(1, 1), num_streams=1, **KW)
                      for _ in range(nstreams)]
        self.final = [DeviceFilter(W, H, family=N.YUV, subsampling=(1, 1), num_streams=1, ref=True, **KW)
                      for _ in range(nstreams)]
        self.lay = self.basic[0].entries
        self.streams = [torch.cuda.Stream() for _ in range(nstreams)]

    def upload(self, frames, count: int):
        t = self.torch
        self.bufs, self.outs = [], []
        for i in range(count):
            src = frames[i % len(frames)]
            fb, fo = [], []
            for e, lay in enumerate(self.lay):
                pe = lay.height * lay.pitch
                b = t.zeros(2 * pe, dtype=t.float32, device="cuda")
                host = np.zeros((lay.height, lay.pitch), np.float32)
                host[:, :lay.width] = src[lay.plane[0]]
                b[pe:].copy_(t.from_numpy(host.reshape(-1)))
                fb.append(b)
                fo.append(t.empty(pe, dtype=t.float32, device="cuda"))
            self.bufs.append(fb)
            self.outs.append(fo)
        t.cuda.synchronize()

    def run_frame(self, j: int, fidx: int):
        k = j % self.ns
        st = self.streams[k].cuda_stream
        for e, lay in enumerate(self.lay):
            b = self.bufs[fidx][e]
            pe4 = lay.height * lay.pitch * 4
            self.basic[k].run_entry(e, b.data_ptr() + pe4, b.data_ptr(), st)
            self.final[k].run_entry(e, b.data_ptr(), self.outs[fidx][e].data_ptr(), st)

    def profile(self, on: bool):
        for f in self.basic + self.final:
            f.profile(on)

    def collect(self):
        mm = mn = fm = fn = 0
        for f in self.basic + self.final:
            a, b, c, d = f.profile_collect()
            mm, mn, fm, fn = mm + a, mn + b, fm + c, fn + d
        return mm, mn, fm, fn

    def timed(self, steps: int, start_frame: int = 0) -> float:
        t = self.torch
        s0 = self.streams[0]
        start, end = t.cuda.Event(enable_timing=True), t.cuda.Event(enable_timing=True)
        start.record(s0)
        for s in self.streams[1:]:
            s.wait_event(start)
        n = len(self.bufs)
        for step in range(steps):
            for j in range(BATCH):
                self.run_frame(j, (start_frame + step * BATCH + j) % n)
        for s in self.streams[1:]:
            ev = t.cuda.Event()
            ev.record(s)
            s0.wait_event(ev)
        end.record(s0)
        end.synchronize()
        return start.elapsed_time(end)

    def launches_per_frame(self) -> int:
        # match + filter + finish per plane and pass (1920/960 widths need no clamped-column launch)
        return 2 * len(self.lay) * 3

    def close(self):
        for f in self.basic + self.final:
            f.close()


def run_pilot_form(torch, frames, clip: int, steps: int, warmup: int, psnr_frames: int = 4, nstreams: int = 4,
                   weights: Optional[str] = None, conv_ctas_per_sm: int = 4):
    """Two-pass BM3Dv2 with the learned pilot (zb3d/pilot.py, shipped weights) as the
    step-2 reference in place of the step-1 estimate, on the same frames: device-resident
    Mpix/s, and PSNR against the clean frames next to the plain two-pass form.
    The network runs batched on its own stream: one launch sequence for the luma planes
    of a step's 8 frames and one for their 16 chroma planes, reading the noisy planes and
    writing the references in place inside the frames' [reference | noisy] buffers.  The
    exact step 2 of each frame then runs on one of `nstreams` streams once its batch's
    network is done, overlapping the next batch's network."""
    from zb3d import _native as N
    from zb3d import pilot as P
    from zb3d import synth
    from zb3d.device import DeviceFilter
    net = P.PilotNet.load(weights) if weights else P.shipped()
    if N.lib().zb3d_pilot_tc_ctas_per_sm(conv_ctas_per_sm) != 0:
        raise SystemExit(f"unsupported --pilot-conv-ctas {conv_ctas_per_sm}")
    finals = [DeviceFilter(W, H, family=N.YUV, subsampling=(1, 1), num_streams=1, ref=True, **KW)
              for _ in range(nstreams)]
    basic = DeviceFilter(W, H, family=N.YUV, subsampling=(1, 1), num_streams=1, **KW)
    lay = finals[0].entries
    assert all(l.pitch == l.width for l in lay), "dense planes expected"
    ly, lc = lay[0], lay[1]
    assert (lay[2].width, lay[2].height) == (lc.width, lc.height)
    nf = len(frames)
    assert nf % BATCH == 0
    py, pc = ly.height * ly.width, lc.height * lc.width
    # [frame][reference | noisy][luma plane] and [frame][U, V][reference | noisy][chroma plane]
    ybuf = torch.zeros((nf, 2, py), dtype=torch.float32, device="cuda")
    cbuf = torch.zeros((nf, 2, 2, pc), dtype=torch.float32, device="cuda")
    for i in range(nf):
        ybuf[i, 1].copy_(torch.from_numpy(np.ascontiguousarray(frames[i][0], np.float32).reshape(-1)))
        for c in (1, 2):
            cbuf[i, c - 1, 1].copy_(torch.from_numpy(np.ascontiguousarray(frames[i][c], np.float32).reshape(-1)))
    outs = [[torch.empty(l.height * l.width, dtype=torch.float32, device="cuda") for l in lay] for _ in range(nf)]
    net_stream = torch.cuda.Stream()
    streams = [torch.cuda.Stream() for _ in range(nstreams)]
    sig_y = torch.full((BATCH,), SIGMA, dtype=torch.float32, device="cuda")
    sig_c = torch.full((2 * BATCH,), SIGMA, dtype=torch.float32, device="cuda")

    def ref_ptr(i, e):  # the plane's [reference | noisy] pair, as step 2 reads it
        return ybuf[i, 0].data_ptr() if e == 0 else cbuf[i, e - 1, 0].data_ptr()

    def pilot_batch(f0, count):
        """network over frames f0 .. f0 + count - 1 on the net stream; returns its event"""
        with torch.cuda.stream(net_stream):
            st = net_stream.cuda_stream
            yv = ybuf[f0:f0 + count].view(count, 2, ly.height, ly.width)
            net.forward(yv[:, 1], sig_y[:count], out=yv[:, 0], stream=st)
            cv = cbuf[f0:f0 + count].view(2 * count, 2, lc.height, lc.width)
            net.forward(cv[:, 1], sig_c[:2 * count], out=cv[:, 0], stream=st)
        ev = torch.cuda.Event()
        ev.record(net_stream)
        return ev

    def step2(i, k, after=None):
        s = streams[k]
        if after is not None:
            s.wait_event(after)
        for e in range(3):
            finals[k].run_entry(e, ref_ptr(i, e), outs[i][e].data_ptr(), s.cuda_stream)

    def plain_step1(i, k):
        s = streams[k]
        for e in range(3):
            basic.run_entry(e, ref_ptr(i, e) + 4 * lay[e].height * lay[e].width, ref_ptr(i, e), s.cuda_stream)

    def psnrs(i):
        """per-plane PSNR against the clean frame, and the squared-error sum and pixel count"""
        torch.cuda.synchronize()
        vals, se, cnt = [], 0.0, 0
        for e, l in enumerate(lay):
            o = outs[i][e].view(l.height, l.width).cpu().numpy().astype(np.float64)
            c = synth.clean_plane(l.width, l.height, clip, i, l.plane[0]).astype(np.float64)
            vals.append(synth.psnr(o, c))
            se += float(np.sum((o - c) ** 2))
            cnt += o.size
        return vals, se, cnt

    def batch(b):
        f0 = (b * BATCH) % nf
        ev = pilot_batch(f0, BATCH)
        for j in range(BATCH):
            step2(f0 + j, j % nstreams, ev)

    plain, piloted, se = [], [], [0.0, 0.0, 0]
    for i in range(min(psnr_frames, nf)):
        plain_step1(i, 0)
        step2(i, 0)
        v, e2, c = psnrs(i)
        plain.append(v)
        se[0] += e2
        step2(i, 0, pilot_batch(i, 1))
        v, e2, c = psnrs(i)
        piloted.append(v)
        se[1] += e2
        se[2] += c
    for b in range(max(warmup, 1)):
        batch(b)
    torch.cuda.synchronize()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0.record(net_stream)
    for s in streams:
        s.wait_event(t0)
    for b in range(steps):
        batch(b)
    for s in streams:
        ev = torch.cuda.Event()
        ev.record(s)
        net_stream.wait_event(ev)
    t1.record(net_stream)
    t1.synchronize()
    ms = t0.elapsed_time(t1)
    plain, piloted = np.array(plain), np.array(piloted)
    delta = float(np.mean(piloted - plain))
    # all pixels of all planes pooled (luma weighs 4x a chroma plane): 10 log10 of the MSE ratio
    delta_pooled = float(10.0 * np.log10(se[0] / se[1]))
    for f in finals:
        f.close()
    basic.close()
    return {"value": W * H * steps * BATCH / (ms / 1e3) / 1e6, "unit": "Mpix/s", "ms_per_frame": ms / (steps * BATCH),
            "psnr_plain_two_pass_db": float(np.mean(plain)), "psnr_pilot_two_pass_db": float(np.mean(piloted)),
            "delta_psnr_db": delta, "delta_psnr_db_per_plane": [float(d) for d in np.mean(piloted - plain, 0)],
            "delta_psnr_db_all_pixels": delta_pooled,
            "within_0_05_db": delta >= -0.05 and delta_pooled >= -0.05, "streams": nstreams,
            "conv_ctas_per_sm": conv_ctas_per_sm,
            "what": "pilot (%d x conv3x3, %d ch, BF16 tcgen05 kernels, FP32 accumulation in tensor memory) as step 1 "
                    "on every plane, batched per step (8 luma, 16 chroma planes per launch) on its own stream, then "
                    "the exact step 2 of each frame on %d streams; PSNR over the first %d frames against the clean "
                    "frames" % (net.layers, net.width, nstreams, min(psnr_frames, nf))}


def run_e2e(frames, steps: int, warmup: int, num_streams: int = 4, pinned: bool = True, pilot=None):
    """Same job through the public API on host frames (zb3d.BM3Dv2): page-locked frames (the
    library DMAs them) or pageable ones (copied through its pinned staging).  With `pilot`
    (a zb3d.Pilot) the two steps are one filter, BM3Dv2(clip, pilot=...)."""
    import zb3d
    from zb3d import _native as N
    nfr = BATCH * (steps + warmup)
    host = [frames[i % len(frames)] for i in range(nfr)]
    clip = zb3d.Clip.from_frames(host, family=N.YUV, subsampling=(1, 1), pinned=pinned)
    if pilot is not None:
        final = zb3d.BM3Dv2(clip, pilot=pilot, num_streams=num_streams, **KW)
    else:
        basic = zb3d.BM3Dv2(clip, num_streams=num_streams, **KW)
        final = zb3d.BM3Dv2(clip, ref=basic, num_streams=num_streams, **KW)
    # two request threads per stream keep every stream fed while the other thread of the
    # pair waits for its frame; frames are requested continuously (no drain between steps)
    # and each output is dropped once read, so the page-locked output pool stays small
    pool = ThreadPoolExecutor(2 * num_streams)

    def run(lo, hi):
        for out in pool.map(final.get_frame, range(lo, hi)):
            del out

    run(0, warmup * BATCH)
    t0 = time.perf_counter()
    run(warmup * BATCH, (warmup + steps) * BATCH)
    dt = time.perf_counter() - t0
    pool.shutdown()
    # bytes per step: pass 1 uploads the clip, pass 2 the ref and the clip; both download their output
    # (the pilot form uploads the clip once and downloads its output once)
    px = sum(w * h for w, h in plane_dims())
    h2d = (1 if pilot is not None else 3) * px * 4 * BATCH
    d2h = (1 if pilot is not None else 2) * px * 4 * BATCH
    return dt, h2d, d2h


# ---------------------------------------------------------------------------
# the reference's own kernels on the same GPU (drop-in comparison)
# ---------------------------------------------------------------------------
def run_ref_cuda(torch, frames, steps: int, warmup: int, nstreams: int = 4):
    """The reference's kernels, each frame's launch sequence on one of `nstreams` streams
    in turn (the reference host's default is 4 stream slots, vszipcu src/bm3d.zig:1077-1081)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    try:
        import ref_configs as rc
        import refh
    except Exception:
        return None
    specs = {}
    for final in (0, 1):
        for (w, h) in ((W, H), (W // 2, H // 2)):
            s = rc.RefSpec(w=w, h=h, stride=w, sigma=(SIGMA,) * 3, block_step=BLOCK_STEP, bm_range=BM_RANGE,
                           final=final, extractor_exp=EXTRACTOR_EXP)
            if not (refh.available() and refh.has_cubin(s)):
                return None
            specs[(final, w)] = s
    ns = nstreams
    kernels = [{k: refh.RefKernel(s) for k, s in specs.items()} for _ in range(ns)]
    streams = [torch.cuda.Stream() for _ in range(ns)]
    dims = plane_dims()
    bufs, res = [], []
    for i in range(FRAMES_PER_GPU):
        src = frames[i % len(frames)]
        fb = []
        for p, (w, h) in enumerate(dims):
            b = torch.zeros(2 * w * h, dtype=torch.float32, device="cuda")
            b[w * h:].copy_(torch.from_numpy(np.ascontiguousarray(src[p]).reshape(-1)))
            fb.append((b, torch.empty(w * h, dtype=torch.float32, device="cuda")))
        bufs.append(fb)
    for k in range(ns):
        res.append({w: torch.empty(2 * w * h, dtype=torch.float32, device="cuda") for (w, h) in dims})

    def frame(j, fidx):
        k = j % ns
        st = streams[k].cuda_stream
        for p, (w, h) in enumerate(dims):
            b, out = bufs[fidx][p]
            r = res[k][w]
            kernels[k][(0, w)].run(r.data_ptr(), b.data_ptr() + w * h * 4, b.data_ptr(), r.numel() * 4, st)
            kernels[k][(1, w)].run(r.data_ptr(), b.data_ptr(), out.data_ptr(), r.numel() * 4, st)

    def timed(nsteps, first):
        s0 = streams[0]
        a, z = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(s0)
        for st in streams[1:]:
            st.wait_event(a)
        for s in range(nsteps):
            for j in range(BATCH):
                frame(j, (first + s * BATCH + j) % FRAMES_PER_GPU)
        for st in streams[1:]:
            ev = torch.cuda.Event()
            ev.record(st)
            s0.wait_event(ev)
        z.record(s0)
        z.synchronize()
        return a.elapsed_time(z)

    timed(warmup, 0)
    ms = timed(steps, warmup * BATCH)
    for d in kernels:
        for kk in d.values():
            kk.close()
    return ms


# ---------------------------------------------------------------------------
# CPU restatement (FP64 oracle) on the host cores
# ---------------------------------------------------------------------------
def cpu_two_pass_frame(frame, nthreads):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as orc
    import ref_configs as rc
    for p, (w, h) in enumerate(plane_dims()):
        noisy = np.ascontiguousarray(frame[p], np.float32)
        c1 = orc.make_cfg(w, h, w, [rc.scaled_sigma(SIGMA, False)], BLOCK_STEP, BM_RANGE, 0,
                          nthreads=nthreads, extractor_exp=EXTRACTOR_EXP)
        num, den, _ = orc.bm3d_pass(c1, noisy[None, None, None], want_matches=False)
        basic = (num[0, 0] / den[0, 0]).astype(np.float32)
        c2 = orc.make_cfg(w, h, w, [rc.scaled_sigma(SIGMA, True)], BLOCK_STEP, BM_RANGE, 0, final=1,
                          nthreads=nthreads, extractor_exp=EXTRACTOR_EXP)
        src = np.stack([basic, noisy])[:, None, None]
        orc.bm3d_pass(c2, src, want_matches=False)


def cpu_baseline(frames, budget_s: float = 20.0, max_frames: int = 4):
    nthreads = os.cpu_count() or 1
    t0 = time.perf_counter()
    done = 0
    while done < max_frames and (done == 0 or time.perf_counter() - t0 < budget_s):
        cpu_two_pass_frame(frames[done % len(frames)], nthreads)
        done += 1
    dt = time.perf_counter() - t0
    return {"value": W * H * done / dt / 1e6, "unit": "Mpix/s", "cores": nthreads, "kind": "port",
            "sample": f"{done} full 1080p YUV420 frame(s), both passes, all planes, FP64 oracle "
                      f"(FP32 exact-order matching), {dt:.1f} s"}


def reference_arm(args, rank: int, world: int):
    if rank != 0:
        return 0
    nthreads = os.cpu_count() or 1
    frames = synth_frames(0, 2)
    for i in range(args.warmup):
        cpu_two_pass_frame(frames[i % 2], nthreads)
    t0 = time.perf_counter()
    for i in range(args.steps):
        cpu_two_pass_frame(frames[i % 2], nthreads)
    dt = time.perf_counter() - t0
    v = W * H * args.steps / dt / 1e6
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "Mpix/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3 / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "step": "one frame (both passes, all planes) on the CPU"},
            "cpu_baseline": {"value": v, "unit": "Mpix/s", "cores": nthreads, "kind": "port",
                             "sample": f"{args.steps} 1080p YUV420 frames, FP64 restatement of the path "
                                       "(the reference has no CPU BM3D)"},
            "e2e": {"value": v, "unit": "Mpix/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def run_vbm3d(torch, steps: int, warmup: int, filter_form: int = 0):
    """1080p GRAYS VBM3D through BM3Dv2's fused path on the device: radius 2, sigma 15,
    default block_step / bm_range, moving synthetic scene, 120 frames in HBM.  Per
    output frame one window (2r+1 frames) is filtered into an accumulator stack and
    the 2r+1 stacks around it are aggregated; a step is 8 output frames.
    filter_form 1: the precision form (2D transforms on the tensor cores in split TF32);
    then one window's accumulators are also compared with the plain form's and with the
    FP64 oracle's."""
    import ctypes
    from zb3d import _native as N
    from zb3d import synth
    from zb3d.device import DeviceFilter
    # 120 frames, or more so that every timed output frame (8 .. 8 * (steps + 1) - 1) is in the clip
    r, nf, sigma = 2, max(120, BATCH * (steps + 2)), 15.0
    tw = 2 * r + 1
    f = DeviceFilter(W, H, num_frames=nf, sigma=[sigma], radius=r, extractor_exp=EXTRACTOR_EXP, num_streams=1,
                     filter_form=filter_form)
    lay = f.entries[0]
    pe = lay.height * lay.pitch
    distinct = 16
    host = np.zeros((distinct, H, lay.pitch), np.float32)
    for i in range(distinct):
        host[i, :, :W] = synth.noisy_plane(W, H, sigma, frame=i, motion=True)[:, :W]
    frames = torch.empty((nf + 2 * r, H, lay.pitch), dtype=torch.float32, device="cuda")
    # frames[r + n] = frame n; the r frames on each side repeat the first / last frame,
    # so the window of centre m, frames clamp(m-r .. m+r), is frames[m .. m+2r]
    for n in range(nf):
        frames[r + n].copy_(torch.from_numpy(host[n % distinct]))
    for k in range(r):
        frames[k].copy_(frames[r])
        frames[r + nf + k].copy_(frames[r + nf - 1])
    stacks = [torch.empty(tw * 2 * pe, dtype=torch.float32, device="cuda") for _ in range(tw + 1)]
    out = torch.empty((8, H, lay.pitch), dtype=torch.float32, device="cuda")
    st = torch.cuda.Stream()
    lib = N.lib()

    def stack_of(m):
        return stacks[m % len(stacks)]

    def compute(m):
        f.run_entry(0, frames[m].data_ptr(), stack_of(m).data_ptr(), st.cuda_stream)

    def aggregate(n):
        ptrs = (ctypes.c_void_p * tw)(*[stack_of(min(max(n - r + i, 0), nf - 1)).data_ptr() for i in range(tw)])
        zs = (ctypes.c_int * tw)(*[lib.zb3d_agg_z(i, n, nf, r) for i in range(tw)])
        rc = lib.zb3d_vaggregate_device(ptrs, zs, tw, W, H, lay.pitch, 1, 1, out[n % 8].data_ptr(),
                                        ctypes.c_void_p(st.cuda_stream))
        assert rc == 0

    def run(first, count):
        for n in range(first, first + count):
            m = n + r
            if n == 0:  # later runs find centres n-r..n+r-1 in the ring already
                for c in range(0, min(m, nf)):
                    compute(c)
            if m < nf:
                compute(m)
            aggregate(n)

    with torch.cuda.stream(st):
        nw = warm_until(torch, lambda: run(0, BATCH), warmup)
        a, z = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(st)
        run(BATCH, steps * BATCH)
        z.record(st)
        z.synchronize()
    ms = a.elapsed_time(z)
    res = {"metric": "VBM3D 1080p Mpix/s (BM3Dv2 radius 2, fused)", "value": W * H * steps * BATCH / ms * 1e3 / 1e6,
           "unit": "Mpix/s", "ms_per_step": ms / steps, "steps": steps, "warmup": warmup, "warmup_steps_run": nw,
           "config": {"workload": "GRAYS 1920x1080, radius 2, sigma 15, block_step 8, bm_range 9, ps_num 2, "
                                  f"ps_range 4, extractor_exp 3, moving scene, {nf} frames, one window + one "
                                  "temporal aggregation per output frame", "batch_frames_per_step": BATCH,
                      "filter": "precision: 2D transforms on tcgen05, split TF32" if filter_form else
                                "plain: FP32 transforms, bit for bit the reference's"}}
    if filter_form:
        res["precision_error"] = vbm3d_window_errors(torch, f, frames, r, sigma)
    f.close()
    return res


def vbm3d_window_errors(torch, f, frames, r, sigma, centre: int = 10):
    """The accumulator stack of one window (centre `centre`) from the filter f, from the same
    filter in the plain form, and from the FP64 oracle: each slot's estimate num / den where
    den > 0, compared (max and mean absolute difference)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as orc
    import ref_configs as rc
    from zb3d.device import DeviceFilter
    lay = f.entries[0]
    tw = 2 * r + 1
    pe = lay.height * lay.pitch
    plain = DeviceFilter(W, H, num_frames=120, sigma=[sigma], radius=r, extractor_exp=EXTRACTOR_EXP, num_streams=1)
    outs = []
    for flt in (f, plain):
        st = torch.empty(tw * 2 * pe, dtype=torch.float32, device="cuda")
        flt.run_entry(0, frames[centre].data_ptr(), st.data_ptr())
        torch.cuda.synchronize()
        v = st.view(tw, 2, H, lay.pitch)[..., :W].cpu().numpy().astype(np.float64)
        outs.append(v)
    plain.close()
    win = frames[centre:centre + tw].cpu().numpy()  # [tw][H][pitch]
    cfg = orc.make_cfg(W, H, lay.pitch, [rc.scaled_sigma(sigma, False)], 8, 9, r, 2, 4, 0, 0,
                       extractor_exp=EXTRACTOR_EXP)
    t0 = time.perf_counter()
    num, den, _ = orc.bm3d_pass(cfg, np.ascontiguousarray(win[None, None], np.float32), want_matches=False)
    oracle_s = time.perf_counter() - t0
    ref = np.where(den[0] > 0, num[0] / np.where(den[0] > 0, den[0], 1), np.nan)

    def est(v):
        return np.where(v[:, 1] > 0, v[:, 0] / np.where(v[:, 1] > 0, v[:, 1], 1), np.nan)

    def cmp(a, b):
        d = np.abs(a - b)
        d = d[np.isfinite(d)]
        return {"max_abs": float(d.max()), "mean_abs": float(d.mean())}
    p, q = est(outs[0]), est(outs[1])
    return {"window": f"centre frame {centre}, {tw} frames, every slot's estimate num/den where den > 0",
            "precision_vs_fp64_oracle": cmp(p, ref), "plain_vs_fp64_oracle": cmp(q, ref),
            "precision_vs_plain": cmp(p, q), "oracle_s": round(oracle_s, 1)}


def run_pilot4k(torch, steps: int, warmup: int, nstreams: int = 4, weights: Optional[str] = None):
    """Learned-pilot BM3Dv2 on GRAYS 3840x2160: 4 clips of 8 frames, sigma per clip from
    U[5, 25], block_step 4, bm_range 12, with the 48-channel, 10-layer pilot trained on 4K
    planes (shipped weights).  Per clip, the two-pass PSNR against the clean frames is
    measured with the plain step 1 and with the pilot as step 2's reference; the form
    falls back to the plain step 1 where the pilot loses more than 0.05 dB.  Both forms are
    timed (device-resident, `nstreams` streams); `value` is the gated form's Mpix/s.  The
    blind gate (`PilotGate`, calibrated per sigma on held-out 4K frames) is reported beside
    each clip's measured decision."""
    from zb3d import _native as N
    from zb3d import pilot as P
    from zb3d import synth
    from zb3d.device import DeviceFilter
    w, h, nclips, nfr = 3840, 2160, 4, 8
    kw = dict(block_step=4, bm_range=12, extractor_exp=EXTRACTOR_EXP)
    net = P.PilotNet.load(weights or P.WEIGHTS_4K)
    gate = P.PilotGate(net)
    gate.calibrate([5.0, 10.0, 15.0, 20.0, 25.0], frames=1, size=(w, h), **kw)
    rng = np.random.default_rng(4040)
    streams = [torch.cuda.Stream() for _ in range(nstreams)]
    pe = w * h
    total_ms, rows = 0.0, []
    for c in range(nclips):
        sigma = float(rng.uniform(5.0, 25.0))
        basic = [DeviceFilter(w, h, family=N.GRAY, num_streams=1, sigma=[sigma], **kw) for _ in range(nstreams)]
        final = [DeviceFilter(w, h, family=N.GRAY, num_streams=1, sigma=[sigma], ref=True, **kw)
                 for _ in range(nstreams)]
        sig = torch.full((1,), sigma, dtype=torch.float32, device="cuda")
        bufs, outs, clean = [], [], []
        for f in range(nfr):
            b = torch.empty(2 * pe, dtype=torch.float32, device="cuda")  # [reference | noisy]
            b[pe:].copy_(torch.from_numpy(synth.noisy_plane(w, h, sigma, clip=3000 + c, frame=f).reshape(-1)))
            bufs.append(b)
            outs.append(torch.empty(pe, dtype=torch.float32, device="cuda"))
            clean.append(synth.clean_plane(w, h, 3000 + c, f))

        def frame(f, k, pilot):
            s = streams[k]
            with torch.cuda.stream(s):
                b = bufs[f]
                if pilot:
                    net.forward(b[pe:].view(1, h, w), sig, out=b[:pe].view(1, h, w), stream=s.cuda_stream)
                else:
                    basic[k].run(b.data_ptr() + 4 * pe, b.data_ptr(), s.cuda_stream)
                final[k].run(b.data_ptr(), outs[f].data_ptr(), s.cuda_stream)

        def psnrs(pilot):
            for f in range(nfr):
                frame(f, f % nstreams, pilot)
            torch.cuda.synchronize()
            return [synth.psnr(outs[f].view(h, w).cpu().numpy(), clean[f]) for f in range(nfr)]

        def timed(pilot):
            for _ in range(max(warmup, 1)):
                for f in range(nfr):
                    frame(f, f % nstreams, pilot)
            torch.cuda.synchronize()
            t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            t0.record(streams[0])
            for s in streams[1:]:
                s.wait_event(t0)
            for _ in range(steps):
                for f in range(nfr):
                    frame(f, f % nstreams, pilot)
            for s in streams[1:]:
                e = torch.cuda.Event()
                e.record(s)
                streams[0].wait_event(e)
            t1.record(streams[0])
            t1.synchronize()
            return t0.elapsed_time(t1)

        plain, piloted = np.mean(psnrs(False)), np.mean(psnrs(True))
        delta = float(piloted - plain)
        use_pilot = delta >= -0.05
        ms_plain, ms_pilot = timed(False), timed(True)
        total_ms += ms_pilot if use_pilot else ms_plain
        rows.append({"sigma": round(sigma, 3), "delta_psnr_db": delta, "step1": "pilot" if use_pilot else "plain",
                     "blind_gate_step1": "pilot" if gate.accepts(sigma) else "plain",
                     "psnr_plain_two_pass_db": float(plain), "psnr_pilot_two_pass_db": float(piloted),
                     "ms_per_frame_plain": ms_plain / (steps * nfr), "ms_per_frame_pilot": ms_pilot / (steps * nfr)})
        for fl in basic + final:
            fl.close()
        del bufs, outs
    px = w * h * nclips * nfr * steps
    return {"metric": "learned-pilot BM3Dv2 GRAYS 3840x2160 Mpix/s (0.05 dB fallback)",
            "value": px / (total_ms / 1e3) / 1e6, "unit": "Mpix/s", "n_gpus": 1, "steps": steps, "warmup": warmup,
            "ms_per_step": total_ms / steps, "higher_is_better": True, "dtype": "bf16 pilot / f32 BM3D",
            "data": "synthetic",
            "config": {"workload": "GRAYS 3840x2160, 4 clips x 8 frames, sigma per clip U[5,25], block_step 4, "
                                   "bm_range 12, pilot 48 ch x 10 layers trained on 4K planes (tcgen05), plain "
                                   "step 1 where the pilot loses more than 0.05 dB", "streams": nstreams},
            "blind_gate_delta_db_by_sigma": {str(k): round(v, 3) for k, v in gate.delta.items()},
            "clips": rows}


def run_gray640(torch, steps: int, warmup: int):
    """640x480 GRAYS single-pass BM3D, sigma 3, block_step 8, bm_range 9; a step is 8 frames."""
    from zb3d import synth
    from zb3d.device import DeviceFilter
    w, h = 640, 480
    f = DeviceFilter(w, h, num_frames=8, sigma=[3.0], extractor_exp=EXTRACTOR_EXP, num_streams=1)
    lay = f.entries[0]
    src = torch.zeros((8, h, lay.pitch), dtype=torch.float32, device="cuda")
    for i in range(8):
        src[i, :, :w].copy_(torch.from_numpy(synth.noisy_plane(w, h, 3.0, frame=i)[:, :w]))
    out = torch.empty_like(src)
    st = torch.cuda.Stream()

    def step():
        for i in range(8):
            f.run_entry(0, src[i].data_ptr(), out[i].data_ptr(), st.cuda_stream)

    nw = warm_until(torch, step, warmup)
    a, z = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(st)
    for _ in range(steps):
        step()
    z.record(st)
    z.synchronize()
    ms = a.elapsed_time(z)
    f.close()
    return {"warmup_steps_run": nw, "metric": "BM3D 640x480 Mpix/s (sigma 3, block_step 8)", "value": w * h * 8 * steps / ms * 1e3 / 1e6,
            "unit": "Mpix/s", "ms_per_step": ms / steps, "steps": steps, "warmup": warmup,
            "config": {"workload": "GRAYS 640x480 x 8 frames, sigma 3, block_step 8, bm_range 9, dct/dct, "
                                   "extractor_exp 3, single pass"}}


def run_dct_tf32(torch, steps: int, warmup: int):
    """Precision form of the patch transform (zb3d_dct2d_tf32): the 2D DCT of the group stack
    of one 1920x1080 luma plane at block_step 4 (128,851 groups x 8 patches) on the tcgen05
    tensor cores in TF32, with the hi/lo split and without it; the error of each against an
    FP64 transform of a 4096-patch sample, relative to the sample's largest coefficient."""
    from zb3d import _native as N
    from zb3d import synth
    lib = N.lib()
    npat = 128851 * 8
    plane = synth.noisy_plane(W, H, SIGMA, frame=0)
    rng = np.random.default_rng(0)
    ys = rng.integers(0, H - 8, npat)
    xs = rng.integers(0, W - 8, npat)
    pl = torch.from_numpy(np.ascontiguousarray(plane[:, :W])).cuda()
    iy = torch.from_numpy(ys).cuda()[:, None, None] + torch.arange(8, device="cuda")[None, :, None]
    ix = torch.from_numpy(xs).cuda()[:, None, None] + torch.arange(8, device="cuda")[None, None, :]
    x = pl[iy, ix].reshape(npat, 64).contiguous()
    y = torch.empty_like(x)
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    st = torch.cuda.Stream()
    k = np.arange(8)[:, None]
    T = 4.0 * np.where(k == 0, np.sqrt(1 / 8), np.sqrt(2 / 8)) * np.cos(np.pi * (2 * np.arange(8)[None, :] + 1) * k / 16)
    K = np.kron(T, T)
    out = {"metric": "2D DCT of 8x8 patches, tcgen05 TF32 (GB/s of patches in + out)", "unit": "GB/s",
           "steps": steps, "warmup": warmup,
           "config": {"workload": f"{npat} patches (the block_step 4 group stack of a 1920x1080 Y plane), "
                                  "[n][64] FP32 in device memory, inputs larger than L2 (528 MB per call)"}}
    for split in (1, 0):
        def call():
            rc = lib.zb3d_dct2d_tf32(x.data_ptr(), y.data_ptr(), npat, split, status.data_ptr(), st.cuda_stream)
            if rc:
                raise RuntimeError(f"zb3d_dct2d_tf32 returned {rc}")
        warm_until(torch, call, warmup)
        a, z = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(st)
        for _ in range(steps):
            call()
        z.record(st)
        z.synchronize()
        ms = a.elapsed_time(z) / steps
        if int(status.item()):
            raise RuntimeError("zb3d_dct2d_tf32: a wait timed out")
        xs_ = x[:4096].cpu().numpy().astype(np.float64)
        ref = xs_ @ K.T
        err = float(np.abs(y[:4096].cpu().numpy() - ref).max() / np.abs(ref).max())
        key = "split" if split else "single_tf32"
        out[key] = {"ms_per_call": ms, "GB_per_s": npat * 512 / ms / 1e6,
                    "tensor_TFLOP_per_s": npat * 8192 * (3 if split else 1) / ms / 1e9,
                    "rel_max_error_vs_fp64": err}
    out["value"] = out["split"]["GB_per_s"]
    try:
        peak = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["hbm_gbs"]
        src = "measured copy bandwidth (MEASURED_PEAKS.json)"
    except Exception:
        peak, src = 6650.0, "fallback copy bandwidth"
    out["roofline"] = {"bound": "hbm", "achieved": out["value"], "peak": peak, "unit": "GB/s",
                       "frac": out["value"] / peak, "traffic": None, "peak_source": src,
                       "how": "algorithmic bytes (256 B read + 256 B written per patch) / CUDA-event time per call"}
    return out


def run_match1080(torch, steps: int, warmup: int):
    """Block matching alone, the dominant kernel of the metric's workload: the Y, U and V
    entries of a 1920x1080 YUV420 BM3Dv2 filter (block_step 4, bm_range 12), each matched
    with the configuration the autotuner chose (zb3d_match_device), timed per launch with
    CUDA events on the launching stream.  The plane stays resident in L2 between launches
    (the kernel reads it once per launch and is bound by arithmetic, not by HBM)."""
    from zb3d import _native as N
    from zb3d import synth
    from zb3d.device import DeviceFilter
    f = DeviceFilter(W, H, family=N.YUV, subsampling=(1, 1), num_streams=1, **KW)
    src = np.zeros(f.src_elems, np.float32)
    lists, flops, names = [], [], []
    for e, lay in enumerate(f.entries):
        view = src[lay.src_offset:lay.src_offset + lay.src_elems].reshape(lay.height, lay.pitch)
        view[:, :lay.width] = synth.noisy_plane(lay.width, lay.height, SIGMA, plane=e)
        nbx = (lay.width - 8 + BLOCK_STEP - 1) // BLOCK_STEP + 1
        nby = (lay.height - 8 + BLOCK_STEP - 1) // BLOCK_STEP + 1
        lists.append(torch.zeros((nby, nbx, 8, 2), dtype=torch.int32, device="cuda"))
        flops.append(match_flops(lay.width, lay.height, BLOCK_STEP, BM_RANGE))
        names.append(f"{'YUV'[e]} {lay.width}x{lay.height}")
    d_src = torch.from_numpy(src).cuda()
    st = torch.cuda.Stream()
    torch.cuda.synchronize()

    def step(rec=None):
        for e in range(len(lists)):
            a = torch.cuda.Event(enable_timing=True)
            a.record(st)
            f.match(e, d_src.data_ptr(), lists[e].data_ptr(), st.cuda_stream)
            z = torch.cuda.Event(enable_timing=True)
            z.record(st)
            if rec is not None:
                rec.append((e, a, z))

    nw = warm_until(torch, step, warmup)
    rec = []
    g0 = torch.cuda.Event(enable_timing=True)
    g0.record(st)
    for _ in range(steps):
        step(rec)
    g1 = torch.cuda.Event(enable_timing=True)
    g1.record(st)
    g1.synchronize()
    ms = g0.elapsed_time(g1) / steps
    per = {}
    for e, a, z in rec:
        per.setdefault(e, []).append(a.elapsed_time(z))
    planes = {}
    for e in per:
        t = float(np.median(per[e]))
        form, rows = f.tuning(e)
        planes[names[e]] = {"ms": t, "TFLOP_per_s": flops[e] / t / 1e9, "form": FORM_KEYS.get(form, form),
                            "rows_per_cta": rows}
    peak = 148 * 128 * 2 * 1965e6 / 1e12
    achieved = sum(flops) / (ms / 1e3) / 1e12
    f.close()
    return {"metric": "block matching of one 1920x1080 YUV420 frame (Y, U, V), luma Mpix/s", "unit": "Mpix/s",
            "value": W * H / (ms / 1e3) / 1e6, "ms_per_step": ms, "steps": steps, "warmup": warmup,
            "warmup_steps_run": nw, "planes": planes,
            "roofline": {"bound": "fp32", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                         "frac": achieved / peak, "traffic": None,
                         "how": "192 FLOP per candidate over every block's clipped window, 3 launches per step "
                                "/ CUDA-event time; peak: 148 SMs x 128 FP32 lanes x 2 x 1965 MHz (nominal)"},
            "config": {"workload": "zb3d_match_device on the Y, U and V entries of BM3Dv2 YUV420 1920x1080 / "
                                   "960x540, block_step 4, bm_range 12, ssd; autotuned configuration",
                       "l2": "plane resident in L2 between launches (arithmetic-bound kernel)"}}


def run_batched(torch, steps: int, warmup: int, nstreams: int = 4):
    """Uneven batch: 720x480, 1280x720 and 3840x2160 clips of 16 frames, YUV420 per plane or
    YUV444 CBM3D (chroma=1, matched on Y), radius 0 or 1 (stacked output), sigma drawn per
    clip from U[5, 20], autotuned matching.  Every clip frame is one device window, replayed
    as a CUDA graph; windows are spread round-robin over `nstreams` streams.  A step is all
    64 windows.  Latency per window: its CUDA events on its stream, queueing included."""
    from zb3d import _native as N
    from zb3d import synth
    from zb3d.device import DeviceFilter
    rng = np.random.default_rng(2024)
    clips = [dict(w=720, h=480, fam=N.YUV, sub=(1, 1), chroma=0, radius=0),
             dict(w=1280, h=720, fam=N.YUV, sub=(0, 0), chroma=1, radius=0),
             dict(w=1280, h=720, fam=N.YUV, sub=(1, 1), chroma=0, radius=1),
             dict(w=3840, h=2160, fam=N.YUV, sub=(1, 1), chroma=0, radius=0)]
    nfr = 16
    for c in clips:
        c["sigma"] = float(rng.uniform(5.0, 20.0))
        c["filters"] = [DeviceFilter(c["w"], c["h"], family=c["fam"], subsampling=c["sub"], num_streams=1,
                                     num_frames=nfr, sigma=[c["sigma"]] * 3, chroma=c["chroma"], radius=c["radius"],
                                     block_step=4, bm_range=12, extractor_exp=EXTRACTOR_EXP) for _ in range(nstreams)]
        f0 = c["filters"][0]
        c["src"], c["dst"] = [], []
        tw = 2 * c["radius"] + 1
        planes = [synth.noisy_plane(c["w"] >> (p > 0 and c["sub"][0]), c["h"] >> (p > 0 and c["sub"][1]),
                                    c["sigma"], clip=7, frame=0, plane=p) for p in range(3)]
        for n in range(nfr):  # the same content in every window keeps the set-up short; the work is identical
            host = np.zeros(f0.src_elems, np.float32)
            for lay in f0.entries:
                v = host[lay.src_offset:lay.src_offset + lay.src_elems].reshape(
                    lay.nclips, lay.nplanes, lay.tw, lay.height, lay.pitch)
                for i in range(lay.nplanes):
                    v[:, i, :, :, :lay.width] = planes[lay.plane[i]][:, :lay.width]
            c["src"].append(torch.from_numpy(host).cuda())
            c["dst"].append(torch.empty(f0.dst_elems, dtype=torch.float32, device="cuda"))
        c["tw"] = tw
    streams = [torch.cuda.Stream() for _ in range(nstreams)]
    order = [(ci, n) for n in range(nfr) for ci in range(len(clips))]

    def step(record=None):
        for k, (ci, n) in enumerate(order):
            c, j = clips[ci], k % nstreams
            st = streams[j]
            if record is not None:
                a = torch.cuda.Event(enable_timing=True)
                a.record(st)
            c["filters"][j].run(c["src"][n].data_ptr(), c["dst"][n].data_ptr(), st.cuda_stream)
            if record is not None:
                z = torch.cuda.Event(enable_timing=True)
                z.record(st)
                record.append((ci, a, z))

    for _ in range(max(warmup, 1)):
        step()
    torch.cuda.synchronize()
    t0 = torch.cuda.Event(enable_timing=True)
    t0.record(streams[0])
    for s in streams[1:]:
        s.wait_event(t0)
    recs = []
    for _ in range(steps):
        step(recs)
    for s in streams[1:]:
        e = torch.cuda.Event()
        e.record(s)
        streams[0].wait_event(e)
    t1 = torch.cuda.Event(enable_timing=True)
    t1.record(streams[0])
    t1.synchronize()
    ms = t0.elapsed_time(t1)
    lat = {ci: [] for ci in range(len(clips))}
    for ci, a, z in recs:
        lat[ci].append(a.elapsed_time(z))
    px = sum(c["w"] * c["h"] * nfr for c in clips) * steps
    # the same step through zb3d_process_batch: one call per 16 windows (a frame of every clip
    # x 4 frames), each a persistent work-list launch over the windows' eligible planes (the
    # r1 clip's planes run entry by entry inside the call); latency per call
    from zb3d.device import process_batch
    bst = torch.cuda.Stream()
    per_call = 16
    calls = [order[i:i + per_call] for i in range(0, len(order), per_call)]

    def bstep(record=None):
        for call in calls:
            a = torch.cuda.Event(enable_timing=True)
            a.record(bst)
            # windows spread over each clip's filter instances as in the graph form, so that the
            # entries the batch kernel does not take (the r1 clip) run on several slots at once
            process_batch([(clips[ci]["filters"][n % nstreams], clips[ci]["src"][n].data_ptr(),
                            clips[ci]["dst"][n].data_ptr()) for ci, n in call], bst.cuda_stream)
            z = torch.cuda.Event(enable_timing=True)
            z.record(bst)
            if record is not None:
                record.append((a, z))

    for _ in range(max(warmup, 1)):
        bstep()
    torch.cuda.synchronize()
    brec = []
    bt0 = time.perf_counter()
    for _ in range(steps):
        bstep(brec)
    torch.cuda.synchronize()
    bwall = time.perf_counter() - bt0
    blat = np.array([a.elapsed_time(z) for a, z in brec])
    batch_form = {"value": px / bwall / 1e6, "unit": "Mpix/s", "ms_per_step": bwall * 1e3 / steps,
                  "calls_per_step": len(calls), "windows_per_call": per_call,
                  "latency_ms_p50": float(np.percentile(blat, 50)), "latency_ms_p99": float(np.percentile(blat, 99)),
                  "how": f"zb3d_process_batch (synchronous) per {per_call} windows on one stream; value by wall "
                         "clock over the timed steps, latency by CUDA events around each call"}
    # the same step as 4 batches captured once as CUDA graphs (zb3d_batch_create), replayed
    # asynchronously round-robin on 2 streams; the r1 clip's windows use filters of their
    # own with a slot per live batch (each batch holds one slot of such a filter)
    from zb3d.device import Batch
    gfil = {ci: [DeviceFilter(c["w"], c["h"], family=c["fam"], subsampling=c["sub"], num_streams=len(calls),
                              num_frames=nfr, sigma=[c["sigma"]] * 3, chroma=c["chroma"], radius=c["radius"],
                              block_step=4, bm_range=12, extractor_exp=EXTRACTOR_EXP) for _ in range(nstreams)]
            for ci, c in enumerate(clips) if c["radius"] > 0}

    def gfilter(ci, n):
        return gfil[ci][n % nstreams] if ci in gfil else clips[ci]["filters"][n % nstreams]
    batches = [Batch([(gfilter(ci, n), clips[ci]["src"][n].data_ptr(), clips[ci]["dst"][n].data_ptr())
                      for ci, n in call]) for call in calls]
    gst = [torch.cuda.Stream() for _ in range(2)]

    def gstep(record=None):
        for k, bt in enumerate(batches):
            s_ = gst[k % 2]
            a = torch.cuda.Event(enable_timing=True)
            a.record(s_)
            bt.launch(s_.cuda_stream)
            z = torch.cuda.Event(enable_timing=True)
            z.record(s_)
            if record is not None:
                record.append((a, z))

    for _ in range(max(warmup, 1)):
        gstep()
    torch.cuda.synchronize()
    for bt in batches:
        bt.status()
    g0 = torch.cuda.Event(enable_timing=True)
    g0.record(gst[0])
    gst[1].wait_event(g0)
    grec = []
    for _ in range(steps):
        gstep(grec)
    e1 = torch.cuda.Event()
    e1.record(gst[1])
    gst[0].wait_event(e1)
    g1 = torch.cuda.Event(enable_timing=True)
    g1.record(gst[0])
    g1.synchronize()
    for bt in batches:
        bt.status()
    gms = g0.elapsed_time(g1)
    glat = np.array([a.elapsed_time(z) for a, z in grec])
    batch_form["graph"] = {"value": px / (gms / 1e3) / 1e6, "unit": "Mpix/s", "ms_per_step": gms / steps,
                           "latency_ms_p50": float(np.percentile(glat, 50)),
                           "latency_ms_p99": float(np.percentile(glat, 99)),
                           "how": f"{len(batches)} batches of {per_call} windows captured once each "
                                  "(zb3d_batch_create), replayed round-robin on 2 streams; CUDA events"}
    for bt in batches:
        bt.close()
    for fl in gfil.values():
        for f in fl:
            f.close()
    per_clip = []
    for ci, c in enumerate(clips):
        l = np.array(lat[ci])
        per_clip.append({"clip": f"{c['w']}x{c['h']} {'YUV444 CBM3D' if c['chroma'] else 'YUV420'} r{c['radius']}",
                         "sigma": round(c["sigma"], 2), "frames": nfr,
                         "latency_ms_p50": float(np.percentile(l, 50)), "latency_ms_p99": float(np.percentile(l, 99)),
                         "matching": [list(f) for f in (c["filters"][0].tuning(e) for e in range(len(c["filters"][0].entries)))]})
    for c in clips:
        for f in c["filters"]:
            f.close()
    return {"metric": "batched uneven BM3D Mpix/s (luma)", "value": px / (ms / 1e3) / 1e6, "unit": "Mpix/s",
            "ms_per_step": ms / steps, "steps": steps, "warmup": warmup,
            "config": {"workload": "4 clips x 16 frames: 720x480 YUV420 r0, 1280x720 YUV444 CBM3D r0, 1280x720 "
                                   "YUV420 r1 (stacked output), 3840x2160 YUV420 r0; sigma U[5,20] per clip; "
                                   "block_step 4, bm_range 12, single pass", "streams": nstreams,
                       "launch": "one CUDA graph per window (all planes' memsets, matching, filtering, finishing)",
                       "per_clip": per_clip},
            "batch_form": batch_form}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=8)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-ref-cuda", action="store_true")
    ap.add_argument("--no-forms", action="store_true", help="skip timing the other block-matching form")
    ap.add_argument("--no-pilot", action="store_true", help="skip the learned-pilot form")
    ap.add_argument("--no-workloads", action="store_true",
                    help="skip the short runs of the other workloads (gray640, vbm3d, batched, pilot4k)")
    ap.add_argument("--pilot-weights", default=None, help="pilot weights (.npz) instead of the shipped ones")
    ap.add_argument("--pilot-conv-ctas", type=int, default=4,
                    help="cap on the CTAs per SM of the pilot's convolutions (1 leaves room for step 2 of "
                         "other frames)")
    ap.add_argument("--streams", type=int, default=4, help="CUDA streams the device pipeline spreads frames over")
    ap.add_argument("--match-form", type=int, choices=[-1, 0, 1], default=-1,
                    help="block matching: -1 = the library's autotuned choice per plane, 0 = FP32 scan of every "
                         "candidate, 1 = tensor-core bound + exact re-rank")
    ap.add_argument("--precision", action="store_true",
                    help="vbm3d: the precision form of the filter (2D transforms on the tensor cores, split TF32), "
                         "with its error against the plain form and the FP64 oracle")
    ap.add_argument("--workload", choices=["twopass1080", "vbm3d", "gray640", "batched", "pilot4k", "dct_tf32",
                                           "match1080"],
                    default="twopass1080",
                    help="twopass1080 is the metric's workload; the others print their own line")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.match_form >= 0:
        KW["match_form"] = args.match_form

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return reference_arm(args, rank, world)

    import torch
    torch.cuda.set_device(local)
    if args.workload != "twopass1080":
        fn = {"vbm3d": run_vbm3d, "gray640": run_gray640, "batched": run_batched, "pilot4k": run_pilot4k,
              "dct_tf32": run_dct_tf32, "match1080": run_match1080}[args.workload]
        out = fn(torch, args.steps, args.warmup, filter_form=1) if args.precision and args.workload == "vbm3d" \
            else fn(torch, args.steps, args.warmup)
        for k, v in {"n_gpus": 1, "higher_is_better": True, "dtype": "f32", "data": "synthetic"}.items():
            out.setdefault(k, v)
        print(json.dumps(out))
        return 0
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    from zb3d import _native as N
    from zb3d import shard
    N.lib()
    # one clip of FRAMES_PER_GPU frames per rank, sharded into contiguous output ranges
    # (radius 0: a rank's source frames are its output frames); each rank stages the first
    # DISTINCT frames of its range and cycles them through its FRAMES_PER_GPU buffers
    clip_frames = FRAMES_PER_GPU * world
    first, last = shard.source_range(clip_frames, world, rank)
    assert (first, last) == shard.output_range(clip_frames, world, rank) and last - first == FRAMES_PER_GPU
    frames = synth_frames(0, DISTINCT, first=first)
    pipe = DevicePipeline(torch, args.streams)
    pipe.upload(frames, FRAMES_PER_GPU)
    # warm-up: every frame buffer once (each buffer pair's launch graph is captured on first
    # use), then W steps
    pipe.timed(FRAMES_PER_GPU // BATCH)
    pipe.timed(args.warmup)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clocks = ClockSampler(local)
    clocks.start()
    ms = pipe.timed(args.steps, start_frame=args.warmup * BATCH)
    clk = clocks.stop()
    torch.cuda.synchronize()
    # roofline pass: one batch on one stream with CUDA events around every launch,
    # so each matching launch is timed alone
    pipe.profile(True)
    for j in range(BATCH):
        pipe.run_frame(0, j)
    torch.cuda.synchronize()
    pipe.profile(False)
    match_ms, match_n, filt_ms, filt_n = pipe.collect()
    if dist:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    frames_done = args.steps * BATCH * world
    value = W * H * frames_done / (ms / 1e3) / 1e6

    # dominant kernel: block matching; algorithmic FLOPs per frame (both passes, three planes)
    flops_frame = 2 * sum(match_flops(w, h, BLOCK_STEP, BM_RANGE) for (w, h) in plane_dims())
    match_flops_total = flops_frame * BATCH
    sm_max = (clk or {}).get("sm_max_mhz") or 1965.0
    props = torch.cuda.get_device_properties(local)
    peak_fp32 = props.multi_processor_count * 128 * 2 * sm_max * 1e6 / 1e12
    achieved = match_flops_total / (match_ms / 1e3) / 1e12 if match_ms > 0 else None
    # DRAM bytes per matching launch: ncu measured 8.32 MB read and 0 written for the
    # 1920x1080 Y launch, which is the plane read once (4 B per pixel); scaled by plane
    # size to the average of the batch's Y, U and V launches
    plane_px = [w * h for (w, h) in plane_dims()]
    traffic = 8.32e6 * (sum(plane_px) / len(plane_px)) / plane_px[0]

    out = {"metric": METRIC, "value": value, "unit": "Mpix/s", "n_gpus": world, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f32",
           "data": "synthetic: seeded gradient + 20 rectangles + sinusoidal texture, N(0, 10/255) noise",
           "config": {"workload": WORKLOAD, "form": None,
                      "frames_per_gpu": FRAMES_PER_GPU, "batch_frames_per_step": BATCH,
                      "l2": f"inputs larger than L2: {FRAMES_PER_GPU} distinct frame buffers "
                            f"({FRAMES_PER_GPU * 2 * 12.4:.0f} MB) cycled",
                      "parallelism": f"frame shards of one {FRAMES_PER_GPU * world}-frame clip over {world} "
                                     f"GPU(s) (zb3d.shard ranges), no collective",
                      "streams": pipe.ns},
           "gpu_launches": pipe.launches_per_frame() * args.steps * BATCH,
           "roofline": {"bound": "fp32", "achieved": achieved, "peak": peak_fp32, "unit": "TFLOP/s",
                        "frac": (achieved / peak_fp32) if achieved else None, "traffic": traffic,
                        "traffic_how": "DRAM read + write bytes per launch from an ncu capture of the 1920x1080 Y "
                                       "launch (8.32 MB read, 0 written), scaled by plane size to the average "
                                       "launch; algorithmically the plane is read once",
                        "kernel": "zb_match_tiled2<shared, bs4> (block matching, packed FP32x2)",
                        "per_launch_ms": match_ms / max(match_n, 1), "launches": match_n,
                        "how": "algorithmic FLOP (192 per candidate, all clipped windows) of one batch's "
                               "matching launches / their CUDA-event time, one stream, after the timed region",
                        "peak_source": f"nominal FP32: {props.multi_processor_count} SMs x 128 lanes x 2 x "
                                       f"{sm_max:.0f} MHz (MEASURED_PEAKS.json has no FP32 figure)",
                        "filter_ms_per_launch": filt_ms / max(filt_n, 1)},
           "clocks": clk}
    tuned = [pipe.basic[0].tuning(e) for e in range(len(pipe.lay))]
    chosen = args.match_form if args.match_form >= 0 else tuned[0][0]
    out["config"]["form"] = FORM_NAMES[chosen] + ("" if args.match_form >= 0 else " (autotuned)")
    out["config"]["matching_per_plane"] = [{"plane": "YUV"[lay.plane[0]], "form": FORM_KEYS[fm], "rows_per_cta": rw}
                                           for lay, (fm, rw) in zip(pipe.lay, tuned)]
    if chosen == 1:
        out["roofline"]["kernel"] = "zb_match_tc (tensor-core bound + exact FP32 re-rank)"
    # each block-matching form forced on the same frames: same lists and outputs bit for bit
    forms = {}
    if args.match_form >= 0:
        forms[FORM_KEYS[args.match_form]] = {"value": value, "ms_per_step": ms / args.steps,
                                             "match_ms_per_launch": match_ms / max(match_n, 1)}
    for alt in ([] if args.no_forms or rank != 0 else [f for f in (0, 1) if f != args.match_form]):
        if pipe is not None:
            pipe.close()
            pipe = None
        KW["match_form"] = alt
        p2 = DevicePipeline(torch, args.streams)
        p2.upload(frames, FRAMES_PER_GPU)
        p2.timed(FRAMES_PER_GPU // BATCH)
        p2.timed(args.warmup)
        ms2 = p2.timed(args.steps, start_frame=args.warmup * BATCH)
        p2.profile(True)
        for j in range(BATCH):
            p2.run_frame(0, j)
        torch.cuda.synchronize()
        p2.profile(False)
        m2_ms, m2_n, _, _ = p2.collect()
        p2.close()
        forms[FORM_KEYS[alt]] = {"value": W * H * args.steps * BATCH / (ms2 / 1e3) / 1e6,
                                 "ms_per_step": ms2 / args.steps, "match_ms_per_launch": m2_ms / max(m2_n, 1)}
    KW.pop("match_form", None)
    if args.match_form >= 0:
        KW["match_form"] = args.match_form
    forms["note"] = ("both forms give bit-identical match lists and outputs (delta PSNR 0 dB); "
                     "tensor_core = tcgen05 FP16 distance bound in TMEM + exact FP32 re-rank")
    out["forms"] = forms
    # end to end through the public API, before the other forms fill the device and host pools
    if not args.no_e2e:
        if pipe is not None:
            pipe.close()
            pipe = None
        torch.cuda.empty_cache()
        dt, h2d, d2h = run_e2e(frames, args.steps, args.warmup)
        out["e2e"] = {"value": W * H * args.steps * BATCH * world / dt / 1e6, "unit": "Mpix/s",
                      "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                      "how": "zb3d.BM3Dv2 twice (basic, then ref=basic) on host frames in page-locked memory "
                             "(the library DMAs them; outputs land in pooled page-locked frames), 4 streams, "
                             "8 request threads, frames requested continuously, wall clock"}
        dt, h2d, d2h = run_e2e(frames, args.steps, args.warmup, pinned=False)
        out["e2e"]["pageable"] = {
            "value": W * H * args.steps * BATCH * world / dt / 1e6, "unit": "Mpix/s",
            "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
            "how": "the same two filters on pageable host frames (as VapourSynth frames are): the library "
                   "copies them through its page-locked staging buffers"}
    if rank == 0 and not args.no_pilot:
        if pipe is not None:
            pipe.close()
            pipe = None
        # timed over the same K steps as the plain form (8 frames each)
        out["pilot_form"] = run_pilot_form(torch, frames, 0, args.steps, 1, nstreams=args.streams,
                                           weights=args.pilot_weights, conv_ctas_per_sm=args.pilot_conv_ctas)
        if not args.no_e2e and args.pilot_weights is None:
            # the pilot form through the C ABI (zb3d_args.pilot, shipped file and gate) on host frames
            import zb3d
            torch.cuda.empty_cache()
            pl = zb3d.Pilot()
            dt, h2d, d2h = run_e2e(frames, args.steps, args.warmup, pilot=pl)
            out["pilot_form"]["e2e"] = {
                "value": W * H * args.steps * BATCH / dt / 1e6, "unit": "Mpix/s",
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "pilot_used_per_plane": [pl.accepts(SIGMA, w, h) for w, h in plane_dims()],
                "how": "zb3d.BM3Dv2(clip, pilot=zb3d.Pilot()) on host frames in page-locked memory: one filter "
                       "runs the pilot (its gate accepting sigma) and step 2 per frame, 4 streams, 8 request "
                       "threads, wall clock"}
        if args.pilot_weights is None:
            # the 48-channel, 10-layer net of the learned-pilot configuration, on the same frames
            from zb3d import pilot as P
            out["pilot_form_w48_l10"] = run_pilot_form(torch, frames, 0, args.steps, 1, nstreams=args.streams,
                                                       weights=P.WEIGHTS_W48_L10,
                                                       conv_ctas_per_sm=args.pilot_conv_ctas)
    if rank == 0 and not args.no_ref_cuda:
        if pipe is not None:
            pipe.close()
            pipe = None
        by_ns = {}
        for ns in (4, 2):
            rms = run_ref_cuda(torch, frames, args.steps, args.warmup, nstreams=ns)
            if rms:
                by_ns[ns] = (W * H * args.steps * BATCH / (rms / 1e3) / 1e6, rms / args.steps)
        if by_ns:
            rv = by_ns[max(by_ns)][0]
            out["ref_cuda"] = {"value": rv, "unit": "Mpix/s", "ms_per_step": by_ns[max(by_ns)][1],
                               "streams": max(by_ns),
                               "value_by_streams": {str(k): v[0] for k, v in sorted(by_ns.items())},
                               "what": "the reference's own bm3d.cu kernels (NVRTC-built, -use_fast_math) on "
                                       "this GPU, same frames, same two-pass chaining, device-resident; frames "
                                       "spread over the reference host's default 4 stream slots (2 shown too)",
                               "speedup_ours": value / world / rv}
            # the drop-in comparison in one place: this build's forms over the reference's kernels
            # (4 streams, device-resident on both sides; e2e runs through the public API)
            vs = {"ref_cuda_mpix_s": rv, "ref_cuda_streams": max(by_ns), "plain_x": value / world / rv}
            if "pilot_form" in out and out["pilot_form"].get("value"):
                vs["pilot_x"] = out["pilot_form"]["value"] / rv
                if out["pilot_form"].get("e2e"):
                    vs["pilot_e2e_pinned_x"] = out["pilot_form"]["e2e"]["value"] / rv
            if "e2e" in out:
                vs["e2e_pinned_x"] = out["e2e"]["value"] / world / rv
                if out["e2e"].get("pageable"):
                    vs["e2e_pageable_x"] = out["e2e"]["pageable"]["value"] / world / rv
            out["vs_reference_cuda"] = vs
    if pipe is not None:
        pipe.close()
    if rank == 0 and not args.no_workloads:
        # the other configurations of the path, each a short run of its own workload (the same
        # functions as --workload <name>), so that one default run carries their figures
        others = {}
        for name, fn in (("gray640", run_gray640), ("vbm3d", run_vbm3d),
                         ("vbm3d_precision", lambda t, s, w: run_vbm3d(t, s, w, filter_form=1)),
                         ("batched", run_batched), ("pilot4k", run_pilot4k)):
            torch.cuda.empty_cache()
            t0 = time.perf_counter()
            r = fn(torch, 4, 3)
            r["wall_s"] = round(time.perf_counter() - t0, 1)
            others[name] = r
        out["other_workloads"] = others
    if rank == 0 and not args.no_cpu:
        out["cpu_baseline"] = cpu_baseline(frames)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(out))
    return 0


if __name__ == "__main__":
    sys.exit(main())
