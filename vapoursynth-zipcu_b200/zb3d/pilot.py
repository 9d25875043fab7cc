"""Learned pilot: a residual conv net that stands in for BM3D's step-1 estimate.

BM3Dv2's second pass (Wiener) matches blocks on, and takes its empirical Wiener
coefficients from, a reference clip: normally the step-1 hard-threshold estimate.
The pilot produces that reference with a stack of 3x3 convolutions (16, 32 or 48
channels, ReLU, a noise-level input plane; output added to the noisy plane).  It is trained
only on pairs (noisy synthetic frame, plain BM3D step-1 output of it), on the GPU,
by the project's own kernels (csrc/zb3d_pilot.cu: BF16 operands, FP32
accumulation); inference runs on the tensor cores (csrc/zb3d_pilot_tc.cu: tcgen05.mma
with the accumulator in tensor memory, TMA-staged input rows).  Its forward and backward passes are checked against the numpy
oracle (oracle/pilot_oracle.py).  Step 2 keeps exact block matching; the plain
two-pass form remains the fallback: the gate accepts the pilot for a noise level and
plane size only where its two-pass PSNR is, on average over held-out synthetic planes,
within 0.05 dB of the plain two-pass PSNR (`PilotGate` here; for the C ABI the table
measured by `calibrate_file` travels inside the ZB3DPLT1 weights file that
zb3d_pilot_load reads, and BM3Dv2(pilot=...) decides per plane).

torch provides device memory and streams here; every operation on the data is a
zb3d kernel.
"""
from __future__ import annotations

import ctypes
import math
from collections import OrderedDict
from typing import Optional, Sequence

import numpy as np

from . import _native as N
from . import synth



def arch(width: int = 32, layers: int = 6) -> list:
    """(cin, cout) of each layer; the 2 input and 1 output channels are padded to 16."""
    return [(16, width)] + [(width, width)] * (layers - 2) + [(width, 16)]


SHAPES = arch(32, 7)                                 # the default (and shipped) architecture
REAL_IN, REAL_OUT = 2, 1
LEVEL_SCALE = 4.0                                    # noise-level plane = sigma / 255 * LEVEL_SCALE
LOSS_SCALE = 1024.0                                  # keeps BF16 gradients clear of underflow
WS_KEEP = 8                                          # inference buffer sets kept per network


def _p(t) -> int:
    return t.data_ptr() if t is not None else None


def _ok(rc: int, what: str):
    if rc != 0:
        raise RuntimeError(f"zb3d pilot: {what} failed")


class PilotNet:
    """The network, its FP32 master weights and Adam state, on one CUDA device."""

    def __init__(self, seed: int = 0, device: str = "cuda", width: int = 32, layers: int = 7):
        import torch
        self.torch, self.dev = torch, device
        self.width, self.layers = width, layers
        self.shapes = arch(width, layers)
        rng = np.random.default_rng(seed)
        self.w32, self.b32, self.keep = [], [], []
        for l, (cin, cout) in enumerate(self.shapes):
            rin = REAL_IN if l == 0 else cin
            rout = REAL_OUT if l == len(self.shapes) - 1 else cout
            std = math.sqrt(2.0 / (9 * rin)) * (0.1 if l == len(self.shapes) - 1 else 1.0)
            w = np.zeros((cout, 3, 3, cin), np.float32)
            w[:rout, :, :, :rin] = rng.normal(0.0, std, size=(rout, 3, 3, rin))
            k = np.zeros_like(w)
            k[:rout, :, :, :rin] = 1.0
            kb = np.zeros(cout, np.float32)
            kb[:rout] = 1.0
            self.w32.append(torch.from_numpy(w).to(device))
            self.b32.append(torch.zeros(cout, dtype=torch.float32, device=device))
            self.keep.append((torch.from_numpy(k).to(device), torch.from_numpy(kb).to(device)))
        self.w16 = [torch.empty(w.shape, dtype=torch.bfloat16, device=device) for w in self.w32]
        self.wt16 = [torch.empty((cin, 3, 3, cout), dtype=torch.bfloat16, device=device) for cin, cout in self.shapes]
        # inference activation buffers per (n, h, w, stream), reused across calls; the least
        # recently used shapes are dropped beyond WS_KEEP
        self._ws: "OrderedDict[tuple, list]" = OrderedDict()
        self.m = [(torch.zeros_like(w), torch.zeros_like(b)) for w, b in zip(self.w32, self.b32)]
        self.v = [(torch.zeros_like(w), torch.zeros_like(b)) for w, b in zip(self.w32, self.b32)]
        self.step_count = 0
        self._refresh()

    # -- weights ---------------------------------------------------------------------
    def _refresh(self):
        lib = N.lib()
        for l, (cin, cout) in enumerate(self.shapes):
            _ok(lib.zb3d_pilot_to_bf16(_p(self.w32[l]), self.w32[l].numel(), _p(self.w16[l]), None), "to_bf16")
            _ok(lib.zb3d_pilot_flip_weights(_p(self.w16[l]), cin, cout, _p(self.wt16[l]), None), "flip")

    def state(self) -> dict:
        out = {"arch": np.array([self.width, self.layers], np.int32)}
        for l in range(len(self.shapes)):
            out[f"w{l}"] = self.w32[l].cpu().numpy()
            out[f"b{l}"] = self.b32[l].cpu().numpy()
        return out

    def load_state(self, st: dict):
        torch = self.torch
        for l in range(len(self.shapes)):
            self.w32[l].copy_(torch.from_numpy(np.asarray(st[f"w{l}"], np.float32)))
            self.b32[l].copy_(torch.from_numpy(np.asarray(st[f"b{l}"], np.float32)))
        self._refresh()

    def save(self, path: str):
        np.savez_compressed(path, **self.state())

    @classmethod
    def load(cls, path: str, device: str = "cuda") -> "PilotNet":
        with np.load(path) as f:
            st = {k: f[k] for k in f.files}
        width, layers = (int(v) for v in st.get("arch", (48, 10)))
        net = cls(device=device, width=width, layers=layers)
        net.load_state(st)
        return net

    # -- passes ------------------------------------------------------------------------
    def forward(self, noisy, sigma, keep_acts: bool = False, out=None, stream=None, tc: Optional[bool] = None):
        """noisy: float32 [n][h][w] device tensor, sigma: float32 [n] (8-bit scale).
        Returns y = noisy + net output (float32 [n][h][w], written to `out` if given)
        and, with keep_acts, the stored BF16 activations of every layer's input (NHWC, or
        channel-blocked [n][c/8][h][w][8] with tc).
        `stream`: a CUDA stream handle (int) for every launch, or None for torch's current
        stream; it must be torch's current stream (e.g. inside `torch.cuda.stream(s)`), so
        that the allocator orders the reuse of this call's buffers after its kernels.
        tc: convolutions on the tensor cores (tcgen05); default for inference (no keep_acts),
        while the training passes keep the mma.sync kernels their gradients are checked with."""
        torch, lib = self.torch, N.lib()
        if tc is None:
            tc = not keep_acts
        current = torch.cuda.current_stream().cuda_stream
        if stream is None:
            stream = current or None  # the legacy default stream is NULL
        elif stream != current:
            raise ValueError("zb3d pilot: stream must be torch's current stream")
        n, h, w = noisy.shape
        y = out if out is not None else torch.empty((n, h, w), dtype=torch.float32, device=self.dev)
        for t, what in ((noisy, "noisy"), (y, "out")):
            # images may sit any distance apart (e.g. inside [reference | noisy] frame buffers);
            # each image must be dense, and strided images need the tensor-core path
            if tuple(t.shape) != (n, h, w) or t.stride(1) != w or t.stride(2) != 1 or \
                    (not tc and n > 1 and t.stride(0) != h * w):
                raise ValueError(f"zb3d pilot: {what} must be [n][h][w] with dense images")

        def img_stride(t):  # floats between images (a single image's leading stride is arbitrary)
            return t.stride(0) if n > 1 else h * w

        def act(c):  # NHWC for the mma.sync kernels, channel-blocked [n][c/8][h][w][8] for tcgen05
            shape = (n, c // 8, h, w, 8) if tc else (n, h, w, c)
            return torch.empty(shape, dtype=torch.bfloat16, device=self.dev)

        reuse = tc and not keep_acts
        if reuse:
            # input and two ping-pong activation buffers, private to the stream that uses them
            key = (n, h, w, stream)
            if key not in self._ws:
                self._ws[key] = [act(16), act(self.width), act(self.width)]
                while len(self._ws) > WS_KEEP:
                    # the dropped buffers were allocated on, and used on, the stream of their
                    # key, so the allocator orders any reuse of their memory after their kernels
                    self._ws.popitem(last=False)
            self._ws.move_to_end(key)
            ws = self._ws[key]
        x = ws[0] if reuse else act(16)
        if tc:
            rc = lib.zb3d_pilot_pack_input_blocked(_p(noisy), img_stride(noisy), _p(sigma), n, h, w, LEVEL_SCALE,
                                                   _p(x), stream)
        else:
            rc = lib.zb3d_pilot_pack_input(_p(noisy), _p(sigma), n, h, w, LEVEL_SCALE, _p(x), stream)
        _ok(rc, "pack_input")
        acts = [x]
        last = len(self.shapes) - 1

        def conv(x_, l, relu, a_, y0_, resid_):
            cin, cout = self.shapes[l]
            if tc:
                return lib.zb3d_pilot_conv3x3_tc(_p(x_), n, h, w, cin, _p(self.w16[l]), _p(self.b32[l]), cout, relu,
                                                 _p(a_), _p(y0_), _p(resid_), img_stride(y), img_stride(noisy), None,
                                                 stream)
            return lib.zb3d_pilot_conv3x3(_p(x_), n, h, w, cin, _p(self.w16[l]), _p(self.b32[l]), cout, relu,
                                          None, _p(a_), _p(y0_), _p(resid_), stream)

        for l, (cin, cout) in enumerate(self.shapes):
            if l < last:
                a = ws[1 + (l & 1)] if reuse else act(cout)  # hidden layers: cout == width
                _ok(conv(acts[-1], l, 1, a, None, None), f"conv {l}")
                if keep_acts:
                    acts.append(a)
                else:
                    acts = [a]
            else:
                _ok(conv(acts[-1], l, 0, None, y, noisy), "conv out")
        return y, (acts if keep_acts else None)

    def gradients(self, noisy, target, sigma):
        """Loss-scaled gradients (dw, db per layer) of mean (y - target)^2, and the loss."""
        torch, lib = self.torch, N.lib()
        n, h, w = noisy.shape
        y, acts = self.forward(noisy, sigma, keep_acts=True)
        # per-CTA FP32 sums of squared errors, added up on the host (no FP64 on the GPU)
        partials = torch.empty((y.numel() + 255) // 256, dtype=torch.float32, device=self.dev)
        d = torch.empty((n, h, w, 16), dtype=torch.bfloat16, device=self.dev)
        _ok(lib.zb3d_pilot_mse_grad(_p(y), _p(target), y.numel(), LOSS_SCALE, _p(d), _p(partials), None),
            "mse_grad")
        dws = [torch.zeros_like(wt) for wt in self.w32]
        dbs = [torch.zeros_like(b) for b in self.b32]
        for l in range(len(self.shapes) - 1, -1, -1):
            cin, cout = self.shapes[l]
            _ok(lib.zb3d_pilot_conv3x3_wgrad(_p(acts[l]), _p(d), n, h, w, cin, cout, _p(dws[l]), _p(dbs[l]), None),
                f"wgrad {l}")
            if l == 0:
                break
            dx = torch.empty((n, h, w, cin), dtype=torch.bfloat16, device=self.dev)
            # backward pass to the layer input (= previous layer's output): conv with the flipped
            # weights, ReLU derivative from the stored activation
            _ok(lib.zb3d_pilot_conv3x3(_p(d), n, h, w, cout, _p(self.wt16[l]), None, cin, 0, _p(acts[l]), _p(dx),
                                       None, None, None), f"dgrad {l}")
            d = dx
        loss = float(partials.cpu().numpy().astype(np.float64).sum())
        return dws, dbs, loss / y.numel(), y

    def train_step(self, noisy, target, sigma, lr: float = 1e-3) -> float:
        lib = N.lib()
        dws, dbs, loss, _ = self.gradients(noisy, target, sigma)
        self.step_count += 1
        for l in range(len(self.shapes)):
            for p, g, m, v, k, w16 in ((self.w32[l], dws[l], self.m[l][0], self.v[l][0], self.keep[l][0], self.w16[l]),
                                       (self.b32[l], dbs[l], self.m[l][1], self.v[l][1], self.keep[l][1], None)):
                _ok(lib.zb3d_pilot_adam(_p(p), _p(m), _p(v), _p(g), p.numel(), lr, 0.9, 0.999, 1e-8,
                                        self.step_count, LOSS_SCALE, _p(k), _p(w16), None), "adam")
        for l, (cin, cout) in enumerate(self.shapes):
            _ok(lib.zb3d_pilot_flip_weights(_p(self.w16[l]), cin, cout, _p(self.wt16[l]), None), "flip")
        return loss

    def denoise(self, plane: np.ndarray, sigma: float) -> np.ndarray:
        """The pilot estimate of one float32 plane (host in, host out)."""
        torch = self.torch
        x = torch.from_numpy(np.ascontiguousarray(plane, np.float32))[None].to(self.dev)
        s = torch.tensor([sigma], dtype=torch.float32, device=self.dev)
        y, _ = self.forward(x, s)
        return y[0].cpu().numpy()


# ---------------------------------------------------------------------------------------
# training data: (noisy synthetic frame, plain BM3D step-1 estimate) pairs
# ---------------------------------------------------------------------------------------
def step1_estimates(noisy: Sequence[np.ndarray], sigma: float, **bm3d_kw) -> list:
    """Plain BM3D step 1 (hard threshold, the reference's defaults unless given) of each plane."""
    import zb3d
    h, w = noisy[0].shape
    clip = zb3d.Clip.from_frames([[p] for p in noisy])
    basic = zb3d.BM3D(clip, sigma=sigma, **bm3d_kw)
    return [np.array(basic.get_frame(i)[0]) for i in range(len(noisy))]


def make_pairs(count: int, size, sigmas: Sequence[float], seed: int = 1, clip0: int = 1000, **bm3d_kw):
    """`count` frames per sigma of size x size (or (width, height)): (noisy, step-1, clean, sigma) lists."""
    w, h = (size, size) if isinstance(size, int) else size
    noisy, target, clean, sig = [], [], [], []
    for si, s in enumerate(sigmas):
        fr = [synth.noisy_plane(w, h, s, clip=clip0 + seed * 100 + si, frame=f) for f in range(count)]
        cl = [synth.clean_plane(w, h, clip0 + seed * 100 + si, f) for f in range(count)]
        noisy += fr
        clean += cl
        target += step1_estimates(fr, s, **bm3d_kw)
        sig += [float(s)] * count
    return noisy, target, clean, sig


def detail_weights(target, strength: float) -> np.ndarray:
    """Sampling weights of the training frames: 1 + strength x (the frame's mean squared
    Laplacian of its step-1 target, over the mean of all frames).  Frames with fine texture,
    which step 1 keeps and a small net tends to smooth, are drawn more often."""
    hf = []
    for t in target:
        t = np.asarray(t, np.float64)
        lap = 4.0 * t[1:-1, 1:-1] - t[:-2, 1:-1] - t[2:, 1:-1] - t[1:-1, :-2] - t[1:-1, 2:]
        hf.append(float(np.mean(lap * lap)))
    hf = np.asarray(hf)
    w = 1.0 + strength * hf / max(float(hf.mean()), 1e-30)
    return w / w.sum()


def train(net: PilotNet, noisy, target, sigma, steps: int, batch: int = 32, crop: int = 64, lr: float = 1e-3,
          seed: int = 0, log_every: int = 0, frame_weights=None) -> list:
    """Adam on random crop x crop patches of the pairs; returns the loss history.
    frame_weights: sampling probability of each pair's frame (None = uniform)."""
    torch = net.torch
    rng = np.random.default_rng(seed)
    dn = [torch.from_numpy(np.ascontiguousarray(a, np.float32)).to(net.dev) for a in noisy]
    dt = [torch.from_numpy(np.ascontiguousarray(a, np.float32)).to(net.dev) for a in target]
    hist = []
    for it in range(steps):
        if frame_weights is None:
            idx = rng.integers(0, len(dn), size=batch)
        else:
            idx = rng.choice(len(dn), size=batch, p=frame_weights)
        xs, ts = [], []
        for i in idx:
            h, w = dn[i].shape
            y0, x0 = rng.integers(0, h - crop + 1), rng.integers(0, w - crop + 1)
            xs.append(dn[i][y0:y0 + crop, x0:x0 + crop])
            ts.append(dt[i][y0:y0 + crop, x0:x0 + crop])
        xb = torch.stack(xs).contiguous()
        tb = torch.stack(ts).contiguous()
        sb = torch.tensor([sigma[i] for i in idx], dtype=torch.float32, device=net.dev)
        lr_t = lr * 0.5 * (1.0 + math.cos(math.pi * it / max(steps, 1)))
        hist.append(net.train_step(xb, tb, sb, lr=lr_t))
        if log_every and it % log_every == 0:
            print(f"step {it} loss {hist[-1]:.3e}")
    return hist


# ---------------------------------------------------------------------------------------
# two-pass BM3Dv2 with the plain step 1 or the pilot, and the 0.05 dB gate
# ---------------------------------------------------------------------------------------
def two_pass(noisy: np.ndarray, sigma: float, ref: Optional[np.ndarray] = None, **kw) -> np.ndarray:
    """BM3Dv2 step 2 (Wiener) of a float32 plane with `ref` as its reference; ref None = plain step 1."""
    import zb3d
    clip = zb3d.Clip.from_frames([[noisy]])
    if ref is None:
        ref = np.array(zb3d.BM3Dv2(clip, sigma=sigma, **kw).get_frame(0)[0])
    rclip = zb3d.Clip.from_frames([[np.ascontiguousarray(ref, np.float32)]])
    return np.array(zb3d.BM3Dv2(clip, ref=rclip, sigma=sigma, **kw).get_frame(0)[0])


class PilotGate:
    """Per noise level: use the pilot only where its two-pass PSNR is within `tol` dB
    of the plain two-pass PSNR on held-out synthetic frames."""

    def __init__(self, net: PilotNet, tol: float = 0.05):
        self.net, self.tol = net, tol
        self.delta: dict = {}

    def calibrate(self, sigmas: Sequence[float], frames: int = 2, size=256, seed: int = 99, **kw) -> dict:
        """Measure the two-pass difference per noise level on held-out synthetic frames of
        `size` (or (width, height)): calibrate at the frame size the gate will serve, since
        the synthetic content's scale changes with it."""
        w, h = (size, size) if isinstance(size, int) else size
        for si, s in enumerate(sigmas):
            d = []
            for f in range(frames):
                cl = synth.clean_plane(w, h, 5000 + seed + si, f)
                nz = synth.noisy_plane(w, h, s, clip=5000 + seed + si, frame=f)
                plain = two_pass(nz, s, **kw)
                piloted = two_pass(nz, s, ref=self.net.denoise(nz, s), **kw)
                d.append(synth.psnr(piloted, cl) - synth.psnr(plain, cl))
            self.delta[float(s)] = float(np.mean(d))
        return dict(self.delta)

    def accepts(self, sigma: float) -> bool:
        if not self.delta:
            return False
        near = min(self.delta, key=lambda s: abs(s - sigma))
        return self.delta[near] >= -self.tol

    def reference(self, noisy: np.ndarray, sigma: float, **kw) -> np.ndarray:
        """Step 2's reference: the pilot where accepted, else the plain step 1."""
        if self.accepts(sigma):
            return self.net.denoise(noisy, sigma)
        import zb3d
        return np.array(zb3d.BM3Dv2(zb3d.Clip.from_frames([[noisy]]), sigma=sigma, **kw).get_frame(0)[0])


# ---------------------------------------------------------------------------------------
# the weights file of the C ABI (zb3d_pilot_load): "ZB3DPLT1"
# ---------------------------------------------------------------------------------------
import os as _os
import struct as _struct
import zlib as _zlib

MAGIC = b"ZB3DPLT1"


def save_weights(path: str, state, gate: Sequence = (), gate_frames: int = 0, tol: float = 0.05,
                 level_scale: float = LEVEL_SCALE) -> None:
    """Write the weights of `state` (PilotNet.state() or a loaded .npz: arch, w{l}, b{l})
    with the gate table [(sigma, plane width, plane height, two-pass delta dB), ...] as the
    ZB3DPLT1 file that zb3d_pilot_load reads (layout in csrc/zb3d_pilot_net.cpp), CRC-32 last."""
    width, layers = (int(v) for v in np.asarray(state["arch"]).ravel()[:2])
    shapes = arch(width, layers)
    out = bytearray(MAGIC)
    out += _struct.pack("<IIIf", 1, width, layers, float(level_scale))
    out += _struct.pack("<IfI", int(gate_frames), float(tol), len(gate))
    for s, gw, gh, d in gate:
        out += _struct.pack("<fIIf", float(s), int(gw), int(gh), float(d))
    for l, (cin, cout) in enumerate(shapes):
        w = np.asarray(state[f"w{l}"], np.float32)
        b = np.asarray(state[f"b{l}"], np.float32)
        if w.shape != (cout, 3, 3, cin) or b.shape != (cout,):
            raise ValueError(f"zb3d pilot: layer {l} has shape {w.shape}/{b.shape}, expected {(cout, 3, 3, cin)}")
        out += np.ascontiguousarray(w).astype("<f4").tobytes() + np.ascontiguousarray(b).astype("<f4").tobytes()
    out += _struct.pack("<I", _zlib.crc32(bytes(out)) & 0xFFFFFFFF)
    tmp = path + ".tmp"
    with open(tmp, "wb") as f:
        f.write(bytes(out))
    _os.replace(tmp, path)


def read_weights(path: str) -> dict:
    """Parse a ZB3DPLT1 file: {arch, version, level_scale, gate_frames, tol, gate, w{l}, b{l}}."""
    with open(path, "rb") as f:
        data = f.read()
    if data[:8] != MAGIC:
        raise ValueError("zb3d pilot: not a ZB3DPLT1 weights file")
    if _zlib.crc32(data[:-4]) & 0xFFFFFFFF != _struct.unpack("<I", data[-4:])[0]:
        raise ValueError("zb3d pilot: weights checksum mismatch")
    at = 8
    version, width, layers, level = _struct.unpack_from("<IIIf", data, at)
    at += 16
    gf, tol, ng = _struct.unpack_from("<IfI", data, at)
    at += 12
    gate = [_struct.unpack_from("<fIIf", data, at + 16 * i) for i in range(ng)]
    at += 16 * ng
    st = {"arch": np.array([width, layers], np.int32), "version": version, "level_scale": level,
          "gate_frames": gf, "tol": tol, "gate": gate}
    for l, (cin, cout) in enumerate(arch(width, layers)):
        n = cout * 9 * cin
        st[f"w{l}"] = np.frombuffer(data, "<f4", n, at).reshape(cout, 3, 3, cin).copy()
        at += 4 * n
        st[f"b{l}"] = np.frombuffer(data, "<f4", cout, at).copy()
        at += 4 * cout
    if at != len(data) - 4:
        raise ValueError("zb3d pilot: weights size does not match the architecture")
    return st


GATE_SIGMAS = (5.0, 7.5, 10.0, 12.5, 15.0, 20.0, 25.0)
GATE_SIZES = ((1920, 1080), (960, 540))   # the planes of 1080p YUV420


def gate_deltas(pilot, sigmas=GATE_SIGMAS, sizes=GATE_SIZES, frames: int = 16, seed: int = 0, **kw) -> list:
    """Per plane size and noise level, the two-pass PSNR difference of each of `frames`
    held-out synthetic planes: BM3Dv2 with the pilot as step 1 (a zb3d.Pilot whose gate
    accepts everything) minus the plain BM3Dv2 two-pass.  kw: BM3Dv2 arguments.
    Returns [(sigma, w, h, [delta per plane])]."""
    import zb3d
    rows = []
    for zi, (w, h) in enumerate(sizes):
        for si, s in enumerate(sigmas):
            d = []
            for fr in range(frames):
                c = 20000 + 1000 * seed + 200 * zi + 20 * si + fr  # frames < 20 per level stay distinct
                cl = synth.clean_plane(w, h, c, 0)
                clip = zb3d.Clip.from_frames([[synth.noisy_plane(w, h, s, clip=c, frame=0)]])
                basic = zb3d.BM3Dv2(clip, sigma=s, **kw)
                plain = np.array(zb3d.BM3Dv2(clip, ref=basic, sigma=s, **kw).get_frame(0)[0])
                piloted = np.array(zb3d.BM3Dv2(clip, sigma=s, pilot=pilot, **kw).get_frame(0)[0])
                d.append(synth.psnr(piloted, cl) - synth.psnr(plain, cl))
            rows.append((float(s), w, h, d))
    return rows


def calibrate_file(weights_npz: str, out: str, sigmas=GATE_SIGMAS, sizes=GATE_SIZES, frames: int = 16,
                   seed: int = 0, tol: float = 0.05, **kw) -> list:
    """Measure the gate of a trained net through the C ABI and write its ZB3DPLT1 file:
    per plane size and noise level, the mean two-pass difference over `frames` held-out
    planes (gate_deltas).  Returns [(sigma, w, h, mean delta dB, per-plane deltas)]."""
    import zb3d
    with np.load(weights_npz) as f:
        st = {k: f[k] for k in f.files}
    # provisional file that accepts every level, to measure the pilot itself
    save_weights(out, st, gate=[(s, w, h, 0.0) for w, h in sizes for s in sigmas], gate_frames=frames, tol=tol)
    pilot = zb3d.Pilot(out)
    rows = gate_deltas(pilot, sigmas, sizes, frames, seed, **kw)
    del pilot
    save_weights(out, st, gate=[(s, w, h, float(np.mean(d))) for s, w, h, d in rows], gate_frames=frames, tol=tol)
    return [(s, w, h, float(np.mean(d)), d) for s, w, h, d in rows]


# ---------------------------------------------------------------------------------------
# the shipped pilot
# ---------------------------------------------------------------------------------------

# 32 ch x 7 layers, trained by `python -m zb3d.pilot train` with its defaults
WEIGHTS = _os.path.join(_os.path.dirname(_os.path.abspath(__file__)), "pilot_bs4_r12.npz")
# the 48-channel, 10-layer net, trained by
# `python -m zb3d.pilot train --width 48 --layers 10` (the default data, steps and detail weighting)
WEIGHTS_W48_L10 = _os.path.join(_os.path.dirname(_os.path.abspath(__file__)), "pilot_w48_l10_bs4_r12.npz")
# 48 ch x 10 layers trained on 3840x2160 planes:
# `python -m zb3d.pilot train --width 48 --layers 10 --dims 3840x2160 --frames 8`
WEIGHTS_4K = _os.path.join(_os.path.dirname(_os.path.abspath(__file__)), "pilot_w48_l10_4k_bs4_r12.npz")
# the default net with its gate, for the C ABI: `python -m zb3d.pilot export` (gate measured
# on 16 held-out 1920x1080 and 960x540 planes per level)
WEIGHTS_BIN = _os.path.join(_os.path.dirname(_os.path.abspath(__file__)), "pilot_bs4_r12.zb3dp")
TRAIN_KW = dict(block_step=4, bm_range=12)   # step-1 configuration the shipped pilot imitates
TRAIN_SIGMAS = (5.0, 10.0, 15.0, 20.0, 25.0)


def shipped(device: str = "cuda", width: int = 32, layers: int = 7) -> PilotNet:
    """A pilot trained by `python -m zb3d.pilot train` (weights next to this file): the
    default 32 ch x 7 layers, or 48 ch x 10 layers."""
    paths = {(32, 7): WEIGHTS, (48, 10): WEIGHTS_W48_L10}
    if (width, layers) not in paths:
        raise ValueError(f"no shipped pilot of {width} channels x {layers} layers")
    return PilotNet.load(paths[(width, layers)], device=device)


def evaluate(net: PilotNet, sigmas=TRAIN_SIGMAS, frames: int = 4, size: int = 384, seed: int = 77, **kw) -> list:
    """Held-out synthetic frames: PSNR against the clean frame of the noisy input, plain
    step 1, the pilot, plain two-pass and pilot two-pass."""
    rows = []
    for si, s in enumerate(sigmas):
        acc = np.zeros(5)
        for f in range(frames):
            cl = synth.clean_plane(size, size, 9000 + seed + si, f)
            nz = synth.noisy_plane(size, size, s, clip=9000 + seed + si, frame=f)
            st1 = step1_estimates([nz], s, **kw)[0]
            pe = net.denoise(nz, s)
            acc += [synth.psnr(nz, cl), synth.psnr(st1, cl), synth.psnr(pe, cl),
                    synth.psnr(two_pass(nz, s, ref=st1, **kw), cl), synth.psnr(two_pass(nz, s, ref=pe, **kw), cl)]
        rows.append((float(s), *(acc / frames)))
    return rows


def time_kernels(width_layers=((32, 6), (48, 10)), w: int = 1920, h: int = 1080, reps: int = 20) -> list:
    """CUDA-event times of the inference convolution per layer shape on one w x h plane
    (tcgen05 and mma.sync), and of whole nets on a YUV420 frame (the plane plus two
    half-size planes).  Lines of text."""
    import torch
    lib = N.lib()

    def timeit(fn, n):
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(n):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / n

    out = []
    shapes = sorted({s for wd, ly in width_layers for s in arch(wd, ly)})
    for cin, cout in shapes:
        xb = torch.randn((1, cin // 8, h, w, 8), device="cuda").to(torch.bfloat16)
        xn = torch.randn((1, h, w, cin), device="cuda").to(torch.bfloat16)
        wt = (torch.randn((cout, 3, 3, cin), device="cuda") * 0.05).to(torch.bfloat16)
        b = torch.zeros(cout, device="cuda")
        yb = torch.empty((1, cout // 8, h, w, 8), dtype=torch.bfloat16, device="cuda")
        yn = torch.empty((1, h, w, cout), dtype=torch.bfloat16, device="cuda")
        st = torch.zeros(1, dtype=torch.int32, device="cuda")
        ttc = timeit(lambda: _ok(lib.zb3d_pilot_conv3x3_tc(_p(xb), 1, h, w, cin, _p(wt), _p(b), cout, 1, _p(yb), None,
                                                           None, 0, 0, _p(st), None), "conv tc"), reps)
        tmm = timeit(lambda: _ok(lib.zb3d_pilot_conv3x3(_p(xn), 1, h, w, cin, _p(wt), _p(b), cout, 1, None, _p(yn),
                                                        None, None, None), "conv"), reps)
        if int(st.item()) != 0:
            raise RuntimeError("zb3d pilot: tensor-core convolution reported a pipeline timeout")
        fl, by = 2.0 * h * w * 9 * cin * cout, h * w * 2.0 * (cin + cout)
        out.append(f"conv {cin}->{cout} {w}x{h}: tcgen05 {ttc * 1e3:7.1f} us ({fl / ttc / 1e9:6.1f} TFLOP/s, "
                   f"{by / ttc / 1e6:6.0f} GB/s)   mma.sync {tmm * 1e3:7.1f} us ({fl / tmm / 1e9:6.1f} TFLOP/s)")
    for wd, ly in width_layers:
        net = PilotNet(seed=0, width=wd, layers=ly)
        y = torch.rand((1, h, w), device="cuda")
        c = torch.rand((1, h // 2, w // 2), device="cuda")
        s1 = torch.tensor([10.0], device="cuda")

        def frame(tc):
            net.forward(y, s1, tc=tc)
            net.forward(c, s1, tc=tc)
            net.forward(c, s1, tc=tc)
        out.append(f"net {wd} ch x {ly} layers per {w}x{h} YUV420 frame: tcgen05 {timeit(lambda: frame(True), 10):.3f} ms"
                   f"   mma.sync {timeit(lambda: frame(False), 5):.3f} ms")
    return out


def main(argv=None):
    import argparse
    ap = argparse.ArgumentParser(prog="python -m zb3d.pilot")
    ap.add_argument("cmd", choices=["train", "eval", "time", "export"])
    ap.add_argument("--frames", type=int, default=32, help="training frames per noise level and frame size")
    ap.add_argument("--dims", default="1920x1080,1920x1080,1920x1080,960x540",
                    help="training frame sizes of the 1080p YUV420 planes; a size listed k times contributes k "
                         "sets of frames (luma-sized planes weigh 3:1 by default)")
    ap.add_argument("--steps", type=int, default=50000, help="Adam steps of 32 crops (50000 = 1.6M crops)")
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--width", type=int, default=32, help="channels of the hidden layers (16, 32 or 48)")
    ap.add_argument("--layers", type=int, default=7, help="number of 3x3 convolutions")
    ap.add_argument("--detail", type=float, default=4.0,
                    help="draw frames with more fine detail (step-1 Laplacian energy) more often: weight "
                         "1 + detail x energy / mean energy")
    ap.add_argument("--out", default=WEIGHTS)
    ap.add_argument("--weights", default=WEIGHTS, help="export: the trained .npz")
    ap.add_argument("--bin", default=WEIGHTS_BIN, help="export: the ZB3DPLT1 file to write")
    ap.add_argument("--gate-frames", type=int, default=16, help="export: held-out planes per plane size and level")
    a = ap.parse_args(argv)
    import time
    if a.cmd == "export":
        t0 = time.time()
        rows = calibrate_file(a.weights, a.bin, frames=a.gate_frames, **TRAIN_KW)
        print(f"gate of {a.weights} on {a.gate_frames} held-out planes per size and level "
              f"({time.time() - t0:.1f} s):")
        for s, w, h, m, d in rows:
            print(f"  {w}x{h} sigma {s:5.1f}: two-pass delta mean {m:+.3f} dB (min {min(d):+.3f}, "
                  f"max {max(d):+.3f}) -> {'pilot' if m >= -0.05 else 'plain step 1'}")
        print(f"saved {a.bin}")
        return
    if a.cmd == "time":
        for line in time_kernels():
            print(line)
        return
    if a.cmd == "train":
        t0 = time.time()
        noisy, target, sig = [], [], []
        for k, d in enumerate(a.dims.split(",")):
            wd, ht = (int(v) for v in d.split("x"))
            nz, tg, _, sg = make_pairs(a.frames, (wd, ht), TRAIN_SIGMAS, seed=11 + k, **TRAIN_KW)
            noisy, target, sig = noisy + nz, target + tg, sig + sg
        print(f"{len(noisy)} training pairs ({a.dims}, step 1 with {TRAIN_KW}) in {time.time() - t0:.1f} s")
        net = PilotNet(seed=0, width=a.width, layers=a.layers)
        t0 = time.time()
        fw = detail_weights(target, a.detail) if a.detail > 0 else None
        hist = train(net, noisy, target, sig, steps=a.steps, batch=32, crop=64, lr=a.lr, seed=5, frame_weights=fw)
        net.torch.cuda.synchronize()
        print(f"{a.steps} steps x 32 crops of 64x64 in {time.time() - t0:.1f} s; "
              f"loss {np.mean(hist[:50]):.3e} -> {np.mean(hist[-50:]):.3e}")
        net.save(a.out)
        print(f"saved {a.out}")
    else:
        net = PilotNet.load(a.out)
    print("sigma  noisy  step1  pilot  two-pass(step1)  two-pass(pilot)  delta")
    for s, n0, s1, p1, tp, tq in evaluate(net, **TRAIN_KW):
        print(f"{s:5.1f} {n0:6.2f} {s1:6.2f} {p1:6.2f} {tp:10.2f} {tq:15.2f} {tq - tp:+8.3f}")


if __name__ == "__main__":
    main()
