"""Seeded synthetic frames for the benchmarks and tests.

A clean frame is a linear gradient ``0.25 + 0.5 * (x/W + y/H) / 2``, twenty
axis-aligned rectangles of uniform intensity in [0, 1] painted in order, and a
sinusoidal texture ``0.1 * sin(2*pi*(x cos(theta) + y sin(theta)) / P)`` with
P ~ U[6, 40] px and theta ~ U[0, pi).  Noise is i.i.d. N(0, sigma/255); nothing
is clamped.  With ``motion`` the scene translates by an integer global shift of
0..3 px/frame and eight extra rectangles move with velocities ~ U[-4, 4] px/frame.

Seeds: ``0xB3D0000 + 1000 * clip + frame`` for still clips, the clip seed alone
for the moving scene (noise still differs per frame), plus ``100 * plane``.
"""
from __future__ import annotations

import numpy as np

BASE_SEED = 0xB3D0000


def frame_seed(clip: int, frame: int) -> int:
    return BASE_SEED + 1000 * clip + frame


def _paint(img, x0, y0, rw, rh, val):
    h, w = img.shape
    xa, xb = max(int(x0), 0), min(int(x0 + rw), w)
    ya, yb = max(int(y0), 0), min(int(y0 + rh), h)
    if xa < xb and ya < yb:
        img[ya:yb, xa:xb] = val


def _scene(w: int, h: int, seed: int, shift=(0, 0), t: int = 0, motion: bool = False) -> np.ndarray:
    rng = np.random.Generator(np.random.PCG64(seed))
    sx, sy = int(shift[0]), int(shift[1])
    xs = np.arange(w, dtype=np.float64) + sx
    ys = np.arange(h, dtype=np.float64) + sy
    img = 0.25 + 0.5 * (xs[None, :] / w + ys[:, None] / h) / 2.0
    for _ in range(20):
        x0 = rng.integers(-w // 8, w)
        y0 = rng.integers(-h // 8, h)
        rw = rng.integers(4, max(5, w // 3))
        rh = rng.integers(4, max(5, h // 3))
        val = rng.uniform(0.0, 1.0)
        _paint(img, x0 - sx, y0 - sy, rw, rh, val)
    period = rng.uniform(6.0, 40.0)
    theta = rng.uniform(0.0, np.pi)
    img += 0.1 * np.sin(2.0 * np.pi * (xs[None, :] * np.cos(theta) + ys[:, None] * np.sin(theta)) / period)
    if motion:
        for _ in range(8):
            x0 = rng.uniform(0, w)
            y0 = rng.uniform(0, h)
            rw = rng.integers(8, max(9, w // 6))
            rh = rng.integers(8, max(9, h // 6))
            vx, vy = rng.uniform(-4.0, 4.0, size=2)
            val = rng.uniform(0.0, 1.0)
            _paint(img, round(x0 + vx * t), round(y0 + vy * t), rw, rh, val)
    return img


def clean_plane(w: int, h: int, clip: int = 0, frame: int = 0, plane: int = 0, motion: bool = False) -> np.ndarray:
    if motion:
        seed = BASE_SEED + 1000 * clip + 100 * plane
        g = np.random.Generator(np.random.PCG64(seed + 7))
        gx, gy = g.integers(0, 4, size=2)
        return _scene(w, h, seed, shift=(gx * frame, gy * frame), t=frame, motion=True).astype(np.float32)
    return _scene(w, h, frame_seed(clip, frame) + 100 * plane).astype(np.float32)


def noisy_plane(w: int, h: int, sigma: float, clip: int = 0, frame: int = 0, plane: int = 0,
                motion: bool = False, stride: int | None = None) -> np.ndarray:
    """Clean plane plus N(0, sigma/255) noise, float32 [h][stride] (pad columns are 0)."""
    img = clean_plane(w, h, clip, frame, plane, motion)
    rng = np.random.Generator(np.random.PCG64(frame_seed(clip, frame) * 7919 + 31 * plane + 1))
    img = img + rng.normal(0.0, sigma / 255.0, size=img.shape).astype(np.float32)
    stride = stride or w
    out = np.zeros((h, stride), np.float32)
    out[:, :w] = img
    return out


def psnr(a: np.ndarray, b: np.ndarray, peak: float = 1.0) -> float:
    mse = float(np.mean((a.astype(np.float64) - b.astype(np.float64)) ** 2))
    return float("inf") if mse == 0 else 10.0 * np.log10(peak * peak / mse)
