"""CPU oracle of the learned pilot's network (test infrastructure only).

A float64 numpy restatement of the forward pass and the backward pass of the
residual 3x3 conv net in vapoursynth-zipcu_b200/csrc/zb3d_pilot.cu.  It rounds to
BF16 at the same points as the GPU: the packed input, each stored activation, the
weights, and the loss gradient.  Only the accumulation (float64 here, FP32 there)
differs, so gradients can be compared tightly.

The pilot has no counterpart in the reference (it is an addition of this project);
parity here means GPU kernels == this restatement, checked by tests/test_pilot_gpu.py.
"""
from __future__ import annotations

import numpy as np


def bf16(x):
    """Round to bfloat16 (round to nearest even), returned as float64."""
    a = np.asarray(x, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def conv3x3(x, w, b=None):
    """x [n][h][w][cin], w [cout][3][3][cin] -> [n][h][w][cout], zero padding."""
    n, h, wd, cin = x.shape
    xp = np.zeros((n, h + 2, wd + 2, cin))
    xp[:, 1:-1, 1:-1] = x
    y = np.zeros((n, h, wd, w.shape[0]))
    for ky in range(3):
        for kx in range(3):
            y += np.einsum("nhwc,oc->nhwo", xp[:, ky:ky + h, kx:kx + wd], w[:, ky, kx, :])
    if b is not None:
        y += b
    return y


def pack_input(noisy, sigma, level_scale):
    n, h, w = noisy.shape
    x = np.zeros((n, h, w, 16))
    x[..., 0] = bf16(noisy)
    x[..., 1] = bf16((np.asarray(sigma, np.float32) * np.float32(1.0 / 255.0) * np.float32(level_scale))[:, None, None]
                     * np.ones((n, h, w), np.float32))
    return x


def forward(weights, biases, noisy, sigma, level_scale):
    """Activations (stored, BF16-rounded) and the FP32-like output y = noisy + out[..., 0]."""
    acts = [pack_input(noisy, sigma, level_scale)]
    L = len(weights)
    for l in range(L):
        pre = conv3x3(acts[-1], bf16(weights[l]), biases[l])
        if l < L - 1:
            acts.append(bf16(np.maximum(pre, 0.0)))
        else:
            out = pre[..., 0]
    return acts, noisy.astype(np.float64) + out


def backward(weights, acts, y, target, scale):
    """Loss-scaled gradients (dw, db per layer) of sum (y - t)^2 / count, as the GPU
    computes them: dy rounded to BF16, each pre-activation gradient rounded to BF16."""
    L = len(weights)
    count = y.size
    d = np.zeros(acts[-1].shape[:3] + (weights[-1].shape[0],))
    d[..., 0] = bf16(np.float32(scale) * np.float32(2.0) * (y - target).astype(np.float32) / np.float32(count))
    dws, dbs = [None] * L, [None] * L
    for l in range(L - 1, -1, -1):
        x = acts[l]
        n, h, w, cin = x.shape
        xp = np.zeros((n, h + 2, w + 2, cin))
        xp[:, 1:-1, 1:-1] = x
        dw = np.zeros_like(weights[l], dtype=np.float64)
        for ky in range(3):
            for kx in range(3):
                dw[:, ky, kx, :] = np.einsum("nhwo,nhwc->oc", d, xp[:, ky:ky + h, kx:kx + w])
        dws[l], dbs[l] = dw, d.sum(axis=(0, 1, 2))
        if l == 0:
            break
        wf = bf16(weights[l])[:, ::-1, ::-1, :].transpose(3, 1, 2, 0)  # [cin][3][3][cout]
        dx = conv3x3(d, wf)
        d = bf16(np.where(acts[l] > 0, dx, 0.0))
    return dws, dbs
