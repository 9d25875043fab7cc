"""The learned pilot's kernels (csrc/zb3d_pilot.cu) against the numpy oracle
(oracle/pilot_oracle.py), its training, and what it does for two-pass BM3Dv2.

* forward output and the loss-scaled weight / bias gradients of all 10 layers equal
  the float64 restatement (same BF16 rounding points) to FP32-accumulation accuracy,
  on a ragged input (partial 8 x 16 tiles);
* Adam steps on (noisy, step-1) crops lower the loss;
* a trained pilot as step 2's reference: its PSNR is reported against the plain
  two-pass result and the clean frame, and the 0.05 dB gate decides per noise level.
"""
import numpy as np
import pytest

import pilot_oracle as po
from zb3d import pilot as P
from zb3d import synth

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-30))


def test_pilot_forward_and_gradients_match_oracle():
    import torch
    net = P.PilotNet(seed=3)
    rng = np.random.default_rng(4)
    for l in range(len(P.SHAPES)):  # non-zero biases (real output channels only)
        b = np.zeros(P.SHAPES[l][1], np.float32)
        real = P.REAL_OUT if l == len(P.SHAPES) - 1 else P.SHAPES[l][1]
        b[:real] = rng.normal(0, 0.05, real)
        net.b32[l].copy_(torch.from_numpy(b))
    n, h, w = 2, 20, 24
    noisy = rng.uniform(0.0, 1.0, (n, h, w)).astype(np.float32)
    target = (noisy + rng.normal(0, 0.05, (n, h, w))).astype(np.float32)
    sigma = np.array([7.0, 19.0], np.float32)
    dn, dt, ds = (torch.from_numpy(a).cuda() for a in (noisy, target, sigma))
    dws, dbs, loss, y = net.gradients(dn, dt, ds)
    torch.cuda.synchronize()
    W = [wt.cpu().numpy().astype(np.float64) for wt in net.w32]
    B = [b.cpu().numpy().astype(np.float64) for b in net.b32]
    acts, y_ref = po.forward(W, B, noisy, sigma, P.LEVEL_SCALE)
    assert _rel(y.cpu().numpy(), y_ref) < 1e-3  # a BF16 rounding point can flip by one ulp
    rw, rb = po.backward(W, acts, y_ref, target, P.LOSS_SCALE)
    for l in range(len(P.SHAPES)):
        ew, eb = _rel(dws[l].cpu().numpy(), rw[l]), _rel(dbs[l].cpu().numpy(), rb[l])
        assert ew < 2e-2 and eb < 2e-2, (l, ew, eb)
    assert abs(loss - float(np.mean((y_ref - target) ** 2))) < 1e-3 * loss


def test_pilot_training_lowers_the_loss():
    noisy, target, _, sig = P.make_pairs(3, 128, [10.0, 20.0], seed=2)
    net = P.PilotNet(seed=0)
    hist = P.train(net, noisy, target, sig, steps=150, batch=16, crop=64, lr=2e-3, seed=1)
    first, last = np.mean(hist[:10]), np.mean(hist[-10:])
    assert last < 0.5 * first, (first, last)


def test_trained_pilot_as_step2_reference_and_the_gate():
    noisy, target, _, sig = P.make_pairs(6, 256, [5.0, 10.0, 15.0, 20.0, 25.0], seed=4)
    net = P.PilotNet(seed=0)
    P.train(net, noisy, target, sig, steps=2000, batch=32, crop=64, lr=1e-3, seed=1)
    gate = P.PilotGate(net)
    delta = gate.calibrate([10.0, 20.0], frames=1, size=256)
    for s, d in delta.items():
        cl = synth.clean_plane(256, 256, 7000, 0)
        nz = synth.noisy_plane(256, 256, s, clip=7000, frame=0)
        pilot_est = net.denoise(nz, s)
        # the pilot alone denoises (well above the noisy input) ...
        assert synth.psnr(pilot_est, cl) > synth.psnr(nz, cl) + 3.0
        # ... and the gate follows the measured two-pass difference
        assert gate.accepts(s) == (d >= -0.05)
        print(f"sigma {s}: two-pass PSNR with the pilot minus plain two-pass = {d:+.3f} dB, "
              f"{'pilot' if gate.accepts(s) else 'plain step 1'} used")
