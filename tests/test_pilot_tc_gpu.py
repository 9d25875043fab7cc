"""The tensor-core inference convolution (csrc/zb3d_pilot_tc.cu: tcgen05.mma, TMA-staged
rows) against the mma.sync convolution of zb3d_pilot.cu and the numpy oracle
(oracle/pilot_oracle.py).

Both kernels multiply the same BF16 operands and sum in FP32; only the order of the
sums differs, so a stored BF16 activation may differ by one BF16 rounding step (2^-8 to
2^-7 of the value) where the FP32 sum sits next to a rounding boundary, and nowhere by more.
Shapes: every supported (cin, cout), images narrower than one 128-pixel strip, ragged
strips, several images, rows split over CTAs.  The tensor-core kernel takes and gives
the channel-blocked layout [n][c/8][h][w][8]; the tests convert from and to NHWC.
"""
import numpy as np
import pytest

import pilot_oracle as po
from zb3d import _native as N
from zb3d import pilot as P

pytestmark = pytest.mark.gpu

SHAPES = [(16, 48), (48, 48), (48, 16), (16, 32), (32, 32), (32, 16), (16, 16)]
SIZES = [(1, 9, 20), (2, 37, 150), (1, 70, 384), (3, 16, 257)]
ULP = 2.0 ** -7  # one BF16 rounding step, relative to the value (2^-8 .. 2^-7)


def _bf16_to_f32(t):
    import torch
    return t.float().cpu().numpy()


def blocked(x):
    """NHWC -> channel-blocked [n][c/8][h][w][8]"""
    n, h, w, c = x.shape
    return x.reshape(n, h, w, c // 8, 8).permute(0, 3, 1, 2, 4).contiguous()


def nhwc(x):
    n, cb, h, w, _ = x.shape
    return x.permute(0, 2, 3, 1, 4).reshape(n, h, w, cb * 8).contiguous()


def _conv(kind, x, w16, bias, n, h, w, cin, cout, relu, status=None):
    import torch
    lib = N.lib()
    y = torch.empty((n, h, w, cout), dtype=torch.bfloat16, device="cuda")
    if kind == "tc":
        xb = blocked(x)
        yb = torch.empty((n, cout // 8, h, w, 8), dtype=torch.bfloat16, device="cuda")
        rc = lib.zb3d_pilot_conv3x3_tc(xb.data_ptr(), n, h, w, cin, w16.data_ptr(), bias.data_ptr(), cout, relu,
                                       yb.data_ptr(), None, None, 0, 0,
                                       status.data_ptr() if status is not None else None, None)
        assert rc == 0
        return nhwc(yb)
    else:
        rc = lib.zb3d_pilot_conv3x3(x.data_ptr(), n, h, w, cin, w16.data_ptr(), bias.data_ptr(), cout, relu, None,
                                    y.data_ptr(), None, None, None)
    assert rc == 0
    return y


@pytest.mark.parametrize("cin,cout", SHAPES)
@pytest.mark.parametrize("n,h,w", SIZES)
def test_tc_conv_matches_mma_sync_and_oracle(cin, cout, n, h, w):
    import torch
    rng = np.random.default_rng(cin * 131 + cout * 7 + h)
    x32 = rng.uniform(-1.0, 1.0, (n, h, w, cin)).astype(np.float32)
    wt = rng.normal(0.0, 1.0 / np.sqrt(9 * cin), (cout, 3, 3, cin)).astype(np.float32)
    b = rng.normal(0.0, 0.1, cout).astype(np.float32)
    x = torch.from_numpy(x32).cuda().to(torch.bfloat16)
    w16 = torch.from_numpy(wt).cuda().to(torch.bfloat16)
    bias = torch.from_numpy(b).cuda()
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    for relu in (1, 0):
        yt = _bf16_to_f32(_conv("tc", x, w16, bias, n, h, w, cin, cout, relu, status))
        ym = _bf16_to_f32(_conv("mma", x, w16, bias, n, h, w, cin, cout, relu))
        torch.cuda.synchronize()
        assert int(status.item()) == 0
        ref = po.conv3x3(x.float().cpu().numpy().astype(np.float64), w16.float().cpu().numpy().astype(np.float64), b)
        if relu:
            ref = np.maximum(ref, 0.0)
        ref16 = po.bf16(ref)
        scale = np.maximum(np.abs(ref16), 1e-3)
        for y in (yt, ym):
            err = np.abs(y - ref16) / scale
            assert err.max() <= 1.01 * ULP, err.max()         # at most one rounding step
            assert np.mean(y != ref16) < 0.02                # and rarely that
        assert np.mean(yt != ym) < 0.02


def test_tc_last_layer_fp32_output_and_residual():
    import torch
    lib = N.lib()
    rng = np.random.default_rng(5)
    n, h, w, cin, cout = 2, 33, 200, 48, 16
    x = torch.from_numpy(rng.uniform(-1, 1, (n, h, w, cin)).astype(np.float32)).cuda().to(torch.bfloat16)
    w16 = torch.from_numpy(rng.normal(0, 0.05, (cout, 3, 3, cin)).astype(np.float32)).cuda().to(torch.bfloat16)
    bias = torch.from_numpy(rng.normal(0, 0.1, cout).astype(np.float32)).cuda()
    resid = torch.from_numpy(rng.uniform(0, 1, (n, h, w)).astype(np.float32)).cuda()
    outs = []
    xb = blocked(x)
    for kind in ("tc", "mma"):
        y0 = torch.full((n, h, w), np.nan, dtype=torch.float32, device="cuda")
        if kind == "tc":
            rc = lib.zb3d_pilot_conv3x3_tc(xb.data_ptr(), n, h, w, cin, w16.data_ptr(), bias.data_ptr(), cout, 0,
                                           None, y0.data_ptr(), resid.data_ptr(), 0, 0, None, None)
        else:
            rc = lib.zb3d_pilot_conv3x3(x.data_ptr(), n, h, w, cin, w16.data_ptr(), bias.data_ptr(), cout, 0, None,
                                        None, y0.data_ptr(), resid.data_ptr(), None)
        assert rc == 0
        outs.append(y0.cpu().numpy())
    ref = po.conv3x3(x.float().cpu().numpy().astype(np.float64), w16.float().cpu().numpy().astype(np.float64),
                     bias.cpu().numpy())[..., 0] + resid.cpu().numpy()
    for o in outs:
        assert np.isfinite(o).all()
        assert np.abs(o - ref).max() < 1e-5 * max(1.0, np.abs(ref).max())


@pytest.mark.parametrize("width,layers", [(48, 10), (32, 8), (16, 8)])
def test_tc_network_forward_matches_mma_sync(width, layers):
    import torch
    net = P.PilotNet(seed=2, width=width, layers=layers)
    rng = np.random.default_rng(6)
    for l in range(len(net.shapes)):
        b = np.zeros(net.shapes[l][1], np.float32)
        real = P.REAL_OUT if l == len(net.shapes) - 1 else net.shapes[l][1]
        b[:real] = rng.normal(0, 0.05, real)
        net.b32[l].copy_(torch.from_numpy(b))
    noisy = torch.from_numpy(rng.uniform(0, 1, (2, 45, 300)).astype(np.float32)).cuda()
    sigma = torch.tensor([8.0, 21.0], dtype=torch.float32, device="cuda")
    yt, _ = net.forward(noisy, sigma, tc=True)
    ym, _ = net.forward(noisy, sigma, tc=False)
    yt, ym = yt.cpu().numpy(), ym.cpu().numpy()
    rel = np.linalg.norm(yt - ym) / np.linalg.norm(ym - noisy.cpu().numpy())
    assert rel < 2e-2, rel  # one-step BF16 flips of hidden activations, relative to the net's output


def test_tc_network_on_strided_frame_buffers():
    """Images inside [reference | noisy] frame buffers (2 h w floats apart), as step 2 reads
    them: the pilot reads the noisy halves and writes the reference halves in place."""
    import torch
    net = P.PilotNet(seed=5)
    rng = np.random.default_rng(8)
    n, h, w = 3, 40, 200
    noisy = rng.uniform(0, 1, (n, h, w)).astype(np.float32)
    sigma = torch.tensor([6.0, 12.0, 20.0], dtype=torch.float32, device="cuda")
    dense, _ = net.forward(torch.from_numpy(noisy).cuda(), sigma, tc=True)
    frames = torch.full((n, 2, h, w), np.nan, dtype=torch.float32, device="cuda")
    frames[:, 1] = torch.from_numpy(noisy).cuda()
    net.forward(frames[:, 1], sigma, out=frames[:, 0], tc=True)
    assert torch.equal(frames[:, 0], dense)
    assert torch.equal(frames[:, 1].cpu(), torch.from_numpy(noisy))
    with pytest.raises(ValueError):
        net.forward(frames[:, 1], sigma, tc=False)  # the NHWC path takes dense images only
    # one image whose leading (size-1) dimension carries an arbitrary stride, as numpy gives it
    padded = np.zeros((h, w + 3), np.float32)
    padded[:, :w] = noisy[0]
    one = torch.from_numpy(padded[:, :w][None].astype(np.float32)).cuda()
    assert one.stride(0) != h * w
    y1, _ = net.forward(one, sigma[:1], tc=True)
    assert torch.equal(y1, dense[:1])


def test_pilot_runs_on_torchs_current_stream():
    """Launches follow torch's current stream (its allocator orders the buffer reuse); a
    different explicit stream is refused."""
    import torch
    net = P.PilotNet(seed=1)
    x = torch.rand((1, 24, 160), device="cuda")
    sig = torch.tensor([10.0], device="cuda")
    ref, _ = net.forward(x, sig, tc=True)
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        y, _ = net.forward(x, sig, tc=True)  # on s, with buffers of its own
        y2, _ = net.forward(x, sig, tc=True, stream=s.cuda_stream)
    torch.cuda.synchronize()
    assert torch.equal(y, ref) and torch.equal(y2, ref)
    with pytest.raises(ValueError):
        net.forward(x, sig, tc=True, stream=s.cuda_stream)  # s is not the current stream here
    # the buffer cache stays bounded across many shapes
    for k in range(P.WS_KEEP + 4):
        net.forward(torch.rand((1, 16, 64 + 8 * k), device="cuda"), sig, tc=True)
    assert len(net._ws) <= P.WS_KEEP
