"""The precision form of the patch transform (csrc/zb3d_dct_tc.cu): the 2D DCT of
8x8 patches on the tcgen05 tensor cores in TF32 with FP32 accumulation, split into
hi/lo products, against an FP64 restatement of the transform.  The matrix is the
closed form from which the CPU oracle builds its DCT (oracle/bm3d_oracle.c,
build_matrices): the orthonormal DCT-II scaled by 4 per axis.

Errors are the largest absolute difference from the FP64 result, relative to the
largest coefficient of the stack.  Three are compared:
  * numpy's float32 product of the same operands: the rounding of an FP32 GEMM;
  * split = 0: one TF32 product, about 2^-11;
  * split = 1: the three hi/lo products.  It must stay within 1e-6 (measured 0.8-2.2e-7,
    the level of the FP32 GEMM) and gain at least 200x over the single TF32 product
    (measured about 3e-4).
"""
import numpy as np
import pytest

from zb3d import _native as N
from zb3d import synth

pytestmark = pytest.mark.gpu

SPLIT_MAX = 1e-6      # relative to the largest coefficient
SPLIT_GAIN = 200.0    # single-TF32 error / split error, at least


def dct_matrix():
    k = np.arange(8)[:, None]
    m = np.arange(8)[None, :]
    a = np.where(k == 0, np.sqrt(1.0 / 8.0), np.sqrt(2.0 / 8.0))
    return 4.0 * a * np.cos(np.pi * (2 * m + 1) * k / 16.0)


def patches(n, seed):
    """n row-major 8x8 patches of a synthetic noisy plane (pixel-valued, sigma 10)"""
    plane = synth.noisy_plane(256, 256, 10.0, clip=seed % 7, frame=0, plane=0)
    rng = np.random.default_rng(seed)
    ys = rng.integers(0, 256 - 8, n)
    xs = rng.integers(0, 256 - 8, n)
    return np.stack([plane[y:y + 8, x:x + 8] for y, x in zip(ys, xs)]).reshape(n, 64).astype(np.float32)


def run(x, split):
    import torch
    lib = N.lib()
    dx = torch.from_numpy(x).cuda()
    dy = torch.full_like(dx, float("nan"))
    st = torch.zeros(1, dtype=torch.int32, device="cuda")
    rc = lib.zb3d_dct2d_tf32(dx.data_ptr(), dy.data_ptr(), x.shape[0], split, st.data_ptr(),
                             torch.cuda.current_stream().cuda_stream)
    assert rc == 0
    torch.cuda.synchronize()
    assert int(st.item()) == 0
    return dy.cpu().numpy()


@pytest.mark.parametrize("n", [1, 127, 128, 1000, 40000])
def test_dct2d_tf32_split_against_fp64(n):
    K = np.kron(dct_matrix(), dct_matrix())  # [r * 8 + c][i * 8 + j]
    x = patches(n, n)
    ref = x.astype(np.float64) @ K.T
    scale = np.abs(ref).max()
    e_fp32 = np.abs(x @ K.T.astype(np.float32) - ref).max() / scale
    e_tf32 = np.abs(run(x, 0) - ref).max() / scale
    y = run(x, 1)
    e_split = np.abs(y - ref).max() / scale
    print(f"n={n}: relative max error  fp32 GEMM {e_fp32:.2e}  TF32 {e_tf32:.2e}  TF32 hi/lo split {e_split:.2e}")
    assert np.isfinite(y).all()
    assert e_split <= SPLIT_MAX
    assert e_tf32 >= SPLIT_GAIN * e_split
    np.testing.assert_array_equal(run(x, 1), y)  # the same bits on a second call

