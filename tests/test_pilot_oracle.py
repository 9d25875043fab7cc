"""The pilot's CPU oracle checked against finite differences (BF16 rounding
switched off): its analytic backward pass is the gradient of its forward pass."""
import numpy as np

import pilot_oracle as po


def test_oracle_backward_equals_finite_differences(monkeypatch):
    monkeypatch.setattr(po, "bf16", lambda x: np.asarray(x, np.float64))
    rng = np.random.default_rng(0)
    shapes = [(16, 8), (8, 8), (8, 16)]
    W = [rng.normal(0, 0.3, (co, 3, 3, ci)) for ci, co in shapes]
    W[0][:, :, :, 2:] = 0.0
    B = [rng.normal(0, 0.1, co) for _, co in shapes]
    n, h, w = 1, 5, 6
    noisy = rng.uniform(0, 1, (n, h, w))
    target = rng.uniform(0, 1, (n, h, w))
    sigma = np.array([12.0])

    def loss(Ws, Bs):
        _, y = po.forward(Ws, Bs, noisy, sigma, 4.0)
        return float(np.mean((y - target) ** 2))

    acts, y = po.forward(W, B, noisy, sigma, 4.0)
    dws, dbs = po.backward(W, acts, y, target, 1.0)
    eps = 1e-6
    for l in range(len(W)):
        for idx in [(0, 1, 1, 0), (min(3, W[l].shape[0] - 1), 0, 2, 1), (1, 2, 0, min(5, W[l].shape[3] - 1))]:
            if l == 0 and idx[3] >= 2:
                continue
            Wp = [x.copy() for x in W]
            Wm = [x.copy() for x in W]
            Wp[l][idx] += eps
            Wm[l][idx] -= eps
            fd = (loss(Wp, B) - loss(Wm, B)) / (2 * eps)
            assert abs(fd - dws[l][idx]) <= 1e-5 * max(1.0, abs(fd)), (l, idx, fd, dws[l][idx])
        Bp = [x.copy() for x in B]
        Bm = [x.copy() for x in B]
        Bp[l][0] += eps
        Bm[l][0] -= eps
        fd = (loss(W, Bp) - loss(W, Bm)) / (2 * eps)
        assert abs(fd - dbs[l][0]) <= 1e-5 * max(1.0, abs(fd))
