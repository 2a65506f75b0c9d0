"""CPU reference of the learned-initial-pose network (oracle/posenet_ref.py):
its analytic gradient against central finite differences (float64 form, no
BF16 rounding), and the BF16 rounding helper against known values."""
import numpy as np

import posenet_ref as R


def _data(seed=3, B=3):
    rng = np.random.default_rng(seed)
    scans, guesses, targets = [], [], []
    for b in range(B):
        n = [40, 300, 5][b % 3]
        s = np.ones((n, 4), np.float32)
        s[:, :3] = rng.uniform(-20, 20, (n, 3))
        scans.append(s)
        T = np.eye(4, dtype=np.float32)
        T[:3, 3] = rng.uniform(-5, 5, 3)
        guesses.append(T.reshape(16))
        targets.append(rng.normal(0, 1, 6))
    return scans, guesses, targets


def test_gradient_matches_finite_differences():
    w = R.init_weights(1).astype(np.float64)
    w[R.oB1:R.oW2] = 0.1
    w[R.oB2:R.oW3] = 0.05
    w[R.oB3:R.oW4] = 0.05
    scans, guesses, targets = _data()
    center, scale = (0.0, 0.0, 0.0), 25.0
    loss, g = R.loss_and_grad(w, scans, guesses, targets, center, scale, bf16_mode=False)
    rng = np.random.default_rng(7)
    # parameters of every block; the max-pool routing is held fixed (it is
    # piecewise constant, and the step is far below the gaps between maxima)
    arg = [R.forward_scan(w, s, gs, center, scale, bf16_mode=False)["arg"] for s, gs in zip(scans, guesses)]
    blocks = [(R.oW1, R.oB1), (R.oB1, R.oW2), (R.oW2, R.oB2), (R.oB2, R.oW3), (R.oW3, R.oB3), (R.oB3, R.oW4),
              (R.oW4, R.oB4), (R.oB4, R.NUM_W)]
    eps = 1e-6
    for lo, hi in blocks:
        for i in rng.choice(np.arange(lo, hi), size=min(6, hi - lo), replace=False):
            wp, wm = w.copy(), w.copy()
            wp[i] += eps
            wm[i] -= eps
            lp, _ = R.loss_and_grad(wp, scans, guesses, targets, center, scale, bf16_mode=False, argmaxes=arg)
            lm, _ = R.loss_and_grad(wm, scans, guesses, targets, center, scale, bf16_mode=False, argmaxes=arg)
            fd = (lp - lm) / (2 * eps)
            assert abs(fd - g[i]) <= 1e-6 + 1e-5 * abs(fd), (lo, i, fd, g[i])


def test_bf16_rounding():
    x = np.array([1.0, 1.00390625, 1.0078125, 3.14159265, -2.5e-3, 65504.0], np.float32)
    b = R.bf16(x)
    assert b[0] == 1.0 and b[1] == 1.0          # ties to even (1 + 2^-8 -> 1)
    assert b[2] == np.float32(1.0078125)         # exactly representable
    assert abs(b[3] - 3.140625) < 1e-7
    assert (b.view(np.uint32) & 0xFFFF == 0).all()
