"""The learned-initial-pose network's kernels (csrc/posenet.cu: BF16 tensor
cores via tcgen05 for the shared 64 -> 128 layer, for the head's forward
and for its backward products -- dY W4, dH3 W3 and the weight gradients
dH3^T G, dY^T H3 summed over 128-scan tiles) against the CPU reference
(oracle/posenet_ref.py, which rounds the same operands to BF16) through the
C ABI, on one partial head tile (8 scans) and on three tiles (300 scans).

Tolerances: the max-pool values within 1e-4 relative (the reference sums the
BF16 products exactly, the tensor cores in FP32); the outputs y within 1e-3
of max(1, |y|); the batch gradient (update = 0) within 2e-3 of each block's
largest entry, with the reference evaluated at the kernel's max-pool routing.
"""
import numpy as np
import pytest

import posenet_ref as R

pytestmark = pytest.mark.gpu


def _batch(seed, sizes):
    rng = np.random.default_rng(seed)
    scans, guesses = [], []
    for n in sizes:
        s = np.ones((n, 4), np.float32)
        s[:, :3] = rng.uniform(-30, 30, (n, 3)).astype(np.float32)
        s[:, 2] *= 0.1
        scans.append(s)
        T = np.eye(4, dtype=np.float32)
        c, sn = np.cos(rng.uniform(-3, 3)), np.sin(rng.uniform(-3, 3))
        T[:2, :2] = [[c, -sn], [sn, c]]
        T[:3, 3] = rng.uniform(-40, 40, 3)
        guesses.append(T.reshape(16))
    targets = rng.normal(0, 1, (len(sizes), 6)).astype(np.float32)
    return scans, np.stack(guesses), targets


def _device(torch, scans, guesses, targets):
    offs = np.zeros(len(scans) + 1, np.int32)
    offs[1:] = np.cumsum([len(s) for s in scans])
    pts = np.concatenate(scans) if offs[-1] else np.zeros((1, 4), np.float32)
    d = dict(points=torch.from_numpy(np.ascontiguousarray(pts)).cuda(),
             offsets=torch.from_numpy(offs).cuda(),
             guesses=torch.from_numpy(np.ascontiguousarray(guesses)).cuda(),
             targets=torch.from_numpy(np.ascontiguousarray(targets)).cuda(),
             y=torch.zeros((len(scans), 6), dtype=torch.float32, device="cuda"),
             gmax=torch.zeros((len(scans), 128), dtype=torch.int64, device="cuda"))
    return d


def _close(a, b, tol):
    return np.max(np.abs(a - b)) <= tol * max(1.0, float(np.max(np.abs(b))))


SMALL = [3000, 128, 1, 777, 0, 2048, 129, 64]
TILES = [int(n) for n in np.random.default_rng(9).integers(0, 700, 300)]


@pytest.mark.parametrize("sizes", [SMALL, TILES], ids=["8_scans", "300_scans"])
def test_posenet_forward_and_gradient_match_reference(pkg, sizes):
    torch = pytest.importorskip("torch")
    scans, guesses, targets = _batch(11, sizes)
    center, scale, maxp = (0.0, 0.0, 0.0), 50.0, 1024
    w = R.init_weights(5)
    w[R.oB1:R.oW2] = 0.05
    w[R.oB2:R.oW3] = 0.02
    net = pkg.posenet.PoseNet(center=center, scale=scale)
    net.set_weights(w)
    d = _device(torch, scans, guesses, targets)
    B = len(scans)
    net.forward(B, d["points"].data_ptr(), d["offsets"].data_ptr(), d["guesses"].data_ptr(), d["y"].data_ptr(), maxp)
    net.maxpool(d["gmax"].data_ptr(), B)
    net.synchronize()
    y = d["y"].cpu().numpy()
    gm = d["gmax"].cpu().numpy().view(np.uint64)
    g_gpu = (gm >> np.uint64(32)).astype(np.uint32).view(np.float32)
    arg_gpu = (np.uint64(0xFFFFFFFF) - (gm & np.uint64(0xFFFFFFFF))).astype(np.int64)
    agree = 0
    for b in range(B):
        f = R.forward_scan(w, scans[b], guesses[b], center, scale, maxp)
        assert np.max(np.abs(g_gpu[b] - f["g"])) <= 1e-4 * max(1.0, float(np.max(f["g"]))), b
        if sizes[b] > 0:
            agree += int(np.sum(arg_gpu[b] == f["arg"]))
            fa = R.forward_scan(w, scans[b], guesses[b], center, scale, maxp, argmax=arg_gpu[b])
        else:
            fa = f
        assert _close(y[b], fa["y"], 1e-3), (b, y[b], fa["y"])
    assert agree >= 0.98 * 128 * sum(1 for n in sizes if n > 0)
    # gradient (no update), reference at the kernel's routing
    loss, grad = net.train_step(B, d["points"].data_ptr(), d["offsets"].data_ptr(), d["guesses"].data_ptr(),
                                d["targets"].data_ptr(), update=False, max_points=maxp, want_grad=True)
    net.synchronize()
    rl, rg = R.loss_and_grad(w, scans, guesses, targets, center, scale, maxp,
                             argmaxes=[arg_gpu[b] if sizes[b] > 0 else None for b in range(B)])
    assert abs(loss - rl) <= 1e-3 * max(1.0, abs(rl))
    blocks = [(R.oW1, R.oB1), (R.oB1, R.oW2), (R.oW2, R.oB2), (R.oB2, R.oW3), (R.oW3, R.oB3), (R.oB3, R.oW4),
              (R.oW4, R.oB4), (R.oB4, R.NUM_W)]
    for lo, hi in blocks:
        assert _close(grad[lo:hi], rg[lo:hi], 2e-3), (lo, np.max(np.abs(grad[lo:hi] - rg[lo:hi])))
    net.close()


def test_posenet_training_reduces_loss(pkg):
    """Adam steps on a fixed batch drive the loss down (the targets depend on
    the scans, so the network can fit them)."""
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(2)
    scans, guesses, _ = _batch(21, [512] * 32)
    # target: a smooth function of the guess translation
    targets = np.stack([np.tanh(g.reshape(4, 4)[:3, 3].repeat(2) / 30.0) for g in guesses]).astype(np.float32)
    net = pkg.posenet.PoseNet(center=(0.0, 0.0, 0.0), scale=50.0)
    net.set_weights(R.init_weights(3))
    d = _device(torch, scans, guesses, targets)
    losses = []
    for it in range(300):
        loss, _ = net.train_step(len(scans), d["points"].data_ptr(), d["offsets"].data_ptr(),
                                 d["guesses"].data_ptr(), d["targets"].data_ptr(), lr=3e-3, update=True,
                                 max_points=256)
        losses.append(loss)
    net.synchronize()
    assert np.isfinite(losses).all()
    assert np.mean(losses[-10:]) < 0.3 * np.mean(losses[:10]), (losses[:3], losses[-3:])
    net.close()
