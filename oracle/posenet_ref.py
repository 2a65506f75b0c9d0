"""CPU reference of the learned-initial-pose network (test infrastructure).

Restates daphne-benchmark_b200/csrc/posenet.cu in numpy: the point feature
u = (T x - c) / s in float32 (each operation rounded, the library's order),
layer 1 with the kernel's fused multiply-adds (emulated in float64 and rounded
to float32 after each), layer 2 on BF16-rounded operands with an exact sum,
ReLU, max-pool with the smallest index among ties, the head (its products
on BF16-rounded operands, as the tensor-core head kernel computes them: W3 g,
W4 h3, and in the backward W4^T dy, W3^T dh3, dy h3^T and dh3 g^T, the
per-scan dy = 2 (y - t) / 6 rounded before the batch mean), the loss
mean((y - t)^2) over outputs and scans, and its gradient (the straight-through
gradient of the BF16 roundings, as the kernels take it).  With bf16=False
every rounding is dropped and the arithmetic is float64: the form used for
finite-difference checks.
"""
from __future__ import annotations

import numpy as np

H1, H2, H3, OUT = 64, 128, 64, 6
oW1 = 0
oB1 = oW1 + H1 * 3
oW2 = oB1 + H1
oB2 = oW2 + H2 * H1
oW3 = oB2 + H2
oB3 = oW3 + H3 * H2
oW4 = oB3 + H3
oB4 = oW4 + OUT * H3
NUM_W = oB4 + OUT


def unpack(w):
    w = np.asarray(w)
    return dict(W1=w[oW1:oB1].reshape(H1, 3), b1=w[oB1:oW2], W2=w[oW2:oB2].reshape(H2, H1), b2=w[oB2:oW3],
                W3=w[oW3:oB3].reshape(H3, H2), b3=w[oB3:oW4], W4=w[oW4:oB4].reshape(OUT, H3), b4=w[oB4:NUM_W])


def init_weights(seed=0):
    """He-style initialisation (the library's Python side uses the same)."""
    rng = np.random.default_rng(seed)
    w = np.zeros(NUM_W, np.float32)
    w[oW1:oB1] = rng.normal(0, np.sqrt(2.0 / 3), H1 * 3)
    w[oW2:oB2] = rng.normal(0, np.sqrt(2.0 / H1), H2 * H1)
    w[oW3:oB3] = rng.normal(0, np.sqrt(2.0 / H2), H3 * H2)
    w[oW4:oB4] = rng.normal(0, np.sqrt(1.0 / H3) * 0.1, OUT * H3)
    return w


def bf16(x):
    """Round float32 to bfloat16 (nearest, ties to even), returned as float32."""
    b = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    b = ((b + 0x7FFF + ((b >> 16) & 1)) >> 16) << 16
    return b.astype(np.uint32).view(np.float32)


def sample_indices(n, max_points):
    P = min(n, max_points)
    return (np.arange(P, dtype=np.int64) * n) // P if P > 0 else np.zeros(0, np.int64)


def features(scan, guess16, center, scale, bf16_mode=True):
    """u of every point (float32 in the library's operation order)."""
    T = np.asarray(guess16, np.float32).reshape(4, 4)
    x = np.asarray(scan, np.float32)
    if not bf16_mode:
        T64 = T.astype(np.float64)
        p = x[:, :3].astype(np.float64) @ T64[:3, :3].T + T64[:3, 3]
        return (p - np.asarray(center, np.float64)) / float(scale)
    f = np.float32
    cols = []
    for r in range(3):
        v = ((T[r, 0] * x[:, 0] + T[r, 1] * x[:, 1]) + T[r, 2] * x[:, 2]) + T[r, 3]
        cols.append(((v - f(center[r])) * f(f(1.0) / f(scale))).astype(np.float32))
    return np.stack(cols, 1)


def _fma32(a, b, c):
    return (a.astype(np.float64) * b.astype(np.float64) + c.astype(np.float64)).astype(np.float32)


def layer1(u, P, bf16_mode=True):
    if not bf16_mode:
        return np.maximum(u @ P["W1"].astype(np.float64).T + P["b1"].astype(np.float64), 0.0)
    W1, b1 = P["W1"].astype(np.float32), P["b1"].astype(np.float32)
    t = _fma32(W1[None, :, 2], u[:, None, 2], np.broadcast_to(b1[None, :], (u.shape[0], H1)))
    t = _fma32(W1[None, :, 1], u[:, None, 1], t)
    t = _fma32(W1[None, :, 0], u[:, None, 0], t)
    return np.maximum(t, np.float32(0))


def forward_scan(w, scan, guess16, center, scale, max_points=1024, bf16_mode=True, argmax=None):
    """Returns dict(u, h1, g, arg, h3, y) for one scan.  argmax (128 sample
    indices) may be given to evaluate at a fixed max-pool routing."""
    P = unpack(w)
    idx = sample_indices(len(scan), max_points)
    u = features(scan[idx], guess16, center, scale, bf16_mode) if len(idx) else np.zeros((0, 3))
    h1 = layer1(u, P, bf16_mode)
    if bf16_mode:
        a = bf16(h1).astype(np.float64)
        W2 = bf16(P["W2"].astype(np.float32)).astype(np.float64)
        b2 = P["b2"].astype(np.float64)
    else:
        a, W2, b2 = h1, P["W2"].astype(np.float64), P["b2"].astype(np.float64)
    if len(idx):
        h2 = np.maximum(a @ W2.T + b2, 0.0)
        arg = np.argmax(h2, axis=0) if argmax is None else np.asarray(argmax)
        g = h2[arg, np.arange(H2)]
    else:
        h2 = np.zeros((0, H2))
        arg = np.zeros(H2, np.int64)
        g = np.zeros(H2)
    W3, b3 = P["W3"].astype(np.float64), P["b3"].astype(np.float64)
    W4, b4 = P["W4"].astype(np.float64), P["b4"].astype(np.float64)
    if bf16_mode:  # the head's products run on the tensor cores: BF16 operands, FP32 sums
        h3 = np.maximum(_b(W3) @ _b(g) + b3, 0.0)
        y = _b(W4) @ _b(h3) + b4
    else:
        h3 = np.maximum(W3 @ g + b3, 0.0)
        y = W4 @ h3 + b4
    return dict(u=u, h1=h1, a=a, W2=W2, g=g, arg=arg, h3=h3, y=y)


def _b(x):
    """float64 values rounded to float32, then to BF16 (a tensor-core operand)."""
    return bf16(np.asarray(x, np.float64).astype(np.float32)).astype(np.float64)


def loss_and_grad(w, scans, guesses, targets, center, scale, max_points=1024, bf16_mode=True, argmaxes=None):
    """Batch loss mean_b mean_i (y_bi - t_bi)^2 and its gradient (float64)."""
    P = unpack(w)
    B = len(scans)
    grad = np.zeros(NUM_W)
    G = unpack(grad)  # views into grad
    loss = 0.0
    W3, W4 = P["W3"].astype(np.float64), P["W4"].astype(np.float64)
    W1, b1 = P["W1"].astype(np.float64), P["b1"].astype(np.float64)
    for b in range(B):
        f = forward_scan(w, scans[b], guesses[b], center, scale, max_points, bf16_mode,
                         None if argmaxes is None else argmaxes[b])
        dy = f["y"] - np.asarray(targets[b], np.float64)
        loss += float(np.mean(dy ** 2))
        if bf16_mode:
            # per-scan head gradient on the tensor cores (BF16 operands), the batch mean taken at the end
            dy = dy * (2.0 / OUT)
            G["W4"] += np.outer(_b(dy), _b(f["h3"])) / B
            G["b4"] += dy / B
            dh3 = (_b(W4).T @ _b(dy)) * (f["h3"] > 0)
            G["W3"] += np.outer(_b(dh3), _b(f["g"])) / B
            G["b3"] += dh3 / B
            dg = (_b(W3).T @ _b(dh3)) * (f["g"] > 0) / B
        else:
            dy = dy * (2.0 / OUT) / B
            G["W4"] += np.outer(dy, f["h3"])
            G["b4"] += dy
            dh3 = (W4.T @ dy) * (f["h3"] > 0)
            G["W3"] += np.outer(dh3, f["g"])
            G["b3"] += dh3
            dg = (W3.T @ dh3) * (f["g"] > 0)
        if len(f["u"]) == 0:
            continue
        rows = f["arg"]
        a_rows = f["a"][rows]            # (128, 64) operands of the argmax points
        G["W2"] += dg[:, None] * a_rows
        G["b2"] += dg
        # through W2 (its BF16 value in bf16 mode), the ReLU of layer 1, to W1, b1
        dz1 = (dg[:, None] * f["W2"]) * (f["h1"][rows] > 0)   # (128 channels, 64)
        u_rows = f["u"][rows].astype(np.float64)
        G["W1"] += dz1.T @ u_rows
        G["b1"] += dz1.sum(axis=0)
    return loss / B, grad
