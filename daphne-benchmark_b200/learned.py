"""Learned initial pose for batched NDT: training-pair generation with the
plain GPU NDT, training of the point-feature network on the GPU, and the
proposal -> judge -> refine pipeline.

Pipeline for a batch of (scan, guess):
  1. the network proposes a corrected pose from the scan seen at its guess
     (`PoseNet.forward`, tensor-core kernels);
  2. the NDT judges: the score of the scan at the proposal and at the raw
     guess (`Context.score_batch_device`, one derivative pass each); the
     start pose is the proposal where its score is at least the guess's, the
     raw guess otherwise (the fallback);
  3. the plain NDT refines every alignment from its start pose (one batch).

Training pairs: (scan, perturbed guess -> converged pose), generated on the
GPU by the same library: the converged pose is where the plain NDT settles
for the scan from a near-correct start (label_scans), the guess a
perturbation of the scan's pose, and the network's target the correction from
the guess to the converged pose (posenet.correction_targets).  (Running the
NDT from the perturbed guesses themselves labels nothing useful when the
perturbations exceed its capture range: it stops near the guess.)  Only
pairs whose NDT run reports convergence are kept.
"""
from __future__ import annotations

import dataclasses
import math
import time

import numpy as np

from . import posenet, synth


@dataclasses.dataclass
class Pairs:
    scans: list            # S full scans (n_s x 4 float32)
    truths: np.ndarray     # S x 4 x 4
    pair_scan: np.ndarray  # P: scan index of each pair
    guesses: np.ndarray    # P x 16 float32
    targets: np.ndarray | None = None    # P x 16 converged poses (float32)
    keep: np.ndarray | None = None       # P bool (converged)


def perturbed_guess(truth, rng, dt, dyaw_deg):
    """Ground truth with uniform +-dt translation on x, y and +-dyaw on yaw."""
    ang = math.radians(dyaw_deg) * (rng.random() * 2 - 1)
    c, s = math.cos(ang), math.sin(ang)
    R = np.array([[c, -s, 0], [s, c, 0], [0, 0, 1.0]])
    g = np.eye(4)
    g[:3, :3] = truth[:3, :3] @ R
    g[:3, 3] = truth[:3, 3]
    g[0, 3] += (rng.random() * 2 - 1) * dt
    g[1, 3] += (rng.random() * 2 - 1) * dt
    return g.astype(np.float32).reshape(16)


def make_pairs(cfg, scene, n_scans, per_scan, dt, dyaw_deg, seed, first_index=100000, fine_frac=0.0,
               fine=0.25):
    """n_scans fresh scans of the scene (indices first_index + i, disjoint from
    a config's evaluation alignments), per_scan perturbed guesses each: up to
    +-dt / +-dyaw_deg, or, for a fraction fine_frac of them, up to fine times
    that (so that the network also learns the small corrections that a second
    pass over its own proposal needs)."""
    rng = np.random.default_rng(seed)
    scans, truths, pair_scan, guesses = [], [], [], []
    for i in range(n_scans):
        a = synth.make_alignment(cfg, scene, first_index + i)
        scans.append(a.scan)
        truths.append(a.truth)
        for _ in range(per_scan):
            f = fine if rng.random() < fine_frac else 1.0
            pair_scan.append(i)
            guesses.append(perturbed_guess(a.truth, rng, dt * f, dyaw_deg * f))
    return Pairs(scans, np.stack(truths), np.asarray(pair_scan, np.int64), np.stack(guesses))


class DeviceScans:
    """Scans resident on the device (concatenated), with helpers that build
    packed batches of pairs by gathering on the device."""

    def __init__(self, torch, scans, max_points=None):
        self.torch = torch
        if max_points:
            scans = [s[(np.arange(min(len(s), max_points)) * len(s)) // max(1, min(len(s), max_points))]
                     for s in scans]
        self.sizes = np.array([len(s) for s in scans], np.int64)
        self.starts = np.zeros(len(scans) + 1, np.int64)
        self.starts[1:] = np.cumsum(self.sizes)
        self.points = torch.from_numpy(np.ascontiguousarray(np.concatenate(scans))).cuda()

    def batch(self, scan_idx):
        """Points (concatenated) and offsets (int32) of the given scans, on the device."""
        t = self.torch
        scan_idx = np.asarray(scan_idx, np.int64)
        sizes = self.sizes[scan_idx]
        offs = np.zeros(len(scan_idx) + 1, np.int64)
        offs[1:] = np.cumsum(sizes)
        src = np.repeat(self.starts[scan_idx] - offs[:-1], sizes) + np.arange(offs[-1])
        idx = t.from_numpy(src).cuda()
        pts = self.points.index_select(0, idx)
        offs_d = t.from_numpy(offs.astype(np.int32)).cuda()
        t.cuda.current_stream().synchronize()  # the library works on its own streams
        return pts, offs_d, int(offs[-1])


def ndt_align_device(ctx, torch, pts, offs, total, guesses_np):
    """Plain batched NDT from the given guesses; returns (out, conv, fit, status) on the host."""
    B = len(guesses_np)
    g = torch.from_numpy(np.ascontiguousarray(guesses_np, np.float32)).cuda()
    out = torch.zeros((B, 16), dtype=torch.float32, device="cuda")
    conv = torch.zeros(B, dtype=torch.int32, device="cuda")
    fit = torch.zeros(B, dtype=torch.float64, device="cuda")
    st = torch.zeros(B, dtype=torch.int32, device="cuda")
    torch.cuda.current_stream().synchronize()
    ctx.align_batch_device(B, pts.data_ptr(), offs.data_ptr(), total, g.data_ptr(), out.data_ptr(), conv.data_ptr(),
                           fit.data_ptr(), st.data_ptr())
    ctx.synchronize()
    return out.cpu().numpy(), conv.cpu().numpy(), fit.cpu().numpy(), st.cpu().numpy()


def label_scans(ctx, torch, pairs: Pairs, chunk=4096):
    """Labels every pair with the pose the plain NDT converges to for its scan
    from a near-correct start (the scan's sensor pose): the training target
    is that pose, reached from the pair's perturbed guess."""
    dev = DeviceScans(torch, pairs.scans)
    S = len(pairs.scans)
    conv_pose = np.zeros((S, 16), np.float32)
    ok = np.zeros(S, bool)
    starts = pairs.truths.astype(np.float32).reshape(S, 16)
    for lo in range(0, S, chunk):
        hi = min(S, lo + chunk)
        pts, offs, total = dev.batch(np.arange(lo, hi))
        out, conv, _, st = ndt_align_device(ctx, torch, pts, offs, total, starts[lo:hi])
        conv_pose[lo:hi] = out
        ok[lo:hi] = (conv != 0) & (st == 0) & np.isfinite(out).all(axis=1)
    pairs.targets = conv_pose[pairs.pair_scan]
    pairs.keep = ok[pairs.pair_scan]
    return pairs


def label_pairs(ctx, torch, pairs: Pairs, chunk=4096):
    """Runs the plain NDT from every guess; targets = converged poses."""
    dev = DeviceScans(torch, pairs.scans)
    P = len(pairs.guesses)
    targets = np.zeros((P, 16), np.float32)
    keep = np.zeros(P, bool)
    for lo in range(0, P, chunk):
        hi = min(P, lo + chunk)
        pts, offs, total = dev.batch(pairs.pair_scan[lo:hi])
        out, conv, _, st = ndt_align_device(ctx, torch, pts, offs, total, pairs.guesses[lo:hi])
        targets[lo:hi] = out
        keep[lo:hi] = (conv != 0) & (st == 0) & np.isfinite(out).all(axis=1)
    pairs.targets, pairs.keep = targets, keep
    return pairs


def train(net, torch, pairs: Pairs, epochs=4, batch=512, lr=2e-3, max_points=512, seed=0, log=None):
    """Trains the network on the kept pairs (points subsampled to max_points,
    the same points its forward samples at inference)."""
    dev = DeviceScans(torch, pairs.scans, max_points=max_points)
    idx_all = np.flatnonzero(pairs.keep)
    tgt = posenet.correction_targets(pairs.guesses[idx_all], pairs.targets[idx_all], net.delta_scale)
    rng = np.random.default_rng(seed)
    losses = []
    steps = max(1, len(idx_all) // batch)
    total_steps = epochs * steps
    k = 0
    for ep in range(epochs):
        order = rng.permutation(len(idx_all))
        for s in range(steps):
            sel = order[s * batch:(s + 1) * batch]
            pi = idx_all[sel]
            pts, offs, _ = dev.batch(pairs.pair_scan[pi])
            g = torch.from_numpy(np.ascontiguousarray(pairs.guesses[pi])).cuda()
            t = torch.from_numpy(np.ascontiguousarray(tgt[sel])).cuda()
            torch.cuda.current_stream().synchronize()
            rate = lr * 0.5 * (1 + math.cos(math.pi * k / total_steps))  # cosine decay
            loss, _ = net.train_step(len(pi), pts.data_ptr(), offs.data_ptr(), g.data_ptr(), t.data_ptr(),
                                     lr=rate, update=True, max_points=max_points)
            losses.append(loss)
            k += 1
        if log:
            log(f"epoch {ep}: loss {np.mean(losses[-steps:]):.4f}")
    net.synchronize()
    return np.asarray(losses)


def propose(net, torch, pts, offs, guesses_np, max_points=512):
    """Network proposals (B x 16 float32) for scans at their guesses."""
    B = len(guesses_np)
    g = torch.from_numpy(np.ascontiguousarray(guesses_np, np.float32)).cuda()
    y = torch.zeros((B, 6), dtype=torch.float32, device="cuda")
    torch.cuda.current_stream().synchronize()
    net.forward(B, pts.data_ptr(), offs.data_ptr(), g.data_ptr(), y.data_ptr(), max_points)
    net.synchronize()
    yh = y.cpu().numpy()
    return posenet.apply_corrections(guesses_np, yh, net.delta_scale), yh


def score(ctx, torch, pts, offs, total, poses_np):
    B = len(poses_np)
    p = torch.from_numpy(np.ascontiguousarray(poses_np, np.float32)).cuda()
    s = torch.zeros(B, dtype=torch.float64, device="cuda")
    torch.cuda.current_stream().synchronize()
    ctx.score_batch_device(B, pts.data_ptr(), offs.data_ptr(), total, p.data_ptr(), s.data_ptr())
    ctx.synchronize()
    return s.cpu().numpy()


class LearnedBatch:
    """Device buffers of the learned pipeline for one batch; run() enqueues
    proposal passes, the two score passes, the judge and the refinement on the
    NDT context's stream (the network is put on that stream), with one
    synchronisation at the end."""

    def __init__(self, ctx, net, torch, pts, offs, total, guesses_np, max_points=512, passes=3):
        B = len(guesses_np)
        self.ctx, self.net, self.torch = ctx, net, torch
        self.pts, self.offs, self.total, self.B = pts, offs, total, B
        self.max_points, self.passes = max_points, passes
        f32 = dict(dtype=torch.float32, device="cuda")
        self.g = torch.from_numpy(np.ascontiguousarray(guesses_np, np.float32)).cuda()
        self.y = torch.zeros((B, 6), **f32)
        self.prop = torch.zeros((B, 16), **f32)
        self.start = torch.zeros((B, 16), **f32)
        self.s_p = torch.zeros(B, dtype=torch.float64, device="cuda")
        self.s_g = torch.zeros(B, dtype=torch.float64, device="cuda")
        self.used = torch.zeros(B, dtype=torch.int32, device="cuda")
        self.out = torch.zeros((B, 16), **f32)
        self.conv = torch.zeros(B, dtype=torch.int32, device="cuda")
        self.fit = torch.zeros(B, dtype=torch.float64, device="cuda")
        self.st = torch.zeros(B, dtype=torch.int32, device="cuda")
        torch.cuda.current_stream().synchronize()
        net.set_stream(ctx.stream)

    def run(self):
        n, c, B = self.net, self.ctx, self.B
        n.propose_device(B, self.pts.data_ptr(), self.offs.data_ptr(), self.g.data_ptr(), self.y.data_ptr(),
                         self.prop.data_ptr(), self.passes, self.max_points)
        c.score_batch_device(B, self.pts.data_ptr(), self.offs.data_ptr(), self.total, self.prop.data_ptr(),
                             self.s_p.data_ptr())
        c.score_batch_device(B, self.pts.data_ptr(), self.offs.data_ptr(), self.total, self.g.data_ptr(),
                             self.s_g.data_ptr())
        n.judge_device(B, self.prop.data_ptr(), self.g.data_ptr(), self.s_p.data_ptr(), self.s_g.data_ptr(),
                       self.start.data_ptr(), self.used.data_ptr())
        c.align_batch_device(B, self.pts.data_ptr(), self.offs.data_ptr(), self.total, self.start.data_ptr(),
                             self.out.data_ptr(), self.conv.data_ptr(), self.fit.data_ptr(), self.st.data_ptr())
        c.synchronize()

    def results(self):
        return (self.out.cpu().numpy(), self.conv.cpu().numpy(), self.fit.cpu().numpy(), self.st.cpu().numpy(),
                self.used.cpu().numpy() != 0, self.prop.cpu().numpy(), self.start.cpu().numpy())

    def close(self):
        self.net.set_stream(None)


def learned_align(ctx, net, torch, pts, offs, total, guesses_np, max_points=512, passes=1):
    """Proposal (the network applied `passes` times, each pass to the previous
    proposal) -> judge -> refine.  Returns (out, conv, fit, status, used_proposal)."""
    prop = guesses_np
    for _ in range(passes):
        prop, _ = propose(net, torch, pts, offs, prop, max_points)
    s_prop = score(ctx, torch, pts, offs, total, prop)
    s_guess = score(ctx, torch, pts, offs, total, guesses_np)
    use = s_prop >= s_guess
    start = np.where(use[:, None], prop, guesses_np).astype(np.float32)
    out, conv, fit, st = ndt_align_device(ctx, torch, pts, offs, total, start)
    return out, conv, fit, st, use


def pose_errors(out, truths):
    """Translation (m) and rotation (deg) error of each result against its truth."""
    dt = np.linalg.norm(out.reshape(-1, 4, 4)[:, :3, 3] - truths[:, :3, 3], axis=1)
    d = out.reshape(-1, 4, 4)[:, :3, :3].astype(np.float64) - truths[:, :3, :3]
    dr = np.degrees(2 * np.arcsin(np.clip(np.linalg.norm(d, axis=(1, 2)) / math.sqrt(8), 0, 1)))
    return dt, dr


def timed(fn, torch):
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    r = fn()
    torch.cuda.synchronize()
    return r, time.perf_counter() - t0
