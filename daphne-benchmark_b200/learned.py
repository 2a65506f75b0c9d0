"""Learned initial pose for batched NDT: training-pair generation with the
plain GPU NDT, training of the point-feature network on the GPU, and the
proposal -> judge -> refine pipeline.

Pipeline for a batch of (scan, guess) (`LearnedBatch`, one call of the C
entry point ndt_align_batch_learned_device; `learned_align` restates it step
by step through the single-purpose entry points):
  1. the network proposes corrected poses from K starts around the guess (a
     grid of translations and yaw offsets; `PoseNet`, tensor-core kernels),
     each start refined by `passes` network passes;
  2. the NDT judges: the score of every proposal and of the raw guess at a
     coarse level (`Context.score_batch_device` on a strided subsample of the
     scan); the start pose is the best-scoring candidate, the raw guess when
     no proposal scores higher (the fallback);
  3. the plain NDT refines every alignment from its start pose through the
     levels (coarse to fine resolution; `refinement_levels`), the last level
     being the plain NDT of the configuration.

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

# Points the network reads per scan (evenly strided), in training and in the
# pipeline: the library's default (ndt_learned_params_default).  On the 16 m
# noiseless-wall scans of the c5 workload 1024 points reach the truth more
# often than 512 at the same batch time (31.7% against 27.5%).
NET_POINTS = 1024


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


def subsample(scan, max_points):
    """The evenly strided subsample a pipeline level reads (the library's
    subsample_kernel): point (j n) / m of the scan for j < m = min(n,
    max_points); the whole scan when max_points is 0 or None."""
    n = len(scan)
    if not max_points or n <= max_points:
        return scan
    return np.ascontiguousarray(scan[(np.arange(max_points) * n) // max_points])


class DeviceScans:
    """Scans resident on the device (concatenated), with helpers that build
    packed batches of pairs by gathering on the device."""

    def __init__(self, torch, scans, max_points=None):
        self.torch = torch
        if max_points:
            scans = [subsample(s, max_points) for s in scans]
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


def train(net, torch, pairs: Pairs, epochs=4, batch=512, lr=2e-3, max_points=NET_POINTS, seed=0, log=None):
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


def propose(net, torch, pts, offs, guesses_np, max_points=NET_POINTS):
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


def refinement_levels(resolution, step=0.1, max_iterations=30, eps=0.01):
    """The refinement levels, coarse to fine: dicts of the corrected-NDT
    parameters that differ per level, and the points per scan each level
    reads (an evenly strided subsample; 0 = all).  4 r and 2 r take longer
    steps (the step limits how far one Newton iteration moves the pose: 2 r
    and 0.8 r; on c5 these reach the truth on 32.4 % of the alignments against
    29.5 % with 1 r and 0.4 r, at 5 % more time) on 4096 and 8192 points; the
    last level is the plain NDT of the configuration (its own r, step,
    iterations and epsilon) on every point."""
    return [dict(resolution=4.0 * resolution, step_size=2.0 * resolution, max_iterations=max_iterations,
                 transformation_epsilon=eps, points_per_scan=4096),
            dict(resolution=2.0 * resolution, step_size=0.8 * resolution, max_iterations=max_iterations,
                 transformation_epsilon=eps, points_per_scan=8192),
            dict(resolution=resolution, step_size=step, max_iterations=max_iterations, transformation_epsilon=eps,
                 points_per_scan=0)]


def pipeline_params(levels, **kw):
    """ndt_learned_params for `levels` (refinement_levels): the library defaults with each level's point
    count, overridden by keyword."""
    kw.setdefault("level_points", [lvl.get("points_per_scan", 0) for lvl in levels])
    return posenet.learned_params(**kw)


def level_params(prm, level):
    """Sets a level's NDT fields on a corrected-NDT parameter struct (ndt.Params or the oracle's); returns it."""
    for k, v in level.items():
        if k != "points_per_scan":
            setattr(prm, k, v)
    return prm


def level_contexts(ndt, cloud, resolution, device=0, levels=None):
    """Corrected-NDT contexts holding `cloud` at every refinement level."""
    out = []
    for lvl in (levels or refinement_levels(resolution)):
        c = ndt.Context(level_params(ndt.corrected_params(lvl["resolution"]), lvl), device=device)
        c.set_map(cloud)
        out.append(c)
    return out


class LearnedBatch:
    """Device buffers of the learned pipeline for one batch; run() enqueues the
    whole pipeline (ndt_align_batch_learned_device: proposals from the starts,
    the judge's score pass, refinement through the levels) and waits for the
    last level."""

    def __init__(self, levels, net, torch, pts, offs, total, guesses_np, params=None):
        B = len(guesses_np)
        self.levels, self.net, self.torch = levels, net, torch
        self.pts, self.offs, self.total, self.B = pts, offs, total, B
        self.params = params if params is not None else pipeline_params(refinement_levels(1.0))
        self.g = torch.from_numpy(np.ascontiguousarray(guesses_np, np.float32)).cuda()
        self.out = torch.zeros((B, 16), dtype=torch.float32, device="cuda")
        self.conv = torch.zeros(B, dtype=torch.int32, device="cuda")
        self.fit = torch.zeros(B, dtype=torch.float64, device="cuda")
        self.st = torch.zeros(B, dtype=torch.int32, device="cuda")
        self.choice = torch.zeros(B, dtype=torch.int32, device="cuda")
        self.start = torch.zeros((B, 16), dtype=torch.float32, device="cuda")
        torch.cuda.current_stream().synchronize()

    def run(self):
        self.net.align_learned_device(self.levels, self.params, self.B, self.pts.data_ptr(), self.offs.data_ptr(),
                                      self.total, self.g.data_ptr(), self.out.data_ptr(), self.conv.data_ptr(),
                                      self.fit.data_ptr(), self.st.data_ptr(), self.choice.data_ptr(),
                                      self.start.data_ptr())
        self.levels[-1].synchronize()
        if self.net.synchronize_status():
            raise RuntimeError("tensor-core wait gave up in the network's kernels")

    def results(self):
        """(out, conv, fit, status, choice, start): choice = K for the raw guess (the fallback), start = the
        pose the refinement started from."""
        return (self.out.cpu().numpy(), self.conv.cpu().numpy(), self.fit.cpu().numpy(), self.st.cpu().numpy(),
                self.choice.cpu().numpy(), self.start.cpu().numpy())

    def close(self):
        pass


def start_offsets(params):
    """(dx, dy, dyaw_rad) of the K starts in the order of the C pipeline (start_kernel)."""
    gxy, gyaw = params.grid_xy, params.grid_yaw
    out = []
    for k in range(gxy * gxy * gyaw):
        iyaw, ixy = k % gyaw, k // gyaw
        ix, iy = ixy % gxy, ixy // gxy
        out.append(((ix - 0.5 * (gxy - 1)) * params.step_xy, (iy - 0.5 * (gxy - 1)) * params.step_xy,
                    math.radians((iyaw - 0.5 * (gyaw - 1)) * params.step_yaw_deg)))
    return out


def learned_align(levels, net, torch, scans, guesses_np, params=None):
    """The learned pipeline step by step through the single-purpose entry
    points (network proposals, score pass, plain NDT per level), with the
    judge's choice made here on the host.  Same arithmetic as LearnedBatch:
    returns (out, conv, fit, status, choice)."""
    params = params if params is not None else pipeline_params(refinement_levels(1.0))
    B = len(guesses_np)
    dev = DeviceScans(torch, scans)
    pts, offs, total = dev.batch(np.arange(B))
    cands = []
    for dx, dy, dyaw in start_offsets(params):
        p = posenet.poses_from_matrices(guesses_np)
        c, s_ = np.cos(p[:, 5]), np.sin(p[:, 5])
        p[:, 0] += c * dx - s_ * dy
        p[:, 1] += s_ * dx + c * dy
        p[:, 5] += dyaw
        g = posenet.matrices_from_poses(p)
        if params.passes > 0:
            g = propose_passes(net, torch, pts, offs, g, params.passes, params.max_points)
        cands.append(g)
    cands.append(np.asarray(guesses_np, np.float32))
    judge = levels[params.judge_level]
    sub = DeviceScans(torch, scans, max_points=params.judge_points or None)
    sp, so, st = sub.batch(np.arange(B))
    scores = np.stack([score(judge, torch, sp, so, st, g) for g in cands])
    K = len(cands) - 1
    choice = np.full(B, K, np.int64)
    best = scores[K].copy()
    for k in range(K):
        win = (scores[k] > best) | (np.isnan(best) & ~np.isnan(scores[k]))
        choice[win] = k
        best[win] = scores[k][win]
    cur = np.stack(cands)[choice, np.arange(B)]
    status = np.zeros(B, np.int32)
    out = conv = fit = None
    for l, ctx in enumerate(levels):
        cap = params.level_points[l]
        if cap > 0:
            lv = DeviceScans(torch, scans, max_points=cap)
            lp_, lo_, lt_ = lv.batch(np.arange(B))
        else:
            lp_, lo_, lt_ = pts, offs, total
        out, conv, fit, st_l = ndt_align_device(ctx, torch, lp_, lo_, lt_, cur)
        status |= st_l
        cur = out
    return out, conv, fit, status, choice.astype(np.int32)


def propose_passes(net, torch, pts, offs, guesses_np, passes, max_points=NET_POINTS):
    """The network's proposals after `passes` passes (device-side application, ndt_mlp_propose_device)."""
    B = len(guesses_np)
    g = torch.from_numpy(np.ascontiguousarray(guesses_np, np.float32)).cuda()
    y = torch.zeros((B, 6), dtype=torch.float32, device="cuda")
    prop = torch.zeros((B, 16), dtype=torch.float32, device="cuda")
    torch.cuda.current_stream().synchronize()
    net.propose_device(B, pts.data_ptr(), offs.data_ptr(), g.data_ptr(), y.data_ptr(), prop.data_ptr(), passes,
                       max_points)
    net.synchronize()
    return prop.cpu().numpy()


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
