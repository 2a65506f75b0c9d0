"""What the learned initial pose gains (GPU).

On a small map (60 x 60 m, 30 walls, 2000-point scans, guesses +-1 m /
+-5 deg, corrected NDT, refinement levels 4 m -> 2 m -> 1 m) the network is
trained on the GPU on pairs the plain NDT labels (1500 scans x 20 perturbed
guesses, 20 epochs); then 256 fresh alignments run
  * the plain NDT at 1 m from the raw guesses,
  * the learned pipeline (ndt_align_batch_learned_device: network proposals
    from a 3 x 3 grid of starts, the NDT judge at 4 m, refinement through the
    levels),
  * the same pipeline without the network (passes = 0: the judge picks among
    the starts themselves),
  * the pipeline restated step by step on the host through the
    single-purpose entry points (`learned.learned_align`).
Checks: the proposals are closer to the truth than the guesses; the learned
pipeline reaches the truth (<= 2 cm, <= 0.1 deg) far more often than the
plain NDT and more often than the pipeline without the network; the device
pipeline makes the host restatement's choices; and its refinement chain,
run by the FP64 oracle level by level from the same chosen starts, agrees
within 2 cm / 0.1 deg.
"""
import math

import numpy as np
import pytest

from test_gpu_parity import check_fp32_against_oracle

pytestmark = pytest.mark.gpu


def _rot_deg(A, B):
    d = A.reshape(4, 4)[:3, :3].astype(np.float64) - B.reshape(4, 4)[:3, :3].astype(np.float64)
    return math.degrees(2.0 * math.asin(min(1.0, float(np.linalg.norm(d)) / math.sqrt(8.0))))


@pytest.fixture(scope="module")
def trained(pkg):
    torch = pytest.importorskip("torch")
    L, synth, ndt = pkg.learned, pkg.synth, pkg.ndt
    cfg = synth.Config("learn_t", 60_000, 60.0, 30, 1.0, 256, 2000, 2000, False, 1.0, 5.0, seed=77)
    scene = synth.make_scene(cfg)
    levels = L.level_contexts(ndt, scene.map, cfg.resolution)
    pairs = L.make_pairs(cfg, scene, 1500, 20, cfg.dt, cfg.dyaw_deg, seed=3, fine_frac=0.5)
    L.label_scans(levels[-1], torch, pairs)
    assert pairs.keep.mean() > 0.95
    net = pkg.posenet.PoseNet(center=(0.0, 0.0, 0.0), scale=4.0)
    net.set_weights(pkg.posenet.init_weights(1))
    losses = L.train(net, torch, pairs, epochs=20, batch=256, lr=2e-3)
    assert losses[-50:].mean() < 0.5 * losses[:50].mean()
    aligns = [synth.make_alignment(cfg, scene, i) for i in range(256)]
    yield cfg, scene, levels, net, aligns
    net.close()
    for c in levels:
        c.close()


def _ok(L, out, truths):
    dt, dr = L.pose_errors(out, truths)
    return (dt <= 0.02) & (dr <= 0.1)


def test_learned_pipeline_gain(pkg, trained):
    torch = pytest.importorskip("torch")
    L = pkg.learned
    cfg, scene, levels, net, aligns = trained
    dev = L.DeviceScans(torch, [a.scan for a in aligns])
    pts, offs, total = dev.batch(np.arange(len(aligns)))
    guesses = np.stack([a.guess for a in aligns])
    truths = np.stack([a.truth for a in aligns])
    prop = L.propose_passes(net, torch, pts, offs, guesses, 3)
    g_dt, _ = L.pose_errors(guesses, truths)
    p_dt, _ = L.pose_errors(prop, truths)
    assert np.median(p_dt) < 0.6 * np.median(g_dt)

    plain = L.ndt_align_device(levels[-1], torch, pts, offs, total, guesses)
    prm = pkg.posenet.learned_params(grid_xy=3, grid_yaw=1, passes=3, step_xy=0.5, judge_points=1024)
    lb = L.LearnedBatch(levels, net, torch, pts, offs, total, guesses, prm)
    lb.run()
    out, conv, fit, st, choice, _ = lb.results()
    nonet = L.LearnedBatch(levels, net, torch, pts, offs, total, guesses,
                           pkg.posenet.learned_params(grid_xy=3, grid_yaw=1, step_xy=0.5, judge_points=1024, passes=0))
    nonet.run()
    out0 = nonet.results()[0]
    ok_plain, ok_learned, ok_nonet = (float(_ok(L, o, truths).mean()) for o in (plain[0], out, out0))
    print(f"median error guess {np.median(g_dt):.3f} m, proposal {np.median(p_dt):.3f} m; within 2 cm / 0.1 deg "
          f"of truth: plain {ok_plain:.3f}, without the network {ok_nonet:.3f}, learned {ok_learned:.3f}; "
          f"raw guess kept for {np.mean(choice == 9):.3f}")
    assert (st == 0).all() and (conv != 0).all()
    assert ok_learned >= ok_plain + 0.15
    assert ok_learned >= ok_nonet + 0.05
    assert choice.min() >= 0 and choice.max() <= 9

    # the same pipeline restated on the host through the single-purpose entry points
    h_out, _, _, h_st, h_choice = L.learned_align(levels, net, torch, [a.scan for a in aligns], guesses, prm)
    agree = choice == h_choice
    assert agree.mean() >= 0.97, agree.mean()
    same = np.all(out[agree].view(np.uint32) == h_out[agree].view(np.uint32), axis=1)
    assert same.mean() >= 0.97, same.mean()
    assert abs(float(_ok(L, h_out, truths).mean()) - ok_learned) <= 0.03


def test_learned_refinement_vs_fp64_oracle(pkg, trained, binding_mod, oracle):
    """The refinement levels from the judge's chosen starts (the pipeline's
    d_start16 output), run by the FP64 oracle level by level (same
    resolutions and step sizes), against the device pipeline's result:
    <= 2 cm / 0.1 deg on a sample, except where the oracle's own chain is
    not reproducible at that start (check_fp32_against_oracle)."""
    torch = pytest.importorskip("torch")
    L = pkg.learned
    cfg, scene, levels, net, aligns = trained
    sample = aligns[:32]
    scans = [a.scan for a in sample]
    guesses = np.stack([a.guess for a in sample])
    prm = pkg.posenet.learned_params(grid_xy=3, grid_yaw=1, passes=3, step_xy=0.5, judge_points=1024)
    dev = L.DeviceScans(torch, scans)
    pts, offs, total = dev.batch(np.arange(len(sample)))
    lb = L.LearnedBatch(levels, net, torch, pts, offs, total, guesses, prm)
    lb.run()
    out, conv, _, st, choice, cur = lb.results()
    starts = cur.copy()
    prms = []
    for lvl in L.refinement_levels(cfg.resolution):
        prms.append((L.level_params(binding_mod.corrected_params(lvl["resolution"]), lvl), lvl["points_per_scan"]))

    def chain(i, g):
        for op, cap in prms:  # each level on the points the pipeline gives it
            g = oracle.align(op, L.subsample(scans[i], cap), g, scene.map)[0]
        return g

    ref = np.stack([chain(i, starts[i]) for i in range(len(sample))])
    runs = [lambda g, i=i: chain(i, g) for i in range(len(sample))]
    bad, worst = check_fp32_against_oracle(out, ref, conv, conv, st, runs, starts, max_frac=0.1)
    print(f"learned refinement vs FP64 oracle: {len(sample) - len(bad)}/{len(sample)} within 2 cm / 0.1 deg, "
          f"worst {worst[0]:.2e} m, {worst[1]:.2e} deg")


def test_learned_pipeline_edge_cases(pkg, trained):
    """Ragged and empty scans, a batch of one, the same call twice (bit-identical),
    and bad arguments (NDT_E_ARG, nothing enqueued)."""
    torch = pytest.importorskip("torch")
    import ctypes as C
    L = pkg.learned
    cfg, scene, levels, net, aligns = trained
    sizes = [0, 1, 5, 3000, 64, 0, 700]
    scans = []
    for k, n in enumerate(sizes):
        s = aligns[k].scan
        scans.append(np.ascontiguousarray(s[(np.arange(n) * len(s)) // max(n, 1)]) if n else np.zeros((0, 4), np.float32))
    guesses = np.stack([aligns[k].guess for k in range(len(sizes))])
    dev = L.DeviceScans(torch, scans)
    pts, offs, total = dev.batch(np.arange(len(sizes)))
    prm = pkg.posenet.learned_params(grid_xy=2, grid_yaw=2, step_xy=0.5, step_yaw_deg=3.0, judge_points=512,
                                     level_points=[256, 512, 0])
    lb = L.LearnedBatch(levels, net, torch, pts, offs, total, guesses, prm)
    lb.run()
    r1 = lb.results()
    lb.run()
    r2 = lb.results()
    for a, b in zip(r1, r2):
        assert np.array_equal(np.asarray(a).view(np.uint8), np.asarray(b).view(np.uint8))
    out, conv, fit, st, choice, start = r1
    assert np.isfinite(out).all() and (st == 0).all()
    assert choice.min() >= 0 and choice.max() <= 8
    for k, n in enumerate(sizes):
        if n == 0:
            assert fit[k] == 0.0
    one = L.LearnedBatch(levels, net, torch, *dev.batch(np.array([3])), guesses[3:4], prm)
    one.run()
    assert np.array_equal(one.results()[0].view(np.uint32), out[3:4].view(np.uint32))  # batch-independent
    # argument errors
    arr = (C.c_void_p * len(levels))(*[c.h.value for c in levels])
    f = net.L.ndt_align_batch_learned_device
    bad = [pkg.posenet.learned_params(grid_xy=0), pkg.posenet.learned_params(judge_level=3),
           pkg.posenet.learned_params(max_points=0)]
    for p in bad:
        rc = f(net.h, arr, len(levels), C.byref(p), len(sizes), C.c_void_p(pts.data_ptr()),
               C.c_void_p(offs.data_ptr()), total, C.c_void_p(lb.g.data_ptr()), C.c_void_p(lb.out.data_ptr()),
               C.c_void_p(lb.conv.data_ptr()), C.c_void_p(lb.fit.data_ptr()), None, None, None)
        assert rc == -1  # NDT_E_ARG
    rc = f(net.h, arr, 0, C.byref(prm), len(sizes), C.c_void_p(pts.data_ptr()), C.c_void_p(offs.data_ptr()), total,
           C.c_void_p(lb.g.data_ptr()), C.c_void_p(lb.out.data_ptr()), C.c_void_p(lb.conv.data_ptr()),
           C.c_void_p(lb.fit.data_ptr()), None, None, None)
    assert rc == -1
