"""What the learned initial pose gains over the plain NDT (GPU).

On a small map (60 x 60 m, 30 walls, 2000-point scans, guesses +-1 m /
+-5 deg, corrected NDT at 1 m resolution) the network is trained on the GPU
on pairs the plain NDT labels (1500 scans x 20 perturbed guesses, 20
epochs), then 256 fresh alignments run both pipelines.  The test checks that
the proposals are closer to the truth than the guesses, that the learned
pipeline (proposal -> NDT judge -> NDT refinement) reaches the truth
(<= 2 cm, <= 0.1 deg) far more often than the plain NDT from the raw
guesses, and that its refinement still agrees with the FP64 oracle run from
the same start poses.
"""
import numpy as np
import pytest

import posenet_ref

pytestmark = pytest.mark.gpu


def test_learned_initial_pose_beats_plain(pkg, binding_mod):
    torch = pytest.importorskip("torch")
    L, synth, ndt = pkg.learned, pkg.synth, pkg.ndt
    cfg = synth.Config("learn_t", 60_000, 60.0, 30, 1.0, 256, 2000, 2000, False, 1.0, 5.0, seed=77)
    scene = synth.make_scene(cfg)
    ctx = ndt.Context(ndt.corrected_params(cfg.resolution))
    ctx.set_map(scene.map)
    pairs = L.make_pairs(cfg, scene, 1500, 20, cfg.dt, cfg.dyaw_deg, seed=3, fine_frac=0.5)
    L.label_scans(ctx, torch, pairs)
    assert pairs.keep.mean() > 0.95
    net = pkg.posenet.PoseNet(center=(0.0, 0.0, 0.0), scale=4.0)
    net.set_weights(posenet_ref.init_weights(1))
    losses = L.train(net, torch, pairs, epochs=20, batch=256, lr=2e-3)
    assert losses[-50:].mean() < 0.5 * losses[:50].mean()
    aligns = [synth.make_alignment(cfg, scene, i) for i in range(256)]
    dev = L.DeviceScans(torch, [a.scan for a in aligns])
    pts, offs, total = dev.batch(np.arange(len(aligns)))
    guesses = np.stack([a.guess for a in aligns])
    truths = np.stack([a.truth for a in aligns])
    prop = guesses
    for _ in range(3):
        prop, _ = L.propose(net, torch, pts, offs, prop)
    g_dt, _ = L.pose_errors(guesses, truths)
    p_dt, _ = L.pose_errors(prop, truths)
    plain = L.ndt_align_device(ctx, torch, pts, offs, total, guesses)
    learned = L.learned_align(ctx, net, torch, pts, offs, total, guesses, passes=3)
    pl_dt, pl_dr = L.pose_errors(plain[0], truths)
    le_dt, le_dr = L.pose_errors(learned[0], truths)
    ok_plain = np.mean((pl_dt <= 0.02) & (pl_dr <= 0.1))
    ok_learned = np.mean((le_dt <= 0.02) & (le_dr <= 0.1))
    print(f"median error guess {np.median(g_dt):.3f} m, proposal {np.median(p_dt):.3f} m; "
          f"within 2 cm / 0.1 deg of truth: plain {ok_plain:.3f}, learned {ok_learned:.3f}")
    assert np.median(p_dt) < 0.6 * np.median(g_dt)
    assert ok_learned >= ok_plain + 0.15
    # the same pipeline enqueued on one stream with device-side proposals and judge
    lb = L.LearnedBatch(ctx, net, torch, pts, offs, total, guesses, passes=3)
    lb.run()
    d_out, d_conv, _, d_st, d_used, _, _ = lb.results()
    lb.close()
    d_dt, d_dr = L.pose_errors(d_out, truths)
    ok_device = np.mean((d_dt <= 0.02) & (d_dr <= 0.1))
    assert (d_st == 0).all()
    assert ok_device >= ok_plain + 0.15
    assert abs(ok_device - ok_learned) <= 0.05
    # the refinement from the chosen starts against the FP64 oracle (sample)
    s_p = L.score(ctx, torch, pts, offs, total, prop)
    s_g = L.score(ctx, torch, pts, offs, total, guesses)
    starts = np.where((s_p >= s_g)[:, None], prop, guesses).astype(np.float32)
    gpu = L.ndt_align_device(ctx, torch, pts, offs, total, starts)[0][:24]
    orc = binding_mod.Oracle()
    ref, _, _, _ = orc.align_batch(binding_mod.corrected_params(cfg.resolution), [a.scan for a in aligns[:24]],
                                   list(starts[:24]), scene.map)
    e_t = np.linalg.norm(gpu.reshape(-1, 4, 4)[:, :3, 3] - ref.reshape(-1, 4, 4)[:, :3, 3], axis=1)
    assert e_t.max() <= 0.02
    net.close()
    ctx.close()
