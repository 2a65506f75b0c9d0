"""Probe-window table against the dense-index probe and the FP64 oracle.

The FP32 derivative pass finds a point's voxels through the probe-window table
(one record per usable voxel of the 3 x 3 x 3 cells around the point's first
probe coordinate) unless the context is created with dense_probe = 1, in which
case it reads the 27 dense-index entries like the reference's loop
(voxelRadiusSearch, src/CPU/ndt_mapping/kernel.cpp:246-286).  Both must accept
exactly the reference's (point, voxel) pairs, so:
  * the probe, occupied-probe and pair counters of the two paths are equal;
  * the pair count equals the FP64 oracle's;
  * the derivatives agree with the oracle's (FP32 pairs: 2e-3 relative to the
    largest entry of each block; FP64 pairs: 1e-9).
Inputs: points spread uniformly over the map's bounding box grown by 2.5 cells
on every side, plus points placed exactly on each face of the box and one
float step either side of it, so that windows with base cell -2 and dim - 1
and both sides of every bounding-box test occur.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _edge_cloud(lo, hi, res, rng):
    n = 20000
    pts = rng.uniform(lo - 2.5 * res, hi + 2.5 * res, size=(n, 3)).astype(np.float32)
    faces = []
    for e in range(3):
        for v in (lo[e], hi[e], np.nextafter(lo[e], np.float32(-np.inf)), np.nextafter(hi[e], np.float32(np.inf)),
                  np.nextafter(lo[e], np.float32(np.inf)), np.nextafter(hi[e], np.float32(-np.inf))):
            f = rng.uniform(lo, hi, size=(400, 3)).astype(np.float32)
            f[:, e] = v
            faces.append(f)
    pts = np.concatenate([pts] + faces)
    out = np.ones((pts.shape[0], 4), np.float32)
    out[:, :3] = pts
    return out


def _close(a, b, tol):
    return np.max(np.abs(np.asarray(a) - np.asarray(b))) <= tol * max(1.0, float(np.max(np.abs(b))))


@pytest.mark.parametrize("compat", [1, 0])
@pytest.mark.parametrize("precision", [0, 1])
def test_window_pairs_equal_dense_and_oracle(pkg, oracle, binding_mod, compat, precision):
    cfg = pkg.synth.small_config("win", 20000, 40.0, 16, 1500, seed=41)
    scene = pkg.synth.make_scene(cfg)
    make = pkg.ndt.reference_params if compat else pkg.ndt.corrected_params
    omake = binding_mod.reference_params if compat else binding_mod.corrected_params
    rng = np.random.default_rng(7)
    p6 = np.array([0.1, -0.2, 0.05, 0.01, -0.02, 0.3])
    results = {}
    for dense in (0, 1):
        with pkg.ndt.Context(make(precision=precision, dense_probe=dense)) as ctx:
            ctx.set_map(scene.map)
            W, E = ctx.window_info()
            if dense:
                assert (W, E) == (0, 0)
            else:
                assert W > 0 and E > 0
            bbox, _, _ = ctx.grid_info()
            if dense == 0:
                cloud = _edge_cloud(bbox[:3], bbox[3:], cfg.resolution, rng)
                scan = pkg.synth.make_alignment(cfg, scene, 0)
                # a second input: a real scan at its guess
                G = scan.guess.reshape(4, 4)
                strans = np.zeros_like(scan.scan)
                for r in range(3):
                    strans[:, r] = ((G[r, 0] * scan.scan[:, 0] + G[r, 1] * scan.scan[:, 1]) +
                                    G[r, 2] * scan.scan[:, 2]) + G[r, 3]
                inputs = [(cloud, cloud), (scan.scan, strans)]
            res = []
            for src, trans in inputs:
                s, g, H = ctx.derivatives(src, trans, p6)
                k = ctx.counters()
                res.append((s, g, H, k["probes"], k["occupied_probes"], k["pairs"]))
            results[dense] = res
    tol = 1e-9 if precision == 1 else 2e-3
    for idx, (src, trans) in enumerate(inputs):
        w, d = results[0][idx], results[1][idx]
        assert w[3:] == d[3:], ("counters differ between window and dense probe", idx, w[3:], d[3:])
        rs, rg, rH, rpairs = oracle.derivatives(omake(), scene.map, src, trans, p6)
        assert w[5] == rpairs, (idx, w[5], rpairs)
        assert w[5] > 0
        for s, g, H in ((w[0], w[1], w[2]), (d[0], d[1], d[2])):
            assert _close([s], [rs], tol), (idx, s, rs)
            assert _close(g, rg, tol), (idx, g, rg)
            assert _close(H, rH, tol), (idx, H, rH)


def test_window_align_equals_dense(pkg):
    """Whole compat alignments: same converged flags and translation, rotation
    within the FP32 tolerance of the parity tests (only the pair order in the
    FP32 sums differs)."""
    cfg = pkg.synth.small_config("win2", 40000, 60.0, 24, 4000, seed=42)
    scene = pkg.synth.make_scene(cfg)
    aligns = [pkg.synth.make_alignment(cfg, scene, i) for i in range(8)]
    outs = []
    for dense in (0, 1):
        with pkg.ndt.Context(pkg.ndt.reference_params(dense_probe=dense)) as ctx:
            ctx.set_map(scene.map)
            out, conv, fit, status = ctx.align_batch([a.scan for a in aligns], [a.guess for a in aligns])
            k = ctx.counters()
            outs.append((out, conv, status, k["probes"], k["occupied_probes"], k["pairs"]))
            # every derivative pass covers each point and tile of its alignment once
            n = {len(a.scan) for a in aligns}
            assert len(n) == 1
            n = n.pop()
            tile = pkg.ndt.kernel_variants()[ctx.kernel_variant()][0]
            assert k["points"] == n * k["evaluations"], (k["points"], n, k["evaluations"])
            assert k["tiles"] == -(-n // tile) * k["evaluations"]
    (o0, c0, s0, *k0), (o1, c1, s1, *k1) = outs
    assert k0 == k1
    assert np.array_equal(c0, c1) and (s0 == 0).all() and (s1 == 0).all()
    T0, T1 = o0.reshape(-1, 4, 4), o1.reshape(-1, 4, 4)
    assert np.array_equal(T0[:, :, 3].view(np.uint32), T1[:, :, 3].view(np.uint32))
    assert np.nanmax(np.abs(T0[:, :3, :3] - T1[:, :3, :3])) <= 2e-3
