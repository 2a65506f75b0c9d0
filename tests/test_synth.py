"""The synthetic workload generator is deterministic and shaped like the
benchmark configurations."""
import numpy as np


def test_deterministic(pkg):
    cfg = pkg.synth.small_config("t", 3000, 20.0, 5, 300, seed=3)
    s1 = pkg.synth.make_scene(cfg)
    s2 = pkg.synth.make_scene(cfg)
    a1 = pkg.synth.make_alignment(cfg, s1, 4)
    a2 = pkg.synth.make_alignment(cfg, s2, 4)
    assert pkg.synth.digest(s1.map, a1.scan, a1.guess) == pkg.synth.digest(s2.map, a2.scan, a2.guess)


def test_shapes_and_perturbation(pkg):
    cfg = pkg.synth.small_config("t", 5000, 30.0, 8, 400, seed=4, dt=0.5, dyaw_deg=3.0)
    scene = pkg.synth.make_scene(cfg)
    assert scene.map.shape == (5000, 4) and scene.map.dtype == np.float32
    assert np.all(scene.map[:, 3] == 1.0)
    for i in range(5):
        a = pkg.synth.make_alignment(cfg, scene, i)
        assert a.scan.shape == (400, 4)
        G = a.guess.reshape(4, 4).astype(np.float64)
        d = G[:2, 3] - a.truth[:2, 3]
        assert np.all(np.abs(d) <= 0.5 + 1e-6)
        dyaw = np.degrees(np.arctan2(G[1, 0], G[0, 0]) - np.arctan2(a.truth[1, 0], a.truth[0, 0]))
        dyaw = (dyaw + 180) % 360 - 180
        assert abs(dyaw) <= 3.0 + 1e-6
        # the scan is the map's surfaces seen from the true pose: within 40 m
        assert np.all(np.linalg.norm(a.scan[:, :3].astype(np.float64), axis=1) < 40.0 + 1e-3)


def test_leaf_order(pkg):
    cfg = pkg.synth.small_config("t", 5000, 30.0, 8, 400, seed=4)
    scene = pkg.synth.make_scene(cfg)
    a = pkg.synth.make_alignment(cfg, scene, 0)
    q = np.floor(a.scan[:, :3].astype(np.float64) / 2.0).astype(np.int64) + 1024
    key = (q[:, 2] * 2048 + q[:, 1]) * 2048 + q[:, 0]
    assert np.all(np.diff(key) >= 0)


def test_configs_match_benchmark_sizes(pkg):
    C = pkg.synth.CONFIGS
    assert (C["c1"].map_points, C["c1"].scan_min, C["c1"].area, C["c1"].walls) == (60_000, 2000, 60.0, 30)
    assert (C["c2"].map_points, C["c2"].aligns, C["c2"].scan_min) == (400_000, 256, 8000)
    assert (C["c3"].aligns, C["c3"].scan_min, C["c3"].scan_max, C["c3"].dt, C["c3"].dyaw_deg) == (1024, 1000, 16000, 1.0, 5.0)
    assert (C["c5"].map_points, C["c5"].resolution, C["c5"].aligns, C["c5"].scan_max) == (2_000_000, 0.5, 4096, 32000)
    for i in range(20):
        n = pkg.synth.scan_size(C["c3"], i)
        assert 1000 <= n <= 16000
