"""ndt_dat_align: test cases read from a memory-mapped ndt_input.dat and
aligned in chunks that share a map give, case by case, the same results bit
for bit as aligning each case's scan against its own map with the batch call
(including a grown map, a new map and chunks of more than 512 cases)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _write(pkg, tmp_path, cfg, scene, n_same, grow_pts=4000):
    al = [pkg.synth.make_alignment(cfg, scene, i) for i in range(n_same + 4)]
    A = scene.map
    rng = np.random.default_rng(3)
    lo, hi = A[:, :3].min(0), A[:, :3].max(0)
    extra = np.ones((grow_pts, 4), np.float32)
    extra[:, :3] = (lo + (hi - lo) * rng.random((grow_pts, 3))).astype(np.float32)
    grown = np.concatenate([A, extra])
    B = A[::2].copy()
    maps = [A] * n_same + [grown, grown, B, A]
    cases = [(a.guess, a.scan, mp) for a, mp in zip(al, maps)]
    path = tmp_path / "ndt_input.dat"
    pkg.datfile.write_input(path, cases)
    return path, cases


@pytest.mark.parametrize("n_same,scan_pts", [(6, None), (600, 300)])
def test_dat_align_equals_batches(pkg, tmp_path, n_same, scan_pts):
    cfg = pkg.synth.small_config("dat", 30000, 50.0, 20, scan_pts or 2000, seed=71)
    scene = pkg.synth.make_scene(cfg)
    path, cases = _write(pkg, tmp_path, cfg, scene, n_same)
    prm = pkg.ndt.reference_params(cfg.resolution)
    with pkg.ndt.DatFile(path) as f, pkg.ndt.Context(prm) as ctx, pkg.ndt.Context(prm) as ref:
        D = pkg.ndt.DatFile
        assert f.relation(n_same) == D.MAP_GROWN and f.relation(n_same + 2) == D.MAP_NEW
        out, conv, fit, status = f.align(ctx)
        # the same cases through the batch call, one batch per run of equal maps
        i = 0
        while i < len(cases):
            j = i + 1
            while j < len(cases) and cases[j][2] is cases[i][2]:
                j += 1
            ref.set_map(cases[i][2])
            o, c, ft, st = ref.align_batch([c_[1] for c_ in cases[i:j]], np.stack([c_[0] for c_ in cases[i:j]]))
            assert np.array_equal(out[i:j].view(np.uint32), o.view(np.uint32))
            assert np.array_equal(conv[i:j], c) and np.array_equal(status[i:j], st)
            assert np.array_equal(fit[i:j].view(np.uint64), ft.view(np.uint64))
            i = j
        # a sub-range starting inside a run of equal maps
        o2, c2, f2, s2 = f.align(ctx, first=3, count=5)
        assert np.array_equal(o2.view(np.uint32), out[3:8].view(np.uint32))


def test_dat_align_vs_fp64_oracle(pkg, oracle, binding_mod, tmp_path):
    """The file path against the FP64 oracle (the restated reference, pinned
    to it bit for bit) on every case of a small file with a shared, a grown
    and a new map: translation column bit-exact, converged equal, rotation
    within 0.05 deg, and the reference's own acceptance rule."""
    import math
    cfg = pkg.synth.small_config("dat_o", 20000, 40.0, 16, 1500, seed=72)
    scene = pkg.synth.make_scene(cfg)
    path, cases = _write(pkg, tmp_path, cfg, scene, 4, grow_pts=2000)
    prm = binding_mod.reference_params(cfg.resolution)
    with pkg.ndt.DatFile(path) as f, pkg.ndt.Context(pkg.ndt.reference_params(cfg.resolution)) as ctx:
        out, conv, _, status = f.align(ctx)
    assert (status == 0).all()
    for i, (g, s, m) in enumerate(cases):
        ref, rconv, _, _ = oracle.align(prm, s, g, m)
        T, R = out[i].reshape(4, 4), np.asarray(ref, np.float32).reshape(4, 4)
        assert np.array_equal(T[:, 3].view(np.uint32), R[:, 3].view(np.uint32)), i
        assert int(conv[i]) == int(rconv), i
        d = T[:3, :3].astype(np.float64) - R[:3, :3].astype(np.float64)
        assert math.degrees(2 * math.asin(min(1.0, float(np.linalg.norm(d)) / math.sqrt(8)))) <= 0.05, i
        ok, _ = pkg.datfile.reference_check(out[i], conv[i], R.reshape(16), rconv)
        assert ok, i
