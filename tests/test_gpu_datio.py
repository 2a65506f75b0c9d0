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
