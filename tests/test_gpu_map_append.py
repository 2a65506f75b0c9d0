"""Map growth (ndt_map_append / ndt_map_append_device): after appending
points to the map, the voxel grid and the alignments equal those of
ndt_set_map on the whole grown map, bit for bit, whether the update was
incremental (new points inside the old points' bounding box) or a rebuild
(new points outside it); the corrected grid is also checked against the FP64
oracle's grid of the grown map."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _params(pkg, compat, res=1.0):
    return pkg.ndt.reference_params(res) if compat else pkg.ndt.corrected_params(res)


def _grid(ctx):
    cell, count, mean, icov = ctx.grid_cells()
    order = np.argsort(cell, kind="stable")
    return cell[order], count[order], mean[order], icov[order], ctx.grid_info()


def _same_grid(a, b):
    for x, y in zip(a[:4], b[:4]):
        assert x.shape == y.shape
        assert np.array_equal(x.view(np.uint8), y.view(np.uint8))
    assert np.array_equal(a[4][0], b[4][0]) and np.array_equal(a[4][1], b[4][1]) and a[4][2] == b[4][2]


def _scene(pkg, seed):
    cfg = pkg.synth.small_config("ap", 30000, 50.0, 20, 3000, seed=seed)
    scene = pkg.synth.make_scene(cfg)
    return cfg, scene


def _batch(pkg, cfg, scene, n=16):
    al = [pkg.synth.make_alignment(cfg, scene, i) for i in range(n)]
    return [a.scan for a in al], np.stack([a.guess for a in al])


@pytest.mark.parametrize("compat", [1, 0])
def test_append_inside_equals_full_build(pkg, compat):
    cfg, scene = _scene(pkg, 61)
    mp = scene.map
    rng = np.random.default_rng(5)
    # grow by a scan's worth of points inside the old points' bounding box, in several appends
    lo, hi = mp[:, :3].min(0), mp[:, :3].max(0)
    extra = np.ones((9000, 4), np.float32)
    extra[:, :3] = (lo + (hi - lo) * rng.random((9000, 3))).astype(np.float32)
    extra[:, 2] = mp[rng.integers(0, len(mp), 9000), 2]  # on the surfaces' heights
    parts = [extra[:100], extra[100:4100], extra[4100:4101], extra[4101:]]
    prm = _params(pkg, compat)
    with pkg.ndt.Context(prm) as inc, pkg.ndt.Context(prm) as full:
        inc.set_map(mp)
        grown = mp
        for p in parts:
            inc.map_append(p)
            grown = np.concatenate([grown, p])
            full.set_map(grown)
            _same_grid(_grid(inc), _grid(full))
        scans, guesses = _batch(pkg, cfg, scene)
        a = inc.align_batch(scans, guesses)
        b = full.align_batch(scans, guesses)
        for x, y in zip(a, b):
            assert np.array_equal(np.asarray(x).view(np.uint8), np.asarray(y).view(np.uint8))


@pytest.mark.parametrize("compat", [1, 0])
def test_append_outside_rebuilds(pkg, compat):
    cfg, scene = _scene(pkg, 62)
    mp = scene.map
    far = mp[:2000].copy()
    far[:, 0] += 80.0  # beyond the old box: the grid layout changes
    prm = _params(pkg, compat)
    with pkg.ndt.Context(prm) as inc, pkg.ndt.Context(prm) as full:
        inc.set_map(mp)
        inc.map_append(far)
        full.set_map(np.concatenate([mp, far]))
        _same_grid(_grid(inc), _grid(full))


def test_append_device_after_set_map_device(pkg):
    torch = pytest.importorskip("torch")
    cfg, scene = _scene(pkg, 63)
    mp = scene.map
    k = 5000
    base, extra = mp[:-k], mp[-k:]  # the last points of the map lie inside the first ones' box
    d_base = torch.from_numpy(np.ascontiguousarray(base)).cuda()
    d_extra = torch.from_numpy(np.ascontiguousarray(extra)).cuda()
    torch.cuda.synchronize()
    prm = _params(pkg, 1)
    with pkg.ndt.Context(prm) as inc, pkg.ndt.Context(prm) as full:
        inc.set_map_device(d_base.data_ptr(), len(base))
        inc.map_append_device(d_extra.data_ptr(), k)
        inc.map_append_device(d_extra.data_ptr(), 0)  # nothing to add
        full.set_map(mp)
        _same_grid(_grid(inc), _grid(full))


def test_append_corrected_vs_oracle(pkg, oracle, binding_mod):
    cfg, scene = _scene(pkg, 64)
    mp = scene.map
    half = len(mp) // 2
    with pkg.ndt.Context(_params(pkg, 0)) as inc:
        inc.set_map(mp[:half])
        inc.map_append(mp[half:])
        cell, count, mean, icov, (bbox, dims, _) = _grid(inc)
    obox, odims, ocells = oracle.grid(binding_mod.corrected_params(1.0), mp)
    assert np.array_equal(bbox.view(np.uint32), obox.view(np.uint32))
    assert np.array_equal(dims, odims)
    keep = ocells[cell, 12] > 0
    cell, count, mean, icov = cell[keep], count[keep], mean[keep], icov[keep]
    ref = ocells[cell]
    assert np.array_equal(count, np.abs(ref[:, 12]).astype(np.int32))
    assert np.array_equal(mean.view(np.uint64), ref[:, 0:3].copy().view(np.uint64))
    assert np.array_equal(icov.view(np.uint64), ref[:, 3:12].copy().view(np.uint64))


def test_append_errors(pkg):
    cfg, scene = _scene(pkg, 65)
    with pkg.ndt.Context(_params(pkg, 1)) as ctx:
        with pytest.raises(pkg.ndt.NdtError, match="NOMAP"):
            ctx.map_append(scene.map[:10])
        ctx.set_map(scene.map)
        before = _grid(ctx)
        bad = scene.map[:10].copy()
        bad[3, 1] = np.nan
        with pytest.raises(pkg.ndt.NdtError, match="ARG"):
            ctx.map_append(bad)
        _same_grid(_grid(ctx), before)  # the failed append left the map as it was
        ctx.map_append(scene.map[:10])
