"""The batched scan pre-filter on the GPU (csrc/voxel_filter.cu through the C
ABI) against the CPU reference (oracle/voxel_filter_ref.py): bit-exact output
points and offsets, edge cases, capacity errors, and the size-independent
properties (idempotence, leaf order) at a full scan batch."""
import numpy as np
import pytest

import voxel_filter_ref as V

pytestmark = pytest.mark.gpu


def _scan(rng, n, spread=30.0, nonfinite=0):
    s = np.ones((n, 4), np.float32)
    s[:, :3] = rng.uniform(-spread, spread, (n, 3)).astype(np.float32)
    s[:, 2] *= 0.1
    s[:, 3] = rng.uniform(0, 255, n).astype(np.float32)
    if nonfinite:
        idx = rng.choice(n, nonfinite, replace=False)
        s[idx, rng.integers(0, 3, nonfinite)] = rng.choice([np.nan, np.inf, -np.inf], nonfinite)
    return s


def _pack(scans):
    offs = np.zeros(len(scans) + 1, np.int64)
    offs[1:] = np.cumsum([len(s) for s in scans])
    pts = np.concatenate(scans) if offs[-1] else np.zeros((0, 4), np.float32)
    return pts, offs


@pytest.fixture(scope="module")
def vf(pkg):
    f = pkg.voxel_filter.VoxelFilter(0)
    yield f
    f.close()


def _check(vf, scans, leaf):
    pts, offs = _pack(scans)
    out, oo = vf.filter(pts, offs, leaf)
    ref, roo = V.filter_batch(pts, offs, leaf)
    assert oo.tolist() == roo.tolist()
    assert out.shape == ref.shape
    assert np.array_equal(out.view(np.uint32), ref.view(np.uint32))
    return out, oo


@pytest.mark.parametrize("leaf", [2.0, 0.5, 1.7])
@pytest.mark.parametrize("seed", [0, 1, 2])
def test_batch_parity(vf, seed, leaf):
    rng = np.random.default_rng(seed)
    sizes = rng.integers(0, 4000, 12)
    sizes[3] = 0
    scans = [_scan(rng, int(n), float(rng.uniform(2, 60)), nonfinite=int(n) // 50) for n in sizes]
    _check(vf, scans, leaf)


def test_edge_cases(vf):
    nan = np.full((3, 4), np.nan, np.float32)
    one = np.array([[1.0, 2.0, 3.0, 4.0]] * 5, np.float32)
    two = np.array([[-0.5, 0, 0, 1], [0.5, 0, 0, 1]], np.float32)
    _check(vf, [one], 2.0)
    _check(vf, [one, nan, np.zeros((0, 4), np.float32), two], 2.0)
    _check(vf, [nan], 2.0)
    _check(vf, [np.zeros((0, 4), np.float32)] * 3, 2.0)
    # one leaf holding every point of a large scan (one long sequential sum)
    rng = np.random.default_rng(5)
    dense = _scan(rng, 50000, 0.9)
    dense[:, :3] = np.abs(dense[:, :3])
    _check(vf, [dense], 2.0)
    # coordinates far out (clamped leaf indices) in a scan of one point per axis extreme
    far = np.array([[3e38, 0, 0, 1]], np.float32)
    _check(vf, [far], 0.25)


def test_capacity_errors(pkg, vf):
    far = np.array([[-1e9, 0, 0, 1], [1e9, 0, 0, 1], [0, -1e9, 0, 1], [0, 1e9, 0, 1]], np.float32)
    with pytest.raises(pkg.ndt.NdtError, match="CAPACITY"):
        vf.filter(far, [0, 4], 0.5)
    a = np.array([[0, 0, 0, 1], [1e6 - 1, 0, 0, 1], [0, 999, 0, 1]], np.float32)
    with pytest.raises(pkg.ndt.NdtError, match="CAPACITY"):
        vf.filter(np.concatenate([a, a, a]), [0, 3, 6, 9], 1.0)
    _check(vf, [a], 1.0)  # the handle stays usable


def test_full_batch_properties(pkg, vf):
    """512 scans of 30k raw points: a sample of scans bit-exact
    against the reference, idempotence on the whole output."""
    rng = np.random.default_rng(11)
    B, n = 512, 30000
    pts = np.ones((B * n, 4), np.float32)
    pts[:, :3] = rng.normal(0, 20, (B * n, 3)).astype(np.float32)
    pts[:, 2] *= 0.05
    offs = np.arange(B + 1, dtype=np.int64) * n
    out, oo = vf.filter(pts, offs, 2.0)
    for b in (0, 17, B - 1):
        ref = V.filter_scan(pts[offs[b]:offs[b + 1]], 2.0)
        assert np.array_equal(out[oo[b]:oo[b + 1]].view(np.uint32), ref.view(np.uint32))
    again, oo2 = vf.filter(out, oo, 2.0)
    assert oo2.tolist() == oo.tolist()
    assert np.array_equal(again.view(np.uint32), out.view(np.uint32))
