"""Euclidean clustering on the GPU (csrc/ec.cu through the C ABI) against the
reference kernel's own results on its own data (tests/golden/ec_cases.npz,
made by tests/golden/make_ec_fixtures.py): extract()'s clusters per distance
ring identical (sizes, point indices, order); segmentByDistance's boxes and
centroids identical bit for bit (the box yaw against the reference's pose
estimate taken with the hull's own length) and the
reference's acceptance rule met; labels against brute force on small clouds."""
import pathlib

import numpy as np
import pytest

import ec_ref

pytestmark = pytest.mark.gpu

GOLDEN = pathlib.Path(__file__).resolve().parent / "golden" / "ec_cases.npz"
RING_TOL = (0.5, 1.1, 1.6, 2.3, float(np.float32(2.6)))


def _rings(xyz):
    x, y = xyz[:, 0], xyz[:, 1]
    d = np.sqrt(x * x + y * y)
    r = np.where(d < 15, 0, np.where(d < 30, 1, np.where(d < 45, 2, np.where(d < 60, 3, 4))))
    return [xyz[r == k] for k in range(5)]


@pytest.fixture(scope="module")
def ecg(pkg):
    h = pkg.ec.EuclideanClusters(0)
    yield h
    h.close()


@pytest.fixture(scope="module")
def gold():
    return np.load(GOLDEN)


def test_extract_equals_reference(ecg, gold):
    for i in range(int(gold["cases"])):
        for k, cloud in enumerate(_rings(gold[f"in{i}"])):
            sizes = gold[f"sizes{i}_{k}"]
            idx = gold[f"idx{i}_{k}"].astype(np.int64)
            ref = np.split(idx, np.cumsum(sizes)[:-1]) if len(sizes) else []
            ours = ecg.extract(cloud, RING_TOL[k])
            assert [len(c) for c in ours] == list(sizes), (i, k)
            for a, b in zip(ours, ref):
                assert np.array_equal(a, b), (i, k)


def test_segment_equals_reference(ecg, gold):
    for i in range(int(gold["cases"])):
        pts, boxes, cen = ecg.segment(gold[f"in{i}"])
        rb, rc = gold[f"boxes{i}"], gold[f"centroids{i}"]
        assert len(pts) == int(gold[f"npts{i}"])
        assert len(boxes) == len(rb) and len(cen) == len(rc)
        # same boxes (position, dimensions) and centroids, bit for bit, in the same order
        assert np.array_equal(boxes[:, [0, 1, 2, 7, 8, 9]].view(np.uint64), rb[:, [0, 1, 2, 7, 8, 9]].copy().view(np.uint64))
        # orientation: (0, 0, z, w) with the pose estimate's yaw (taken with the hull's own length)
        assert np.all(boxes[:, 3:5] == 0.0)
        assert np.array_equal(boxes[:, 5:7].copy().view(np.uint64), gold[f"yaw{i}"].view(np.uint64))
        assert np.array_equal(cen.view(np.uint64), rc.view(np.uint64))
        # the clustered points: ring by ring, cluster by cluster, as the reference appends them
        ref_pts = np.concatenate([ring[gold[f"idx{i}_{k}"].astype(np.int64)]
                                  for k, ring in enumerate(_rings(gold[f"in{i}"]))])
        assert np.array_equal(pts.view(np.uint32), ref_pts.view(np.uint32))
        ok, d = ec_ref.check(pts, ec_ref.boxes10_to_8(boxes), cen, ref_pts, ec_ref.boxes10_to_8(rb), rc)
        assert ok and d == 0.0, d


def test_segment_batch_equals_single(ecg, gold):
    clouds = [gold[f"in{i}"] for i in range(int(gold["cases"]))]
    clouds = clouds + clouds[:4]  # 9 clouds: two passes of up to 8
    batch = ecg.segment_batch(clouds)
    for c, (pts, boxes, cen) in zip(clouds, batch):
        p1, b1, c1 = ecg.segment(c)
        assert np.array_equal(pts.view(np.uint32), p1.view(np.uint32))
        assert np.array_equal(boxes.view(np.uint64), b1.view(np.uint64))
        assert np.array_equal(cen.view(np.uint64), c1.view(np.uint64))


@pytest.mark.parametrize("tol", [0.3, 0.5, 1.0])
def test_labels_vs_brute_force(ecg, tol):
    rng = np.random.default_rng(int(tol * 10))
    xyz = np.concatenate([rng.normal(c, 0.35, (80, 3)) for c in rng.uniform(-6, 6, (15, 3))]).astype(np.float32)
    assert np.array_equal(ecg.labels(xyz, tol), ec_ref.brute_labels(xyz, tol))


def test_edge_cases(pkg, ecg):
    # points exactly one radius apart (accepted: <=), a chain that joins only through its links
    chain = np.zeros((50, 3), np.float32)
    chain[:, 0] = np.arange(50, dtype=np.float32) * 0.5
    assert np.all(ecg.labels(chain, 0.5) == 0)
    assert np.array_equal(ecg.labels(chain, 0.4999), np.arange(50))
    assert len(ecg.labels(np.zeros((0, 3), np.float32), 0.5)) == 0
    same = np.ones((30, 3), np.float32)
    assert [len(c) for c in ecg.extract(same, 0.5)] == [30]
    assert ecg.extract(same[:5], 0.5) == []  # below the minimum size
    bad = chain.copy()
    bad[7, 2] = np.inf
    with pytest.raises(pkg.ndt.NdtError, match="ARG"):
        ecg.labels(bad, 0.5)
