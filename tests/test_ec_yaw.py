"""Box yaw of the euclidean_cluster boxes (csrc/ec_pose.cpp, host code:
ndt_ec_box_yaw) against the reference's pose estimate (kernel.cpp:720-745)
computed by the reference's own convexHull and rotatingCalipers with the
hull's own length (oracle/ec_shim.cpp ref_ec_box_yaw; the reference's
minAreaRectAngle reads past the end of the hull).  Bit for bit on every kept
box of the reference's five clouds (tests/golden/ec_cases.npz) and on
synthetic families in general position and with exact ties; on point sets
collinear to within float rounding the reference's scan order can keep other
nearly collinear hull vertices, and the quaternion then differs by <= 5e-5."""
import math
import zlib
import pathlib

import numpy as np
import pytest

import ec_ref

GOLDEN = pathlib.Path(__file__).resolve().parent / "golden" / "ec_cases.npz"
RING_TOL = (0.5, 1.1, 1.6, 2.3, float(np.float32(2.6)))
needs_ref = pytest.mark.skipif(not ec_ref.Reference.available(), reason="compiled reference (oracle/_ref) not built here")


def _rings(xyz):
    x, y = xyz[:, 0], xyz[:, 1]
    d = np.sqrt(x * x + y * y)
    r = np.where(d < 15, 0, np.where(d < 30, 1, np.where(d < 45, 2, np.where(d < 60, 3, 4))))
    return [xyz[r == k] for k in range(5)]


def _kept(p):
    lo, hi = p.min(0), p.max(0)
    d = hi - lo
    return d[0] > 0 and d[1] > 0 and d[2] > 0 and d[0] < 15 and d[1] < 15 and hi[2] > -1.5 and lo[2] > -1.5 and lo[2] < 1.0


def test_golden_boxes_bit_exact(pkg):
    gold = np.load(GOLDEN)
    for i in range(int(gold["cases"])):
        got = []
        for k, ring in enumerate(_rings(gold[f"in{i}"])):
            sizes, idx = gold[f"sizes{i}_{k}"], gold[f"idx{i}_{k}"].astype(np.int64)
            for c in (np.split(idx, np.cumsum(sizes)[:-1]) if len(sizes) else []):
                if _kept(ring[c]):
                    got.append(pkg.ec.box_yaw(ring[c]))
        assert np.array_equal(np.array(got).view(np.uint64), gold[f"yaw{i}"].view(np.uint64)), i


def _family(rng, kind, n):
    if kind == "blob":
        return rng.normal(0, 0.4, (n, 3)) + np.r_[rng.uniform(-70, 70, 2), 0]
    if kind == "rotated_rectangle":
        a = rng.uniform(0, np.pi)
        u = rng.uniform(-1, 1, (n, 2)) * rng.uniform(0.3, 7, 2)
        R = np.array([[np.cos(a), -np.sin(a)], [np.sin(a), np.cos(a)]])
        return np.c_[u @ R.T + rng.uniform(-60, 60, 2), rng.normal(0, 0.5, n)]
    if kind == "grid":  # exact ties between rectangles and between calipers
        k = int(rng.integers(2, 8))
        g = np.stack(np.meshgrid(np.arange(k), np.arange(k)), -1).reshape(-1, 2) * rng.uniform(0.1, 1)
        return np.c_[g + rng.uniform(-60, 60, 2), np.zeros(len(g))]
    if kind == "quantized":
        return np.round(rng.uniform(-5, 5, (n, 3)) * 2) / 2
    if kind == "polygon":
        m = int(rng.integers(3, 40))
        th = np.arange(m) * 2 * np.pi / m + rng.uniform(0, 1)
        return np.c_[np.cos(th), np.sin(th), np.zeros(m)] * rng.uniform(0.5, 10) + np.r_[rng.uniform(-60, 60, 2), 0]
    if kind == "duplicates":
        return np.repeat(rng.normal(0, 1, (max(n // 5, 1), 3)), 5, axis=0)
    if kind == "tiny":
        return rng.normal(0, 1, (int(rng.integers(1, 4)), 3))
    if kind == "line":  # collinear up to float rounding
        a = rng.uniform(0, np.pi)
        s = rng.uniform(-20, 20, n)
        return np.c_[s * np.cos(a), s * np.sin(a), np.zeros(n)] + np.r_[rng.uniform(-60, 60, 2), 0]
    raise ValueError(kind)


@needs_ref
@pytest.mark.parametrize("kind", ["blob", "rotated_rectangle", "grid", "quantized", "polygon", "duplicates", "tiny"])
def test_families_bit_exact(pkg, kind):
    ref = ec_ref.Reference()
    rng = np.random.default_rng(zlib.crc32(kind.encode()))
    for _ in range(400):
        p = _family(rng, kind, int(rng.integers(3, 200))).astype(np.float32)
        _, qz, qw = ref.box_yaw(p)
        assert pkg.ec.box_yaw(p) == (qz, qw)


@needs_ref
def test_near_collinear_within_bound(pkg):
    ref = ec_ref.Reference()
    rng = np.random.default_rng(5)
    exact = 0
    for _ in range(1000):
        p = _family(rng, "line", int(rng.integers(3, 200))).astype(np.float32)
        _, qz, qw = ref.box_yaw(p)
        oz, ow = pkg.ec.box_yaw(p)
        assert abs(oz - qz) <= 5e-5 and abs(ow - qw) <= 5e-5
        exact += (oz, ow) == (qz, qw)
    assert exact >= 950  # most such sets still match bit for bit


def test_edge_cases(pkg):
    assert pkg.ec.box_yaw(np.zeros((0, 3), np.float32)) == (0.0, 1.0)
    assert pkg.ec.box_yaw(np.ones((1, 3), np.float32)) == (0.0, 1.0)
    assert pkg.ec.box_yaw(np.ones((7, 3), np.float32)) == (0.0, 1.0)  # one distinct point
    # two distinct points: the direction of the segment between them, from the leftmost
    qz, qw = pkg.ec.box_yaw(np.array([[3, 1, 0], [1, 0, 0], [3, 1, 0]], np.float32))
    assert math.isclose(2 * math.atan2(qz, qw), math.atan2(1, 2), abs_tol=1e-6)
    # an axis-aligned box: yaw 0 or a quarter turn
    g = np.array([[x, y, 0] for x in range(4) for y in range(3)], np.float32)
    ang = math.degrees(2 * math.atan2(*pkg.ec.box_yaw(g)))
    assert min(abs(ang - a) for a in (-180, -90, 0, 90, 180)) < 1e-4
    bad = g.copy()
    bad[3, 1] = np.nan
    with pytest.raises(pkg.ndt.NdtError, match="ARG"):
        pkg.ec.box_yaw(bad)


def _golden_clusters():
    gold = np.load(GOLDEN)
    out = []
    for i in range(int(gold["cases"])):
        for k, ring in enumerate(_rings(gold[f"in{i}"])):
            sizes, idx = gold[f"sizes{i}_{k}"], gold[f"idx{i}_{k}"].astype(np.int64)
            out += [ring[c] for c in (np.split(idx, np.cumsum(sizes)[:-1]) if len(sizes) else [])]
    return out


def test_batch_equals_single(pkg):
    clusters = _golden_clusters()
    batch = pkg.ec.box_yaws(clusters)
    single = np.array([pkg.ec.box_yaw(c) for c in clusters])
    assert np.array_equal(batch.view(np.uint64), single.view(np.uint64))
    assert pkg.ec.box_yaws([]).shape == (0, 2)


def _child_yaws(pkg, clusters, conn):
    conn.send(pkg.ec.box_yaws(clusters))
    conn.close()


@pytest.mark.filterwarnings("ignore:This process .* is multi-threaded, use of fork:DeprecationWarning")
def test_batch_in_forked_process(pkg):
    """A process forked after a parallel pass (whose thread pool it does not inherit) still completes."""
    import multiprocessing as mp

    clusters = _golden_clusters()
    parent = pkg.ec.box_yaws(clusters)  # the parallel pass that starts the pool
    ctx = mp.get_context("fork")
    rd, wr = ctx.Pipe(duplex=False)
    child = ctx.Process(target=_child_yaws, args=(pkg, clusters, wr))
    child.start()
    got = rd.recv() if rd.poll(120) else None
    child.join(30)
    if child.is_alive():
        child.kill()
        child.join()
    assert got is not None, "forked process did not finish"
    assert np.array_equal(got.view(np.uint64), parent.view(np.uint64))
