"""The scan pre-filter's CPU reference (oracle/voxel_filter_ref.py): the
vectorised form against the pure-Python restatement, and the properties the
filter has by construction (idempotence, order, capacity errors)."""
import numpy as np
import pytest

import voxel_filter_ref as V


def _scan(rng, n, spread=30.0, nonfinite=0):
    s = np.ones((n, 4), np.float32)
    s[:, :3] = rng.uniform(-spread, spread, (n, 3)).astype(np.float32)
    s[:, 2] *= 0.1
    s[:, 3] = rng.uniform(0, 255, n).astype(np.float32)
    if nonfinite:
        idx = rng.choice(n, nonfinite, replace=False)
        s[idx, rng.integers(0, 3, nonfinite)] = rng.choice([np.nan, np.inf, -np.inf], nonfinite)
    return s


@pytest.mark.parametrize("leaf", [2.0, 0.5, 1.7, 0.3])
@pytest.mark.parametrize("seed", [0, 1])
def test_vectorised_matches_loops(seed, leaf):
    rng = np.random.default_rng(seed)
    s = _scan(rng, 700, 8.0, nonfinite=9)
    a = V.filter_scan(s, leaf)
    b = V.filter_scan_loops(s, leaf)
    assert a.shape == b.shape and a.view(np.uint32).tolist() == b.view(np.uint32).tolist()


def test_idempotent_and_ordered():
    rng = np.random.default_rng(3)
    s = _scan(rng, 5000, 20.0)
    f = V.filter_scan(s, 2.0)
    assert np.array_equal(V.filter_scan(f, 2.0).view(np.uint32), f.view(np.uint32))
    q = V.leaf_indices(f, 2.0)
    key = [(k[2], k[1], k[0]) for k in q.tolist()]
    assert key == sorted(key) and len(set(key)) == len(key)


def test_edge_cases():
    empty = np.zeros((0, 4), np.float32)
    assert V.filter_scan(empty, 2.0).shape == (0, 4)
    nan = np.full((3, 4), np.nan, np.float32)
    assert V.filter_scan(nan, 2.0).shape == (0, 4)
    one = np.array([[1.0, 2.0, 3.0, 4.0]] * 5, np.float32)
    assert np.array_equal(V.filter_scan(one, 2.0), one[:1])
    # negative coordinates round toward -inf: -0.5 and 0.5 are in different leaves
    two = np.array([[-0.5, 0, 0, 1], [0.5, 0, 0, 1]], np.float32)
    assert len(V.filter_scan(two, 2.0)) == 2
    # batch with empty and all-dropped scans keeps their (empty) slots
    pts = np.concatenate([one, nan, two])
    out, oo = V.filter_batch(pts, [0, 5, 5, 8, 10], 2.0)
    assert oo.tolist() == [0, 1, 1, 1, 3]


def test_capacity_errors():
    far = np.array([[-1e9, 0, 0, 1], [1e9, 0, 0, 1], [0, -1e9, 0, 1], [0, 1e9, 0, 1]], np.float32)
    with pytest.raises(V.CapacityError):
        V.filter_scan(far, 0.5)
    # each scan fits, the batch's leaf ranges together do not
    a = np.array([[0, 0, 0, 1], [1e6 - 1, 0, 0, 1], [0, 999, 0, 1]], np.float32)
    pts = np.concatenate([a, a, a])
    with pytest.raises(V.CapacityError):
        V.filter_batch(pts, [0, 3, 6, 9], 1.0)
    V.filter_batch(pts[:3], [0, 3], 1.0)
