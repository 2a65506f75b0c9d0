"""CPU reference of the scan pre-filter (test infrastructure only).

The voxel-grid downsampling that produces the align call's "filtered scan"
inputs upstream (Autoware's mapping node runs the point-cloud library's
VoxelGrid filter, PCL 1.x `pcl::VoxelGrid<PointXYZI>::applyFilter`, with a
2 m leaf; the reference ships only its outputs, as `.dat` files, and has no
call site of the filter).  Restated here from that published algorithm:

  * points with a non-finite x, y or z are dropped;
  * r = 1 / leaf rounded to float; the leaf of a point is
    (floor(x * r), floor(y * r), floor(z * r)), each product rounded to
    float (PCL's `floor(p.x * inverse_leaf_size_[0])`), clamped to +-2^60;
  * one output point per occupied leaf: the mean of its points.  PCL sums in
    float in the order of an unstable sort; here every component is summed in
    float64 in input order and the mean is rounded to float once, which is
    deterministic and within float rounding of PCL's centroid;
  * output ordered by leaf, x fastest, then y, then z (PCL's
    idx = i + j * div_b[0] + k * div_b[0] * div_b[1] order);
  * PCL returns the input unchanged when a scan spans more than INT_MAX
    leaves; the library reports a capacity error instead (`CapacityError`
    here).
"""
from __future__ import annotations

import numpy as np

CLAMP = np.float32(2.0 ** 60)


class CapacityError(ValueError):
    pass


def leaf_indices(points, leaf):
    p = np.asarray(points, np.float32)
    r = np.float32(1.0) / np.float32(leaf)
    with np.errstate(over="ignore"):  # a product beyond float range is +-inf, then clamped
        q = np.floor(p[:, :3] * r).astype(np.float32)
    q = np.clip(q, -CLAMP, CLAMP)
    return q.astype(np.int64)


def _filter(points, leaf):
    """(filtered points, leaf span of the scan's bounding box)."""
    p = np.asarray(points, np.float32).reshape(-1, 4)
    keep = np.isfinite(p[:, :3]).all(axis=1)
    p = p[keep]
    if len(p) == 0:
        return np.zeros((0, 4), np.float32), 0
    q = leaf_indices(p, leaf)
    lo = q.min(axis=0)
    d = q.max(axis=0) - lo + 1
    span = int(d[0]) * int(d[1]) * int(d[2])
    if span >= 2 ** 31:
        raise CapacityError("a scan spans 2^31 leaves or more")
    key = (q[:, 0] - lo[0]) + d[0] * ((q[:, 1] - lo[1]) + d[1] * (q[:, 2] - lo[2]))
    uniq, inv = np.unique(key, return_inverse=True)
    sums = np.zeros((len(uniq), 4), np.float64)
    np.add.at(sums, inv, p.astype(np.float64))  # unbuffered: in input order per leaf
    cnt = np.bincount(inv, minlength=len(uniq)).astype(np.float64)
    return (sums / cnt[:, None]).astype(np.float32), span


def filter_scan(points, leaf):
    """One scan (n x 4 float32) -> its filtered points (k x 4 float32)."""
    return _filter(points, leaf)[0]


def filter_batch(points, offsets, leaf):
    """Packed batch (points: total x 4, offsets: B + 1) -> (out, out_offsets)."""
    points = np.asarray(points, np.float32).reshape(-1, 4)
    offsets = np.asarray(offsets, np.int64)
    res = [_filter(points[offsets[b]:offsets[b + 1]], leaf) for b in range(len(offsets) - 1)]
    if sum(s for _, s in res) >= 2 ** 31 - 1:
        raise CapacityError("the batch spans 2^31 - 1 leaves or more")
    outs = [o for o, _ in res]
    oo = np.zeros(len(outs) + 1, np.int64)
    oo[1:] = np.cumsum([len(o) for o in outs])
    out = np.concatenate(outs) if outs else np.zeros((0, 4), np.float32)
    return out.reshape(-1, 4), oo


def filter_scan_loops(points, leaf):
    """Pure-Python restatement for small cases (checks filter_scan itself)."""
    f32 = np.float32
    r = f32(1.0) / f32(leaf)
    cells = {}
    for pt in np.asarray(points, np.float32).reshape(-1, 4):
        if not all(np.isfinite(pt[:3])):
            continue
        k = tuple(int(min(max(np.floor(f32(pt[a] * r)), -CLAMP), CLAMP)) for a in range(3))
        cells.setdefault(k, []).append(pt)
    out = []
    for k in sorted(cells, key=lambda k: (k[2], k[1], k[0])):
        s = [0.0, 0.0, 0.0, 0.0]
        for pt in cells[k]:
            for a in range(4):
                s[a] += float(pt[a])
        out.append([f32(v / len(cells[k])) for v in s])
    return np.array(out, np.float32).reshape(-1, 4)
