"""Euclidean-clustering checkers (test infrastructure only).

* readers of the reference's data files (src/CPU/euclidean_cluster/kernel.cpp:
  816-904): ec_input.dat = int32 T, then per case int32 n + n x float32[3];
  ec_output.dat = per case int32 n + n x (float32[3] + uint8[3]) clustered
  points, int32 nb + nb x float64[8] boxes (position x, y, orientation x, y,
  z, w, dimensions x, y), int32 nc + nc x float64[3] centroids;
* the reference's acceptance rule (check_next_outputs, :1034-1093): both
  sides sorted, equal sizes, max |difference| of points (x, y, z), boxes
  (position x, y, dimensions x, y, orientation x, y) and centroids <= 0.001;
* brute-force labels (smallest index of each point's component) with the
  reference's float distance test, for small clouds;
* a ctypes binding of the UNMODIFIED reference kernel compiled by
  oracle/Makefile (oracle/_ref/libref_ec.so).
"""
from __future__ import annotations

import ctypes as C
import gzip
import pathlib
import struct

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
REF_LIB = HERE / "_ref" / "libref_ec.so"
MAX_EPS = 0.001


def _open(path):
    path = str(path)
    return gzip.open(path, "rb") if path.endswith(".gz") else open(path, "rb")


def read_input(path):
    with _open(path) as f:
        d = f.read()
    (T,) = struct.unpack_from("<i", d, 0)
    off, out = 4, []
    for _ in range(T):
        (n,) = struct.unpack_from("<i", d, off)
        off += 4
        out.append(np.frombuffer(d, "<f4", 3 * n, off).reshape(n, 3).copy())
        off += 12 * n
    return out


def read_output(path, T):
    with _open(path) as f:
        d = f.read()
    off, out = 0, []
    pt = np.dtype([("xyz", "<f4", (3,)), ("rgb", "u1", (3,))])
    for _ in range(T):
        (n,) = struct.unpack_from("<i", d, off)
        off += 4
        pts = np.frombuffer(d, pt, n, off).copy()
        off += 15 * n
        (nb,) = struct.unpack_from("<i", d, off)
        off += 4
        boxes = np.frombuffer(d, "<f8", 8 * nb, off).reshape(nb, 8).copy()
        off += 64 * nb
        (nc,) = struct.unpack_from("<i", d, off)
        off += 4
        cen = np.frombuffer(d, "<f8", 3 * nc, off).reshape(nc, 3).copy()
        off += 24 * nc
        out.append((pts["xyz"], pts["rgb"], boxes, cen))
    return out


def _lexsort(a, cols):
    return a[np.lexsort(tuple(a[:, c] for c in reversed(cols)))]


def check(points, boxes8, centroids, ref_points, ref_boxes8, ref_centroids):
    """The reference's rule.  boxes8 rows: position x, y, orientation x, y, z,
    w, dimensions x, y (the output file's layout).  Returns (ok, max_delta)."""
    if len(points) != len(ref_points) or len(boxes8) != len(ref_boxes8) or len(centroids) != len(ref_centroids):
        return False, float("inf")
    d = 0.0
    if len(points):
        a, b = _lexsort(np.asarray(points, np.float32), [0, 1, 2]), _lexsort(np.asarray(ref_points, np.float32),
                                                                             [0, 1, 2])
        d = max(d, float(np.abs(a - b).max()))
    if len(boxes8):
        key = [0, 1, 6, 7]
        a, b = _lexsort(np.asarray(boxes8), key), _lexsort(np.asarray(ref_boxes8), key)
        d = max(d, float(np.abs(a[:, [0, 1, 6, 7, 2, 3]] - b[:, [0, 1, 6, 7, 2, 3]]).max()))
    if len(centroids):
        a, b = _lexsort(np.asarray(centroids), [0, 1, 2]), _lexsort(np.asarray(ref_centroids), [0, 1, 2])
        d = max(d, float(np.abs(a - b).max()))
    return d <= MAX_EPS, d


def boxes10_to_8(b10):
    """(position xyz, orientation xyzw, dimensions xyz) -> the file's 8 columns."""
    b10 = np.asarray(b10).reshape(-1, 10)
    return b10[:, [0, 1, 3, 4, 5, 6, 7, 8]]


def brute_labels(xyz, tol):
    """Smallest index of each point's component (float distance test as the reference)."""
    p = np.asarray(xyz, np.float32)
    n = len(p)
    r2 = np.float32(tol) * np.float32(tol)
    parent = np.arange(n)

    def find(x):
        while parent[x] != x:
            parent[x] = parent[parent[x]]
            x = parent[x]
        return x

    for i in range(n):
        d = p[i + 1:] - p[i]
        s = (d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2]
        for j in np.nonzero(s <= r2)[0] + i + 1:
            a, b = find(i), find(int(j))
            if a != b:
                parent[max(a, b)] = min(a, b)
    return np.array([find(i) for i in range(n)])


class Reference:
    def __init__(self):
        if not REF_LIB.exists():
            raise FileNotFoundError(REF_LIB)
        L = C.CDLL(str(REF_LIB))
        L.ref_ec_extract.argtypes = [C.c_void_p, C.c_int, C.c_double, C.c_void_p, C.c_void_p, C.c_int]
        L.ref_ec_segment.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p,
                                     C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)]
        self.L = L

    @staticmethod
    def available():
        return REF_LIB.exists()

    def extract(self, xyz, tol):
        p = np.ascontiguousarray(xyz, np.float32)
        n = len(p)
        sizes = np.zeros(max(n, 1), np.int32)
        idx = np.zeros(max(n, 1), np.int32)
        k = self.L.ref_ec_extract(p.ctypes.data, n, float(tol), sizes.ctypes.data, idx.ctypes.data, n)
        off = np.concatenate([[0], np.cumsum(sizes[:k])])
        return [idx[off[c]:off[c + 1]].copy() for c in range(k)]

    def segment(self, xyz):
        p = np.ascontiguousarray(xyz, np.float32)
        n = len(p)
        pts = np.zeros((max(n, 1), 3), np.float32)
        boxes = np.zeros((max(n, 1), 10))
        cen = np.zeros((max(n, 1), 3))
        nb, nc = C.c_int(), C.c_int()
        k = self.L.ref_ec_segment(p.ctypes.data, n, pts.ctypes.data, n, boxes.ctypes.data, n, cen.ctypes.data, n,
                                  C.byref(nb), C.byref(nc))
        return pts[:k], boxes[:nb.value], cen[:nc.value]

    def box_yaw(self, xyz):
        """clusterAndColor's pose estimate for one cluster (kernel.cpp:720-745) through the reference's
        convexHull and rotatingCalipers, given the hull's own length (minAreaRectAngle hands them the
        cluster's point count and reads past the hull).  Returns (angle_deg, qz, qw)."""
        p = np.ascontiguousarray(xyz, np.float32)
        qz, qw = C.c_double(), C.c_double()
        self.L.ref_ec_box_yaw.restype = C.c_float
        self.L.ref_ec_box_yaw.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double)]
        a = self.L.ref_ec_box_yaw(p.ctypes.data, len(p), C.byref(qz), C.byref(qw))
        return float(a), qz.value, qw.value

    def convex_hull(self, xy):
        """The reference's convexHull (kernel.cpp:376-470), clockwise, as points."""
        p = np.ascontiguousarray(xy, np.float32)
        out = np.zeros((max(len(p), 1), 2), np.float32)
        self.L.ref_ec_convex_hull.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
        k = self.L.ref_ec_convex_hull(p.ctypes.data, len(p), out.ctypes.data)
        return out[:k]
