"""Euclidean clustering: Python side of csrc/ec.cu (include/ndt_b200.h
`ndt_ec_*`), DAPHNE's euclidean_cluster kernel with the radius search and
cluster extraction on the GPU.  Host numpy arrays in and out."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import ndt as _ndt


def _lib():
    L = _ndt.lib()
    if not getattr(L, "_ec_ready", False):
        p = C.c_void_p
        L.ndt_ec_create.argtypes = [C.c_int, C.POINTER(p)]
        L.ndt_ec_destroy.argtypes = [p]
        L.ndt_ec_destroy.restype = None
        L.ndt_ec_last_error.argtypes = [p]
        L.ndt_ec_last_error.restype = C.c_char_p
        L.ndt_ec_labels.argtypes = [p, p, C.c_int, C.c_float, p]
        L.ndt_ec_extract.argtypes = [p, p, C.c_int, C.c_float, C.c_int, C.c_int, C.POINTER(C.c_int), p, p]
        L.ndt_ec_segment.argtypes = [p, p, C.c_int, p, C.POINTER(C.c_int), p, C.POINTER(C.c_int), p,
                                     C.POINTER(C.c_int)]
        L.ndt_ec_segment_batch.argtypes = [p, C.c_int, p, p, p, p, p, p, p]
        L.ndt_ec_box_yaw.argtypes = [p, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.ndt_ec_box_yaws.argtypes = [C.c_int, p, p, p, p]
        for n in ("ndt_ec_create", "ndt_ec_labels", "ndt_ec_extract", "ndt_ec_segment", "ndt_ec_segment_batch",
                  "ndt_ec_box_yaw", "ndt_ec_box_yaws"):
            getattr(L, n).restype = C.c_int
        L._ec_ready = True
    return L


def box_yaw(xyz):
    """Yaw quaternion (z, w) of one cluster's box (host code, no GPU): ndt_ec_box_yaw."""
    L = _lib()
    p = np.ascontiguousarray(xyz, np.float32).reshape(-1, 3)
    qz, qw = C.c_double(), C.c_double()
    rc = L.ndt_ec_box_yaw(p.ctypes.data, len(p), C.byref(qz), C.byref(qw))
    if rc != 0:
        raise _ndt.NdtError(f"ndt_ec_box_yaw: {_ndt.ERRORS.get(rc, rc)}")
    return qz.value, qw.value


def box_yaws(clusters):
    """Yaw quaternions (C x 2: z, w) of many clusters' boxes on the host's threads: ndt_ec_box_yaws."""
    L = _lib()
    parts = [np.ascontiguousarray(c, np.float32).reshape(-1, 3) for c in clusters]
    off = np.zeros(len(parts) + 1, np.int32)
    off[1:] = np.cumsum([len(c) for c in parts])
    xyz = np.concatenate(parts) if parts and off[-1] else np.zeros((1, 3), np.float32)
    qz, qw = np.zeros(max(len(parts), 1)), np.zeros(max(len(parts), 1))
    rc = L.ndt_ec_box_yaws(len(parts), xyz.ctypes.data, off.ctypes.data, qz.ctypes.data, qw.ctypes.data)
    if rc != 0:
        raise _ndt.NdtError(f"ndt_ec_box_yaws: {_ndt.ERRORS.get(rc, rc)}")
    return np.stack([qz[:len(parts)], qw[:len(parts)]], axis=1)


class EuclideanClusters:
    """A clustering handle on one GPU (stream and device buffers)."""

    def __init__(self, device=0):
        self.L = _lib()
        h = C.c_void_p()
        rc = self.L.ndt_ec_create(device, C.byref(h))
        if rc != 0:
            raise _ndt.NdtError(f"ndt_ec_create failed ({_ndt.ERRORS.get(rc, rc)})")
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.L.ndt_ec_destroy(self.h)
            self.h = None

    def __del__(self):  # pragma: no cover
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, rc, what):
        if rc != 0:
            raise _ndt.NdtError(f"{what}: {_ndt.ERRORS.get(rc, rc)}: {self.L.ndt_ec_last_error(self.h).decode()}")

    def labels(self, xyz, tolerance):
        """Smallest point index of each point's cluster."""
        p = np.ascontiguousarray(xyz, np.float32).reshape(-1, 3)
        out = np.zeros(max(len(p), 1), np.int32)
        self._check(self.L.ndt_ec_labels(self.h, p.ctypes.data, len(p), float(tolerance), out.ctypes.data),
                    "ndt_ec_labels")
        return out[:len(p)]

    def extract(self, xyz, tolerance, min_size=20, max_size=100000):
        """The reference's extract(): list of index arrays, in its order."""
        p = np.ascontiguousarray(xyz, np.float32).reshape(-1, 3)
        n = len(p)
        k = C.c_int()
        off = np.zeros(n + 2, np.int32)
        idx = np.zeros(max(n, 1), np.int32)
        self._check(self.L.ndt_ec_extract(self.h, p.ctypes.data, n, float(tolerance), int(min_size), int(max_size),
                                          C.byref(k), off.ctypes.data, idx.ctypes.data), "ndt_ec_extract")
        return [idx[off[c]:off[c + 1]].copy() for c in range(k.value)]

    def segment(self, xyz):
        """segmentByDistance: (clustered points (m, 3), boxes (b, 10), centroids (b, 3))."""
        p = np.ascontiguousarray(xyz, np.float32).reshape(-1, 3)
        n = len(p)
        pts = np.zeros((max(n, 1), 3), np.float32)
        boxes = np.zeros((max(n, 1), 10))
        cen = np.zeros((max(n, 1), 3))
        m, nb, nc = C.c_int(), C.c_int(), C.c_int()
        self._check(self.L.ndt_ec_segment(self.h, p.ctypes.data, n, pts.ctypes.data, C.byref(m), boxes.ctypes.data,
                                          C.byref(nb), cen.ctypes.data, C.byref(nc)), "ndt_ec_segment")
        return pts[:m.value], boxes[:nb.value], cen[:nc.value]

    def segment_batch(self, clouds):
        """segmentByDistance of several clouds, several per GPU pass: a list of (points, boxes, centroids)."""
        clouds = [np.ascontiguousarray(c, np.float32).reshape(-1, 3) for c in clouds]
        C_ = len(clouds)
        off = np.zeros(C_ + 1, np.int32)
        off[1:] = np.cumsum([len(c) for c in clouds])
        n = int(off[-1])
        xyz = np.concatenate(clouds) if n else np.zeros((1, 3), np.float32)
        pts = np.zeros((max(n, 1), 3), np.float32)
        boxes = np.zeros((max(n, 1), 10))
        cen = np.zeros((max(n, 1), 3))
        oo = np.zeros(C_ + 1, np.int32)
        bo = np.zeros(C_ + 1, np.int32)
        self._check(self.L.ndt_ec_segment_batch(self.h, C_, xyz.ctypes.data, off.ctypes.data, pts.ctypes.data,
                                                oo.ctypes.data, boxes.ctypes.data, bo.ctypes.data, cen.ctypes.data),
                    "ndt_ec_segment_batch")
        return [(pts[oo[c]:oo[c + 1]], boxes[bo[c]:bo[c + 1]], cen[bo[c]:bo[c + 1]]) for c in range(C_)]
